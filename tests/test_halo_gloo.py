"""Multi-rank halo path on CPU: gloo ranks each own a block of the lattice
-- two ranks on t slabs, four ranks on a 2 x 2 grid of z x t blocks -- run
HaloDslash (face pack -> exchange -> body without the block-crossing hops ->
face unpack) with the oracle as the compute kernels, and must reproduce the
oracle applied to the whole lattice, for every family, kernel and sign, with
twisted boundary phases in z and t and an antiperiodic time boundary.  The
block CG (TSlabEvenOdd + cg, inner products all-reduced) must solve the
whole lattice's even-odd system to 1e-10 for every family."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import helpers as H
import oracle as O
from qphix_b200 import fields, layout
from qphix_b200.halo import GridComm, HaloDslash, TSlabEvenOdd, cg, grid_geometry
from qphix_b200.lattice import F64, Geometry


class OracleKernels:
    """HaloDslash compute steps on the CPU oracle (float64 torch tensors)."""

    def alloc(self, n):
        return torch.zeros(n, dtype=torch.float64)

    def body(self, g, family, kernel, isign, cb, psi, out, gauge, accumulate=None, **kw):
        prm = O.make_params(coeff_s=kw["coeff_s"], coeff_t_f=kw["coeff_t_f"], coeff_t_b=kw["coeff_t_b"],
                            alpha=kw["alpha"], mu=kw["mu"], muinv=kw["muinv"], rho=kw["rho"],
                            tbc_mask=kw["tbc_mask"], tbc_phases=kw["tbc_phases"], accumulate=accumulate)
        chi = kw["chi"].numpy() if kw["chi"] is not None else None
        cl = kw["clover"].numpy() if kw["clover"] is not None else None
        O.dslash(g, family, kernel, isign, cb, psi.numpy(), gauge.numpy(), chi=chi, clover=cl, params=prm,
                 out=out.numpy())

    def pack(self, g, isign, psi_cb, psi, buf, dir):
        buf.numpy()[:] = O.face_pack(g, isign, psi_cb, psi.numpy(), dir)

    def unpack(self, g, family, isign, cb, buf, gauge, out, dir, **kw):
        cl = kw.pop("clover")
        O.face_unpack(g, family, isign, cb, buf.numpy(), gauge.numpy(), out.numpy(), dir,
                      clover=cl.numpy() if cl is not None else None, **kw)

    def axpby(self, a, x, b, y):
        y.mul_(b).add_(x, alpha=a)

    def dot(self, x, y):
        return float(torch.dot(x, y))


def _fields(G, cb):
    U = fields.random_gauge(G, seed=11)
    psi = fields.random_spinor(G, seed=12)
    chi = fields.random_spinor(G, seed=13)
    A = fields.random_clover(G, seed=14)
    F = fields.random_full_clover(G, seed=15)
    return U, psi, chi, A, F


def _block(G, rank, pz, pt):
    """local geometry of rank and its slices (t slice, z slice, t0, z0)"""
    g = grid_geometry(G, rank, pz, pt)
    z0, t0 = (rank % pz) * g.nz, (rank // pz) * g.nt
    return g, slice(t0, t0 + g.nt), slice(z0, z0 + g.nz), t0, z0


def _worker(rank, world, port, results, G, pz, tbc):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g, ts, zs, t0, z0 = _block(G, rank, pz, world // pz)
        cb = 1
        U, psi, chi, A, F = _fields(G, cb)
        loc = {
            "psi": layout.pack_spinor(g, psi[ts, zs]), "chi": layout.pack_spinor(g, chi[ts, zs]),
            "gauge": layout.pack_gauge(g, U, cb, t0=t0, z0=z0), "clover": layout.pack_clover(g, A[ts, zs]),
            "fclover": layout.pack_full_clover(g, F[ts, zs]),
        }
        op = HaloDslash(g, GridComm(pz), OracleKernels())
        errs = {}
        for fam in H.FAMILIES:
            for kernel in H.KERNELS:
                for isign in (1, -1):
                    pp = H.op_params(fam, kernel, tbc_mask=tbc)
                    pp.pop("accumulate")
                    out = torch.zeros_like(loc["psi"])
                    op.apply(fam, kernel, isign, cb, loc["psi"], out, loc["gauge"], chi=loc["chi"],
                             clover=loc["fclover" if fam == "tm_clover" else "clover"], **pp)
                    errs[(fam, kernel, isign)] = out.numpy()
        results[rank] = errs
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _check_blocks(world, pz, G, tbc):
    mgr = mp.Manager()
    results = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), results, G, pz, tbc), nprocs=world, start_method="spawn")
    cb = 1
    U, psi, chi, A, F = _fields(G, cb)
    glob = {"psi": layout.pack_spinor(G, psi).numpy(), "chi": layout.pack_spinor(G, chi).numpy(),
            "gauge": layout.pack_gauge(G, U, cb).numpy(), "clover": layout.pack_clover(G, A).numpy(),
            "fclover": layout.pack_full_clover(G, F).numpy()}
    for fam in H.FAMILIES:
        for kernel in H.KERNELS:
            for isign in (1, -1):
                pp = H.op_params(fam, kernel, tbc_mask=tbc)
                prm = O.make_params(**pp)
                ref = O.dslash(G, fam, kernel, isign, cb, glob["psi"], glob["gauge"], chi=glob["chi"],
                               clover=glob["fclover" if fam == "tm_clover" else "clover"], params=prm)
                ref_c = layout.unpack_spinor(G, torch.from_numpy(ref))
                for rank in range(world):
                    g, ts, zs, _, _ = _block(G, rank, pz, world // pz)
                    got = layout.unpack_spinor(g, torch.from_numpy(results[rank][(fam, kernel, isign)]))
                    exp = ref_c[ts, zs]
                    err = float((got - exp).abs().max())
                    assert err < 1e-12, (fam, kernel, isign, rank, err)


def test_two_rank_t_slabs_match_global_oracle():
    _check_blocks(2, 1, Geometry(4, 4, 4, 8, soalen=2, veclen=4, ftype=F64, compress12=True, t_boundary=-1.0), 9)


def test_four_rank_z_t_grid_matches_global_oracle():
    # 2 x 2 blocks of 4^4 sites; twisted phases in x, z and t (mask 13)
    _check_blocks(4, 2, Geometry(4, 4, 8, 8, soalen=2, veclen=4, ftype=F64, compress12=True, t_boundary=-1.0), 13)


EO_G = dict(nx=4, ny=4, nz=4, nt=8, soalen=2, veclen=4, ftype=F64, compress12=True, t_boundary=-1.0)


def _eo_canonical(G, family, seed=900, target_cb=1):
    """The canonical fields behind helpers.eo_setup (same seeds): links,
    per-checkerboard clover terms (A on the target, A^-1 on the other) and
    their adjoints, and the source on the target checkerboard."""
    other = 1 - target_cb
    c = {"U": fields.random_gauge(G, seed=seed), "clov": [None, None], "clov_dag": [None, None],
         "b": fields.random_spinor(G, seed=seed + 3)}
    if family == "clover":
        c["clov"][target_cb] = fields.random_clover(G, seed=seed + 1)
        c["clov"][other] = fields.invert_blocks(fields.random_clover(G, seed=seed + 2))
    if family == "tm_clover":
        c["clov"][target_cb] = fields.random_full_clover(G, seed=seed + 1)
        c["clov"][other] = fields.invert_blocks(fields.random_full_clover(G, seed=seed + 2))
        c["clov_dag"] = [m.conj().transpose(-1, -2) for m in c["clov"]]
    return c


def _cg_worker(rank, world, port, results, geo, pz):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        G = Geometry(**geo)
        g, ts, zs, t0, z0 = _block(G, rank, pz, world // pz)
        out = {}
        for fam in H.FAMILIES:
            _, p = H.eo_setup(G, fam)
            c = _eo_canonical(G, fam)
            pack = layout.pack_full_clover if fam == "tm_clover" else layout.pack_clover
            cl = [pack(g, m[ts, zs]) if m is not None else None for m in c["clov"]]
            cld = [pack(g, m[ts, zs]) if m is not None else None for m in c["clov_dag"]]
            gauge = [layout.pack_gauge(g, c["U"], cb, t0=t0, z0=z0) for cb in (0, 1)]
            op = TSlabEvenOdd(HaloDslash(g, GridComm(pz), OracleKernels()), fam, gauge, clov=cl, clov_dag=cld,
                              target_cb=1, **p)
            x, info = cg(op, layout.pack_spinor(g, c["b"][ts, zs]), tol=1e-11, max_iter=500)
            out[fam] = (x.numpy(), info)
        results[rank] = out
    finally:
        dist.destroy_process_group()


def _check_cg(world, pz, geo):
    mgr = mp.Manager()
    results = mgr.dict()
    mp.start_processes(_cg_worker, args=(world, _free_port(), results, geo, pz), nprocs=world,
                       start_method="spawn")
    G = Geometry(**geo)
    for fam in H.FAMILIES:
        f, p = H.eo_setup(G, fam)
        full = torch.zeros(G.nt, G.nz, G.ny, G.nxh, 4, 3, dtype=torch.complex128)
        infos = []
        for rank in range(world):
            x, info = results[rank][fam]
            g, ts, zs, _, _ = _block(G, rank, pz, world // pz)
            full[ts, zs] = layout.unpack_spinor(g, torch.from_numpy(x))
            infos.append(info)
        # the ranks leave the loop together with the same global residual
        assert all(i["iters"] == infos[0]["iters"] > 0 for i in infos), (fam, infos)
        assert all(abs(i["rel_res"] - infos[0]["rel_res"]) <= 1e-15 for i in infos), (fam, infos)
        x = layout.pack_spinor(G, full).numpy()
        mx = H.oracle_schur(G, fam, f, p, x)
        rel = float(np.linalg.norm(f["b"] - mx) / np.linalg.norm(f["b"]))
        assert rel <= 1e-10, (fam, rel, infos[0])
        assert abs(rel - infos[0]["rel_res"]) <= 1e-12, (fam, rel, infos[0])


def test_two_rank_slab_cg_solves_global_system():
    _check_cg(2, 1, EO_G)


def test_four_rank_grid_cg_solves_global_system():
    _check_cg(4, 2, dict(EO_G, nz=8))
