"""Multi-rank halo path on CPU: two gloo ranks each own a t slab, run
TSlabDslash (face pack -> exchange -> body without the slab-crossing hops ->
face unpack) with the oracle as the compute kernels, and must reproduce the
oracle applied to the whole lattice, for every family, kernel and sign, with
twisted boundary phases in t and an antiperiodic time boundary."""
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
from qphix_b200.halo import TComm, TSlabDslash, local_geometry
from qphix_b200.lattice import F64, Geometry


class OracleKernels:
    """TSlabDslash compute steps on the CPU oracle (float64 torch tensors)."""

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


def _fields(G, cb):
    U = fields.random_gauge(G, seed=11)
    psi = fields.random_spinor(G, seed=12)
    chi = fields.random_spinor(G, seed=13)
    A = fields.random_clover(G, seed=14)
    F = fields.random_full_clover(G, seed=15)
    return U, psi, chi, A, F


def _worker(rank, world, port, results):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        G = Geometry(4, 4, 4, 8, soalen=2, veclen=4, ftype=F64, compress12=True, t_boundary=-1.0)
        g = local_geometry(G, rank, world)
        cb = 1
        U, psi, chi, A, F = _fields(G, cb)
        t0, nt = rank * g.nt, g.nt
        sl = slice(t0, t0 + nt)
        loc = {
            "psi": layout.pack_spinor(g, psi[sl]), "chi": layout.pack_spinor(g, chi[sl]),
            "gauge": layout.pack_gauge(g, U, cb, t0=t0), "clover": layout.pack_clover(g, A[sl]),
            "fclover": layout.pack_full_clover(g, F[sl]),
        }
        op = TSlabDslash(g, TComm(), OracleKernels())
        errs = {}
        for fam in H.FAMILIES:
            for kernel in H.KERNELS:
                for isign in (1, -1):
                    pp = H.op_params(fam, kernel, tbc_mask=9)
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


def test_two_rank_t_slabs_match_global_oracle():
    world = 2
    mgr = mp.Manager()
    results = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), results), nprocs=world, start_method="spawn")
    G = Geometry(4, 4, 4, 8, soalen=2, veclen=4, ftype=F64, compress12=True, t_boundary=-1.0)
    cb = 1
    U, psi, chi, A, F = _fields(G, cb)
    glob = {"psi": layout.pack_spinor(G, psi).numpy(), "chi": layout.pack_spinor(G, chi).numpy(),
            "gauge": layout.pack_gauge(G, U, cb).numpy(), "clover": layout.pack_clover(G, A).numpy(),
            "fclover": layout.pack_full_clover(G, F).numpy()}
    for fam in H.FAMILIES:
        for kernel in H.KERNELS:
            for isign in (1, -1):
                pp = H.op_params(fam, kernel, tbc_mask=9)
                prm = O.make_params(**pp)
                ref = O.dslash(G, fam, kernel, isign, cb, glob["psi"], glob["gauge"], chi=glob["chi"],
                               clover=glob["fclover" if fam == "tm_clover" else "clover"], params=prm)
                ref_c = layout.unpack_spinor(G, torch.from_numpy(ref))
                for rank in range(world):
                    g = local_geometry(G, rank, world)
                    got = layout.unpack_spinor(g, torch.from_numpy(results[rank][(fam, kernel, isign)]))
                    exp = ref_c[rank * g.nt:(rank + 1) * g.nt]
                    err = float((got - exp).abs().max())
                    assert err < 1e-12, (fam, kernel, isign, rank, err)
