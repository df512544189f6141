"""GPU face kernels against the FP64 oracle (unrounded results, tolerances
helpers.TOL), and the t-slab decomposition (body without slab-crossing hops +
face pack/exchange/unpack) emulated on one GPU against the full-lattice
kernel."""
import numpy as np
import pytest
import torch

import helpers as H
import oracle as O
from qphix_b200 import fields, layout, ops
from qphix_b200.halo import GPUKernels, face_kind, local_geometry
from qphix_b200.lattice import BF16, F16, F16N, F32, F64, FTYPE_NAMES, Geometry

pytestmark = pytest.mark.gpu
TOL = H.TOL
LAYOUTS = [(1, 1, F32), (4, 16, F32), (16, 16, F32), (2, 4, F64), (8, 8, F16), (8, 8, F16N), (4, 16, BF16)]


def _face_values(g, buf):
    """decoded face values (n, 12) as float64"""
    b = buf.detach().cpu()
    if g.ftype == F16N:
        r = b.reshape(-1, 14)
        return (r[:, :12].double() * r[:, 12:].contiguous().view(torch.float32).double()).numpy()
    return b.double().reshape(-1, 12).numpy()


@pytest.mark.parametrize("soa,vec,ft", LAYOUTS)
def test_face_pack(cuda, soa, vec, ft):
    g = Geometry(max(4, 2 * soa), 8, 4, 6, soalen=soa, veclen=vec, ftype=ft)
    f = H.make_fields(g, cb=0, seed=31)
    psi = H.to_torch(f["psi"], cuda)
    for d in range(8):
        for isign in (1, -1):
            buf = torch.zeros(g.face_elems * g.face_sites(d), dtype=g.dtype, device=cuda)
            ops.face_pack(g, isign, 1, psi, buf, d)
            ref = O.face_pack(g, isign, 1, f["psi"], d, fp64_out=True)
            e = H.record("face pack %s soa%d" % (FTYPE_NAMES[ft], soa), H.face_rel_err(_face_values(g, buf), ref),
                         TOL[ft])
            assert e < TOL[ft], (d, isign, e)


@pytest.mark.parametrize("soa,vec,ft", LAYOUTS)
def test_face_unpack(cuda, soa, vec, ft):
    g = Geometry(max(4, 2 * soa), 8, 4, 6, soalen=soa, veclen=vec, ftype=ft, compress12=(soa % 2 == 0))
    f = H.make_fields(g, cb=0, seed=32)
    rng = np.random.default_rng(5)
    for fam in H.FAMILIES:
        cl_np = f["fclover" if fam == "tm_clover" else "clover"]
        cl = H.to_torch(cl_np, cuda)
        gauge = H.to_torch(f["gauge"], cuda)
        for d in range(8):
            for isign in (1, -1):
                n = g.face_sites(d)
                # a face buffer in the storage format: pack a random spinor's face
                src = H.make_fields(g, cb=1, seed=40 + d)["psi"]
                inbuf_np = O.face_pack(g, isign, 1, src, d ^ 1)
                pp = H.op_params(fam, "dslash")
                tbc = (d + isign) % 3 == 0
                out = H.to_torch(f["chi"], cuda)
                ops.face_unpack(g, fam, isign, 0, H.to_torch(inbuf_np, cuda), gauge, out, d, beta=0.41,
                                clover=cl, mu=pp["mu"], muinv=pp["muinv"], tbc=tbc, tbc_phases=pp["tbc_phases"])
                ref = O.face_unpack(g, fam, isign, 0, inbuf_np, f["gauge"], H.as_f64(g, f["chi"]), d, beta=0.41,
                                    clover=cl_np, mu=pp["mu"], muinv=pp["muinv"], tbc=tbc,
                                    tbc_phases=pp["tbc_phases"], fp64_out=True)
                assert n * g.face_elems == inbuf_np.size
                e = H.site_rel_err(g, H.to_np(out), ref, g.with_(ftype=F64))
                H.record("face unpack %s soa%d" % (FTYPE_NAMES[ft], soa), e, TOL[ft])
                assert e < TOL[ft], (fam, d, isign, e)


@pytest.mark.parametrize("ft", [F32, F64])
def test_two_slab_decomposition_on_one_gpu(cuda, ft):
    """Two t slabs driven on one device: pack both, swap the face buffers,
    then interior + unpack per slab; must equal the undecomposed operator."""
    G = Geometry(8, 8, 4, 8, soalen=4, veclen=8, ftype=ft, compress12=True, t_boundary=-1.0)
    cb = 0
    U = fields.random_gauge(G, seed=41)
    psi, chi = fields.random_spinor(G, seed=42), fields.random_spinor(G, seed=43)
    A, F = fields.random_clover(G, seed=44), fields.random_full_clover(G, seed=45)
    D = lambda t: t.to(cuda)
    full = {"psi": D(layout.pack_spinor(G, psi)), "chi": D(layout.pack_spinor(G, chi)),
            "gauge": D(layout.pack_gauge(G, U, cb)), "clover": D(layout.pack_clover(G, A)),
            "fclover": D(layout.pack_full_clover(G, F))}
    slabs = []
    for r in range(2):
        g = local_geometry(G, r, 2)
        sl = slice(r * g.nt, (r + 1) * g.nt)
        slabs.append((g, {"psi": D(layout.pack_spinor(g, psi[sl])), "chi": D(layout.pack_spinor(g, chi[sl])),
                          "gauge": D(layout.pack_gauge(g, U, cb, t0=r * g.nt)),
                          "clover": D(layout.pack_clover(g, A[sl])), "fclover": D(layout.pack_full_clover(g, F[sl]))}))
    K = GPUKernels(G.dtype, cuda)
    for fam in H.FAMILIES:
        for kernel in H.KERNELS:
            for isign in (1, -1):
                pp = H.op_params(fam, kernel, tbc_mask=8)
                pp.pop("accumulate")
                clk = "fclover" if fam == "tm_clover" else "clover"
                ref = torch.zeros_like(full["psi"])
                ops.dslash(G, fam, kernel, isign, cb, full["psi"], ref, full["gauge"], chi=full["chi"],
                           clover=full[clk], **pp)
                ref_c = layout.unpack_spinor(G, ref.cpu())
                # face buffers: [rank] -> (to forward, to backward)
                sends = []
                for g, f in slabs:
                    n = g.face_sites(6)
                    bf, bb = K.alloc(12 * n), K.alloc(12 * n)
                    K.pack(g, isign, 1 - cb, f["psi"], bf, 7)
                    K.pack(g, isign, 1 - cb, f["psi"], bb, 6)
                    sends.append((bf, bb))
                kind, sg = face_kind(fam, kernel)
                for r, (g, f) in enumerate(slabs):
                    out = torch.zeros_like(f["psi"])
                    K.body(g, fam, kernel, isign, cb, f["psi"], out, f["gauge"], accumulate=[1] * 6 + [0, 0],
                           chi=f["chi"], clover=f[clk], **pp)
                    from_back = sends[(r - 1) % 2][0]
                    from_fwd = sends[(r + 1) % 2][1]
                    bb = sg * pp["coeff_t_b"] * (G.t_boundary if g.t_edge_lo else 1.0)
                    bfw = sg * pp["coeff_t_f"] * (G.t_boundary if g.t_edge_hi else 1.0)
                    cl = f[clk] if kind in ("clover", "tm_clover") else None
                    K.unpack(g, kind, isign, cb, from_back, f["gauge"], out, 6, beta=bb, clover=cl, mu=pp["mu"],
                             muinv=pp["muinv"], tbc=True, tbc_phases=pp["tbc_phases"])
                    K.unpack(g, kind, isign, cb, from_fwd, f["gauge"], out, 7, beta=bfw, clover=cl, mu=pp["mu"],
                             muinv=pp["muinv"], tbc=True, tbc_phases=pp["tbc_phases"])
                    got = layout.unpack_spinor(g, out.cpu())
                    exp = ref_c[r * g.nt:(r + 1) * g.nt]
                    err = float((got - exp).abs().max() / exp.abs().max())
                    H.record("two t slabs vs whole lattice %s" % FTYPE_NAMES[ft], err, TOL[ft])
                    assert err < TOL[ft], (fam, kernel, isign, r, err)
