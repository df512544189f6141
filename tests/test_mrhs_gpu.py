"""Multi-RHS kernels: layout round trip, the multi-RHS dslash against the
single-RHS kernel for every right-hand side, multi-RHS CG, and the
FP16-storage multi-RHS mixed-precision solve to 1e-10 (checked with the
oracle's FP64 operator)."""
import numpy as np
import pytest
import torch

import helpers as H
from qphix_b200 import mrhs, ops
from qphix_b200.lattice import F16, F32, F64, Geometry
from qphix_b200.solver import EvenOddOperator

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("soa,vec,ft,nrhs,ny", [
    (4, 16, F32, 4, 8), (8, 8, F32, 8, 8), (16, 16, F16, 16, 8), (8, 8, F16, 2, 8), (4, 4, F32, 1, 8),
    (16, 16, F32, 2, 8), (4, 8, F16, 8, 8),
    # FP16 with VECLEN == SOALEN: the kernel with the next hop's copies in flight,
    # one to four blocks per warp, and planes that end inside a warp (ny = 6)
    (4, 4, F16, 4, 8), (8, 8, F16, 8, 8), (16, 16, F16, 4, 8), (4, 4, F16, 8, 6), (4, 4, F16, 4, 6)])
def test_mrhs_dslash_matches_single(cuda, soa, vec, ft, nrhs, ny):
    g = Geometry(max(8, 2 * soa), ny, 4, 4, soalen=soa, veclen=vec, ftype=ft, compress12=True, t_boundary=-1.0)
    f = H.make_fields(g, cb=0, seed=61)
    T = lambda a: H.to_torch(a, cuda)
    gauge = T(f["gauge"])
    psis = [T(H.make_fields(g, cb=0, seed=70 + r)["psi"]) for r in range(nrhs)]
    chis = [T(H.make_fields(g, cb=0, seed=90 + r)["chi"]) for r in range(nrhs)]
    mp, mc = mrhs.pack(g, psis), mrhs.pack(g, chis)
    back = mrhs.unpack(g, mp, nrhs)
    assert all(torch.equal(a, b) for a, b in zip(back, psis))
    for fam in H.FAMILIES:
        cl = T(f["fclover" if fam == "tm_clover" else "clover"])
        for kernel in H.KERNELS:
            for isign in (1, -1):
                pp = H.op_params(fam, kernel, tbc_mask=5)
                acc = pp.pop("accumulate")
                out = torch.zeros_like(mp)
                mrhs.dslash(g, nrhs, fam, kernel, isign, 0, mp, out, gauge, chi=mc, clover=cl, accumulate=acc, **pp)
                outs = mrhs.unpack(g, out, nrhs)
                for r in range(nrhs):
                    ref = torch.zeros_like(psis[r])
                    ops.dslash(g, fam, kernel, isign, 0, psis[r], ref, gauge, chi=chis[r], clover=cl, **pp)
                    assert torch.equal(outs[r], ref), (fam, kernel, isign, r)


def _ops(g, family, f, p, dev, dtype=None):
    T = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    conv = (lambda t: t) if dtype is None else (lambda t: None if t is None else t.to(dtype))
    return EvenOddOperator(g, family, gauge=[conv(T(x)) for x in f["gauge"]], clov=[conv(T(x)) for x in f["clov"]],
                           clov_dag=[conv(T(x)) for x in f["clov_dag"]], target_cb=1, **p)


def test_mrhs_cg_and_mixed_fp16(cuda):
    family = "clover"
    g = Geometry(8, 8, 8, 8, soalen=4, veclen=8, ftype=F64, compress12=True, t_boundary=-1.0)
    f, p = H.eo_setup(g, family)
    op64 = _ops(g, family, f, p, cuda)
    nrhs = 4
    rng = np.random.default_rng(8)
    bs = [torch.from_numpy(rng.normal(size=g.spinor_elems)).to(cuda) for _ in range(nrhs)]
    # FP32 multi-RHS CG
    g32 = g.with_(ftype=F32)
    op32 = _ops(g32, family, f, p, cuda, dtype=torch.float32)
    b32 = mrhs.pack(g32, [b.float() for b in bs])
    x32, info = mrhs.cg(op32, nrhs, b32, tol=1e-5, max_iter=1000)
    assert max(info["rel_res"]) < 1e-5, info
    # FP16 multi-RHS corrections of FP64 solutions
    g16 = g.with_(ftype=F16)
    op16 = _ops(g16, family, f, p, cuda, dtype=torch.float16)
    xs, info = mrhs.mixed_solve(op64, op16, bs, tol=1e-10, inner_tol=1e-2)
    assert max(info["rel_res"]) <= 1e-10, info
    for b, x in zip(bs, xs):
        ff = dict(f, b=b.cpu().numpy())
        mx = H.oracle_schur(g, family, ff, p, x.cpu().numpy())
        assert np.linalg.norm(ff["b"] - mx) / np.linalg.norm(ff["b"]) < 2e-10
    print(info)


@pytest.mark.parametrize("lo,nrhs", [(F16, 4), (F16, 8), (F32, 2)])
@pytest.mark.parametrize("family", ["clover", "tm"])
def test_mrhs_reliable_updates(cuda, lo, nrhs, family):
    """Multi-RHS CG with FP64 reliable updates: every solution to 1e-10
    against the oracle, in no more iterations than defect correction."""
    g = Geometry(8, 8, 8, 8, soalen=4, veclen=8, ftype=F64, compress12=True, t_boundary=-1.0)
    f, p = H.eo_setup(g, family)
    op64 = _ops(g, family, f, p, cuda)
    glo = g.with_(ftype=lo)
    oplo = _ops(glo, family, f, p, cuda, dtype=glo.dtype)
    rng = np.random.default_rng(9 + nrhs)
    bs = [torch.from_numpy(rng.normal(size=g.spinor_elems)).to(cuda) for _ in range(nrhs)]
    xs, info = mrhs.mixed_solve(op64, oplo, bs, tol=1e-10, inner_tol=1e-2, solver="cg_reliable")
    assert max(info["rel_res"]) <= 1e-10, info
    for b, x in zip(bs, xs):
        ff = dict(f, b=b.cpu().numpy())
        mx = H.oracle_schur(g, family, ff, p, x.cpu().numpy())
        assert np.linalg.norm(ff["b"] - mx) / np.linalg.norm(ff["b"]) < 2e-10
    _, dc = mrhs.mixed_solve(op64, oplo, bs, tol=1e-10, inner_tol=1e-2)
    assert info["inner_iters"] <= dc["inner_iters"] + 5, (info, dc)


@pytest.mark.parametrize("solver", ["cg_reliable", "cg"])
def test_mrhs_zero_source(cuda, solver):
    """One zero source among eight: its solution stays exactly zero and the
    other seven still reach 1e-10 (a zero residual must not turn the
    recurrence coefficients into 0/0)."""
    family, nrhs = "clover", 8
    g = Geometry(8, 8, 8, 8, soalen=4, veclen=8, ftype=F64, compress12=True, t_boundary=-1.0)
    f, p = H.eo_setup(g, family)
    op64 = _ops(g, family, f, p, cuda)
    g16 = g.with_(ftype=F16)
    op16 = _ops(g16, family, f, p, cuda, dtype=torch.float16)
    rng = np.random.default_rng(31)
    bs = [torch.from_numpy(rng.normal(size=g.spinor_elems)).to(cuda) for _ in range(nrhs)]
    bs[3] = torch.zeros_like(bs[3])
    xs, info = mrhs.mixed_solve(op64, op16, bs, tol=1e-10, inner_tol=1e-2, solver=solver)
    assert all(np.isfinite(info["rel_res"])), info
    assert max(info["rel_res"]) <= 1e-10, info
    assert torch.count_nonzero(xs[3]) == 0
    for i, (b, x) in enumerate(zip(bs, xs)):
        if i == 3:
            continue
        ff = dict(f, b=b.cpu().numpy())
        mx = H.oracle_schur(g, family, ff, p, x.cpu().numpy())
        assert np.linalg.norm(ff["b"] - mx) / np.linalg.norm(ff["b"]) < 2e-10
