"""BLAS with FP64 reductions, the even-odd operator and the solvers on the
GPU.  The operator is checked against the oracle; solutions are checked with
the oracle's FP64 operator (true residual |b - Mhat x| / |b| <= 1e-10)."""
import numpy as np
import pytest
import torch

import helpers as H
from qphix_b200 import _lib, layout
from qphix_b200.lattice import BF16, F16, F16N, F32, F64, Geometry
from qphix_b200.solver import EvenOddOperator, mixed_solve

pytestmark = pytest.mark.gpu


def _op(g, family, f, p, dev, dtype=None):
    T = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    conv = (lambda t: t) if dtype is None else (lambda t: None if t is None else t.to(dtype))
    return EvenOddOperator(g, family, gauge=[conv(T(x)) for x in f["gauge"]], clov=[conv(T(x)) for x in f["clov"]],
                           clov_dag=[conv(T(x)) for x in f["clov_dag"]], target_cb=1, **p)


def _true_res(g, family, f, p, x):
    mx = H.oracle_schur(g, family, f, p, x.astype(np.float64))
    b = f["b"].astype(np.float64)
    return float(np.linalg.norm(b - mx) / np.linalg.norm(b))


def test_blas(cuda):
    L = _lib.lib()
    g = Geometry(8, 8, 4, 4, soalen=4, veclen=8, ftype=F64)
    n = g.spinor_elems
    x = torch.randn(n, dtype=torch.float64, device=cuda)
    y = torch.randn(n, dtype=torch.float64, device=cuda)
    part = torch.zeros(L.qb200_blas_partials_len(), dtype=torch.float64, device=cuda)
    res = torch.zeros(2, dtype=torch.float64, device=cuda)
    st = None
    _lib.check(L.qb200_blas_dot(1, n, x.data_ptr(), y.data_ptr(), res.data_ptr(), part.data_ptr(), st))
    torch.cuda.synchronize()
    assert abs(res[0].item() - float((x * y).sum())) < 1e-9 * n
    y0 = y.clone()
    _lib.check(L.qb200_blas_axpby(1, n, 0.5, x.data_ptr(), -2.0, y.data_ptr(), st))
    torch.cuda.synchronize()
    assert torch.allclose(y, 0.5 * x - 2.0 * y0, rtol=0, atol=1e-13)
    # complex dot on the spinor layout vs the canonical complex vectors
    _lib.check(L.qb200_blas_cdot(g.c_struct(), x.data_ptr(), y.data_ptr(), res.data_ptr(), part.data_ptr(), st))
    torch.cuda.synchronize()
    cx, cy = layout.unpack_spinor(g, x.cpu()), layout.unpack_spinor(g, y.cpu())
    ref = complex((cx.conj() * cy).sum())
    assert abs(res[0].item() - ref.real) < 1e-9 and abs(res[1].item() - ref.imag) < 1e-9
    # conversion to half and back
    h = torch.zeros(n, dtype=torch.float16, device=cuda)
    _lib.check(L.qb200_blas_convert(2, h.data_ptr(), 1, x.data_ptr(), n, 0.25, st))
    torch.cuda.synchronize()
    assert torch.allclose(h.double(), 0.25 * x, rtol=1e-3, atol=1e-4)


@pytest.mark.parametrize("family", ["wilson", "clover", "tm", "tm_clover"])
@pytest.mark.parametrize("isign", [1, -1])
def test_schur_operator_vs_oracle(cuda, family, isign):
    g = Geometry(8, 8, 4, 4, soalen=4, veclen=8, ftype=F64, compress12=True, t_boundary=-1.0)
    f, p = H.eo_setup(g, family)
    op = _op(g, family, f, p, cuda)
    out = op.apply(torch.from_numpy(f["b"]).to(cuda), isign=isign)
    ref = H.oracle_schur(g, family, f, p, f["b"], isign=isign)
    assert H.site_rel_err(g, out.cpu().numpy(), ref) < 1e-12


@pytest.mark.parametrize("family", ["wilson", "clover", "tm", "tm_clover"])
def test_dagger_is_adjoint(cuda, family):
    g = Geometry(8, 8, 4, 4, soalen=4, veclen=8, ftype=F64, t_boundary=-1.0)
    f, p = H.eo_setup(g, family)
    op = _op(g, family, f, p, cuda)
    rng = np.random.default_rng(3)
    a = torch.from_numpy(rng.normal(size=g.spinor_elems)).to(cuda)
    b = torch.from_numpy(f["b"]).to(cuda)
    Ma = op.apply(a, 1)
    Mdb = op.apply(b, -1)
    lhs = complex((layout.unpack_spinor(g, b.cpu()).conj() * layout.unpack_spinor(g, Ma.cpu())).sum())
    rhs = complex((layout.unpack_spinor(g, Mdb.cpu()).conj() * layout.unpack_spinor(g, a.cpu())).sum())
    assert abs(lhs - rhs) < 1e-10 * abs(lhs)


@pytest.mark.parametrize("family", ["wilson", "clover", "tm", "tm_clover"])
def test_cg_and_bicgstab_fp64(cuda, family):
    g = Geometry(8, 8, 8, 8, soalen=4, veclen=8, ftype=F64, compress12=True, t_boundary=-1.0)
    f, p = H.eo_setup(g, family)
    op = _op(g, family, f, p, cuda)
    b = torch.from_numpy(f["b"]).to(cuda)
    x, info = op.cg(b, tol=1e-11, max_iter=2000)
    assert info["rel_res"] < 1e-10, info
    assert _true_res(g, family, f, p, x.cpu().numpy()) < 1e-10
    x2, info2 = op.bicgstab(b, tol=1e-11, max_iter=2000)
    assert info2["rel_res"] < 1e-10, info2
    assert _true_res(g, family, f, p, x2.cpu().numpy()) < 1e-10


@pytest.mark.parametrize("lo", [F32, F16, F16N, BF16])
@pytest.mark.parametrize("solver", ["cg", "bicgstab", "cg_reliable"])
def test_mixed_precision_reaches_1e10(cuda, lo, solver):
    family = "clover"
    g = Geometry(8, 8, 8, 8, soalen=4, veclen=8, ftype=F64, compress12=True, t_boundary=-1.0)
    f, p = H.eo_setup(g, family)
    op64 = _op(g, family, f, p, cuda)
    glo = g.with_(ftype=lo)
    oplo = _op(glo, family, f, p, cuda, dtype=glo.dtype)   # links / clover in the low type
    b = torch.from_numpy(f["b"]).to(cuda)
    inner = (1e-4 if lo == F32 else 1e-2) if solver != "cg_reliable" else (1e-3 if lo == F32 else 0.1)
    x, info = mixed_solve(op64, oplo, b, solver=solver, tol=1e-10, inner_tol=inner)
    assert info["rel_res"] <= 1e-10, info
    assert _true_res(g, family, f, p, x.cpu().numpy()) < 2e-10
    print(solver, lo, info)


@pytest.mark.parametrize("family", ["clover", "tm_clover"])
def test_slab_cg_single_rank(cuda, family):
    """halo.cg over TSlabEvenOdd with the GPU kernels and the library's FP64
    BLAS (one rank: no exchange) solves the even-odd system to 1e-10."""
    from qphix_b200.halo import GPUKernels, TComm, TSlabDslash, TSlabEvenOdd, cg
    g = Geometry(8, 8, 8, 8, soalen=4, veclen=8, ftype=F64, compress12=True, t_boundary=-1.0)
    f, p = H.eo_setup(g, family)
    T = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(cuda)
    op = TSlabEvenOdd(TSlabDslash(g, TComm(), GPUKernels(torch.float64, cuda)), family,
                      [T(x) for x in f["gauge"]], clov=[T(x) for x in f["clov"]],
                      clov_dag=[T(x) for x in f["clov_dag"]], target_cb=1, **p)
    b = T(f["b"])
    x, info = cg(op, b, tol=1e-11, max_iter=2000)
    assert info["rel_res"] <= 1e-10, info
    assert _true_res(g, family, f, p, x.cpu().numpy()) < 1e-10
    # same iterate count as the library's CG on the same system
    x2, info2 = _op(g, family, f, p, cuda).cg(b, tol=1e-11, max_iter=2000)
    assert abs(info["iters"] - info2["iters"]) <= 2, (info, info2)


@pytest.mark.parametrize("family", ["wilson", "tm", "tm_clover"])
def test_reliable_updates_fp16n(cuda, family):
    """CG with FP64 reliable updates on FP16 + norm storage for the other
    families: 1e-10 against the oracle, and no more iterations than defect
    correction needs."""
    g = Geometry(16, 8, 8, 8, soalen=8, veclen=8, ftype=F64, compress12=True, t_boundary=-1.0)
    f, p = H.eo_setup(g, family)
    op64 = _op(g, family, f, p, cuda)
    glo = g.with_(ftype=F16N)
    oplo = _op(glo, family, f, p, cuda, dtype=glo.dtype)
    b = torch.from_numpy(f["b"]).to(cuda)
    x, info = mixed_solve(op64, oplo, b, solver="cg_reliable", tol=1e-10, inner_tol=0.1)
    assert info["rel_res"] <= 1e-10, info
    assert _true_res(g, family, f, p, x.cpu().numpy()) < 2e-10
    _, dc = mixed_solve(op64, oplo, b, solver="cg", tol=1e-10, inner_tol=1e-2)
    assert info["inner_iters"] <= dc["inner_iters"] + 5, (info, dc)


def test_mixed_solver_arguments(cuda):
    g = Geometry(8, 8, 8, 8, soalen=4, veclen=8, ftype=F64, compress12=True, t_boundary=-1.0)
    f, p = H.eo_setup(g, "wilson")
    op64 = _op(g, "wilson", f, p, cuda)
    b = torch.from_numpy(f["b"]).to(cuda)
    with pytest.raises(ValueError):
        mixed_solve(op64, op64, b, solver="gmres")
    with pytest.raises(RuntimeError):
        mixed_solve(op64, op64, b, solver="cg_reliable", inner_tol=1.5)
