"""Multi-right-hand-side operator and solvers (C-ABI qb200_*_mrhs).

A multi-RHS array holds nrhs (1, 2, 4, 8, 16) spinor fields of one
checkerboard with the right-hand side innermost,
FT[block][3][4][2][S][nrhs]; `pack` / `unpack` convert from / to nrhs
single-layout fields.  Links and clover are shared by all right-hand sides.
"""
import ctypes

import torch

from . import _lib
from .lattice import Geometry
from .solver import FAMILY, EvenOddOperator


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptrs(ts):
    return (ctypes.c_void_p * len(ts))(*[t.data_ptr() for t in ts])


def alloc(g: Geometry, nrhs, device):
    return torch.zeros(g.spinor_elems * nrhs, dtype=g.dtype, device=device)


def pack(g: Geometry, fields, out=None):
    out = out if out is not None else alloc(g, len(fields), fields[0].device)
    _lib.check(_lib.lib().qb200_mrhs_pack(ctypes.byref(g.c_struct()), len(fields), _ptrs(fields), out.data_ptr(),
                                          _stream()))
    return out


def unpack(g: Geometry, mr, nrhs, fields=None):
    fields = fields if fields is not None else [torch.zeros(g.spinor_elems, dtype=g.dtype, device=mr.device)
                                                for _ in range(nrhs)]
    _lib.check(_lib.lib().qb200_mrhs_unpack(ctypes.byref(g.c_struct()), nrhs, mr.data_ptr(), _ptrs(fields),
                                            _stream()))
    return fields


def coeffs(coeff_s=1.0, coeff_t_f=1.0, coeff_t_b=1.0, alpha=1.0, mu=0.0, muinv=1.0, rho=0.0, tbc_mask=0,
           tbc_phases=None):
    c = _lib.Coeffs()
    c.coeff_s, c.coeff_t_f, c.coeff_t_b = coeff_s, coeff_t_f, coeff_t_b
    c.alpha, c.mu, c.muinv, c.rho = alpha, mu, muinv, rho
    c.tbc_mask = tbc_mask
    ph = tbc_phases or [[1.0, 0.0]] * 4
    for m in range(4):
        c.tbc_phases[m][0], c.tbc_phases[m][1] = ph[m][0], ph[m][1]
    return c


def dslash(g: Geometry, nrhs, family, kernel, isign, cb, psi, out, gauge, chi=None, clover=None, accumulate=None,
           **kw):
    c = coeffs(**kw)
    P = lambda t: t.data_ptr() if t is not None else None
    _lib.check(_lib.lib().qb200_dslash_mrhs(ctypes.byref(g.c_struct()), nrhs, FAMILY[family],
                                            1 if kernel == "achimbdpsi" else 0, isign, cb, P(psi), P(chi), P(out),
                                            P(gauge), P(clover), ctypes.byref(c), _lib.uint8(accumulate),
                                            _stream()))
    return out


def schur(op: EvenOddOperator, nrhs, x, isign=1, out=None, tmp=None):
    out = out if out is not None else torch.zeros_like(x)
    tmp = tmp if tmp is not None else torch.zeros_like(x)
    _lib.check(_lib.lib().qb200_schur_apply_mrhs(ctypes.byref(op.lat), nrhs, ctypes.byref(op.op), isign,
                                                 x.data_ptr(), out.data_ptr(), tmp.data_ptr(), _stream()))
    return out


def cg(op: EvenOddOperator, nrhs, b, x=None, tol=1e-10, max_iter=10000):
    L = _lib.lib()
    x = x if x is not None else torch.zeros_like(b)
    ws = op.workspace("cg_mrhs", L.qb200_cg_mrhs_workspace_bytes(ctypes.byref(op.lat), nrhs))
    it = ctypes.c_int(0)
    rel = (ctypes.c_double * nrhs)()
    _lib.check(L.qb200_invert_cg_mrhs(ctypes.byref(op.lat), nrhs, ctypes.byref(op.op), b.data_ptr(), x.data_ptr(),
                                      tol, max_iter, ws.data_ptr(), ctypes.byref(it), rel, _stream()))
    return x, {"iters": it.value, "rel_res": list(rel)}


def mixed_solve(op_hi: EvenOddOperator, op_lo: EvenOddOperator, bs, tol=1e-10, inner_tol=1e-2, max_inner=10000,
                max_outer=50, solver="cg"):
    """Solve Mhat x_i = b_i (FP64 single-layout b_i) for all i, iterating all
    right-hand sides together in low precision.  solver "cg": defect
    correction, each correction solved to inner_tol; "cg_reliable": one CG
    with FP64 reliable updates whenever the residuals have fallen by
    inner_tol (max_inner iterations, max_outer updates)."""
    if solver not in ("cg", "cg_reliable"):
        raise ValueError("unknown solver %r" % solver)
    L = _lib.lib()
    nrhs = len(bs)
    lo = ctypes.c_longlong(0)
    hi = L.qb200_mixed_mrhs_workspace_bytes(ctypes.byref(op_hi.lat), ctypes.byref(op_lo.lat), nrhs,
                                            ctypes.byref(lo))
    ws_hi = op_hi.workspace("mixed_mrhs_hi", hi)
    ws_lo = op_lo.workspace("mixed_mrhs_lo", lo.value)
    xs = [torch.zeros_like(b) for b in bs]
    ii, oo = ctypes.c_int(0), ctypes.c_int(0)
    rel = (ctypes.c_double * nrhs)()
    fn = L.qb200_invert_mixed_mrhs if solver == "cg" else L.qb200_invert_reliable_mrhs
    _lib.check(fn(ctypes.byref(op_hi.lat), ctypes.byref(op_hi.op), ctypes.byref(op_lo.lat), ctypes.byref(op_lo.op),
                  nrhs, _ptrs(bs), _ptrs(xs), tol, inner_tol, max_inner, max_outer, ws_hi.data_ptr(),
                  ws_lo.data_ptr(), ctypes.byref(ii), ctypes.byref(oo), rel, _stream()))
    return xs, {"inner_iters": ii.value, "outer_iters": oo.value, "rel_res": list(rel)}
