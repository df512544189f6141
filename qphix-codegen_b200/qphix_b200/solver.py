"""Even-odd preconditioned operator and Krylov solvers (C-ABI in
libqphix_b200.so; see qb200_operator in include/qphix_b200.h).

    op = EvenOddOperator(g, "clover", gauge=(u0, u1), clov=(A_inv_even, A_odd), coeff_s=kappa, ...)
    x, info = op.cg(b, tol=1e-10)
    x, info = mixed_solve(op64, op32, b, tol=1e-10)     # FP64 corrections of an FP32/FP16 solve

The target checkerboard is `target_cb` (1 = odd, as in QPhiX); `clov` and
`gauge` are indexed by checkerboard.  Workspaces are allocated here with
torch and passed down (the library itself allocates nothing); each operator
keeps its solver workspaces between calls, so solves with one operator must
run on one stream, one at a time.
"""
import ctypes

import torch

from . import _lib
from .lattice import F64, Geometry

FAMILY = {"wilson": 0, "clover": 1, "tm": 2, "tm_clover": 3}


def _ptr(t):
    return t.data_ptr() if t is not None else None


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class EvenOddOperator:
    def __init__(self, g: Geometry, family, gauge, clov=(None, None), clov_dag=(None, None), target_cb=1,
                 coeff_s=1.0, coeff_t_f=1.0, coeff_t_b=1.0, alpha=1.0, mu=0.0, muinv=1.0, rho=0.0, tbc_mask=0,
                 tbc_phases=None):
        self.g = g
        self.family = family
        self.keep = [gauge, clov, clov_dag]   # keep the tensors alive
        op = _lib.Operator()
        op.family = FAMILY[family]
        op.target_cb = target_cb
        for cb in (0, 1):
            op.gauge[cb] = _ptr(gauge[cb])
            op.clov[cb] = _ptr(clov[cb])
            op.clov_dag[cb] = _ptr(clov_dag[cb])
        op.coeff_s, op.coeff_t_f, op.coeff_t_b = coeff_s, coeff_t_f, coeff_t_b
        op.alpha, op.mu, op.muinv, op.rho = alpha, mu, muinv, rho
        op.tbc_mask = tbc_mask
        ph = tbc_phases or [[1.0, 0.0]] * 4
        for m in range(4):
            op.tbc_phases[m][0], op.tbc_phases[m][1] = ph[m][0], ph[m][1]
        self.op = op
        self.lat = g.c_struct()
        self.device = gauge[0].device
        self._ws = {}

    def _spinor(self):
        return torch.zeros(self.g.spinor_elems, dtype=self.g.dtype, device=self.device)

    def _bytes(self, n):
        return torch.empty(int(n), dtype=torch.uint8, device=self.device)

    def workspace(self, key, nbytes):
        """Device byte buffer of at least nbytes, kept for later solves."""
        t = self._ws.get(key)
        if t is None or t.numel() < int(nbytes):
            self._ws.pop(key, None)
            t = self._ws[key] = self._bytes(nbytes)
        return t

    def apply(self, x, isign=1, out=None, tmp=None):
        """out = Mhat x (isign +1) or Mhat^dag x (-1)."""
        out = out if out is not None else self._spinor()
        tmp = tmp if tmp is not None else self._spinor()
        _lib.check(_lib.lib().qb200_schur_apply(ctypes.byref(self.lat), ctypes.byref(self.op), isign, _ptr(x),
                                                _ptr(out), _ptr(tmp), _stream()))
        return out

    def _solve(self, fn, wsfn, b, x, tol, max_iter):
        L = _lib.lib()
        x = x if x is not None else self._spinor()
        ws = self.workspace(wsfn, getattr(L, wsfn)(ctypes.byref(self.lat)))
        it = ctypes.c_int(0)
        rel = ctypes.c_double(0.0)
        _lib.check(getattr(L, fn)(ctypes.byref(self.lat), ctypes.byref(self.op), _ptr(b), _ptr(x), tol, max_iter,
                                  _ptr(ws), ctypes.byref(it), ctypes.byref(rel), _stream()))
        return x, {"iters": it.value, "rel_res": rel.value}

    def cg(self, b, x=None, tol=1e-10, max_iter=10000):
        """CG on Mhat^dag Mhat x = Mhat^dag b (x: initial guess, default 0)."""
        return self._solve("qb200_invert_cg", "qb200_cg_workspace_bytes", b, x, tol, max_iter)

    def cg_normal(self, b, x=None, tol=1e-10, max_iter=10000):
        """CG on Mhat^dag Mhat x = b (rel_res: |b - Mhat^dag Mhat x| / |b|)."""
        return self._solve("qb200_invert_cg_normal", "qb200_cg_workspace_bytes", b, x, tol, max_iter)

    def bicgstab(self, b, x=None, tol=1e-10, max_iter=10000):
        return self._solve("qb200_invert_bicgstab", "qb200_bicgstab_workspace_bytes", b, x, tol, max_iter)


SOLVERS = {"cg": 0, "bicgstab": 1, "cg_reliable": 2}


def mixed_solve(op_hi: EvenOddOperator, op_lo: EvenOddOperator, b, solver="cg", tol=1e-10, inner_tol=1e-3,
                max_inner=10000, max_outer=50, x=None):
    """Mixed-precision solve with the FP64 residual and solution in op_hi
    (FP64 storage) and the iterations in op_lo (FP32, FP16, FP16 + norm or
    BF16 storage).  solver "cg" / "bicgstab": defect correction, each
    correction solved to inner_tol (max_inner iterations, max_outer
    corrections).  solver "cg_reliable": one CG on the normal equations with
    reliable updates -- the FP64 residual replaces the low-precision one
    whenever the latter has fallen by inner_tol, keeping the search direction
    (max_inner iterations in all, max_outer updates)."""
    if op_hi.g.ftype != F64:
        raise ValueError("the high-precision operator must use FP64 storage")
    if solver not in SOLVERS:
        raise ValueError("unknown solver %r" % solver)
    L = _lib.lib()
    lo = ctypes.c_longlong(0)
    hi = L.qb200_mixed_workspace_bytes(ctypes.byref(op_hi.lat), ctypes.byref(op_lo.lat), ctypes.byref(lo))
    ws_hi, ws_lo = op_hi.workspace("mixed_hi", hi), op_lo.workspace("mixed_lo", lo.value)
    x = x if x is not None else op_hi._spinor()
    ii, oo, rel = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0.0)
    _lib.check(L.qb200_invert_mixed(ctypes.byref(op_hi.lat), ctypes.byref(op_hi.op), ctypes.byref(op_lo.lat),
                                    ctypes.byref(op_lo.op), SOLVERS[solver], _ptr(b), _ptr(x), tol,
                                    inner_tol, max_inner, max_outer, _ptr(ws_hi), _ptr(ws_lo), ctypes.byref(ii),
                                    ctypes.byref(oo), ctypes.byref(rel), _stream()))
    return x, {"inner_iters": ii.value, "outer_iters": oo.value, "rel_res": rel.value}
