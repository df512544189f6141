"""qb200_schur_apply_noalloc: the even-odd operator for callers that cannot
hand the library device scratch memory (for example a host program whose
device memory is owned by its own allocator and may not call cudaMalloc on
this path).  Its intermediate spinor lives in a static device array inside
the library.  Checked through the C-ABI against qb200_schur_apply, which
takes the scratch from the caller, on two calls in a row (the array keeps
the previous call's contents, which must not leak into the next result).
This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest
import torch

import helpers as H
from qphix_b200 import _lib, fields, layout
from qphix_b200.lattice import F16N, F32, F64, Geometry
from qphix_b200.solver import EvenOddOperator

TOL = H.TOL


def _operator(g, family, dev, seed):
    f, p = H.eo_setup(g, family, seed=seed)
    T = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    op = EvenOddOperator(g, family, gauge=[T(x) for x in f["gauge"]], clov=[T(x) for x in f["clov"]],
                         clov_dag=[T(x) for x in f["clov_dag"]], target_cb=1, **p)
    return op, f


@pytest.mark.gpu
# FP16 + per-site norm has 26 stored halves per site (the norm included), not
# the 24 elements of the other types: the scratch-size check must count them
@pytest.mark.parametrize("ft,family", [(F32, "clover"), (F64, "tm_clover"), (F16N, "tm")])
def test_noalloc_matches_caller_scratch_twice(cuda, ft, family):
    L = _lib.lib()
    g = Geometry(16, 16, 8, 8, soalen=8, veclen=8, ftype=ft, compress12=True, t_boundary=-1.0)
    op, f = _operator(g, family, cuda, seed=700)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call, isign in enumerate((1, -1)):
        src = H.to_torch(layout.pack_spinor(g, fields.random_spinor(g, seed=710 + call)), cuda)
        out_na = torch.full_like(src, float("nan"))
        rc = L.qb200_schur_apply_noalloc(ctypes.byref(op.lat), ctypes.byref(op.op), isign,
                                         ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(out_na.data_ptr()),
                                         stream)
        _lib.check(rc)
        out_ref = torch.zeros_like(src)
        tmp = torch.zeros_like(src)
        rc = L.qb200_schur_apply(ctypes.byref(op.lat), ctypes.byref(op.op), isign, ctypes.c_void_p(src.data_ptr()),
                                 ctypes.c_void_p(out_ref.data_ptr()), ctypes.c_void_p(tmp.data_ptr()), stream)
        _lib.check(rc)
        torch.cuda.synchronize()
        e = H.site_rel_err(g, H.to_np(out_na), H.to_np(out_ref))
        assert e < TOL[ft], (call, e)


@pytest.mark.gpu
def test_noalloc_rejects_lattices_beyond_its_scratch(cuda):
    L = _lib.lib()
    g = Geometry(32, 32, 32, 32, soalen=16, ftype=F32, compress12=True)   # 50 MB spinor > 32 MiB
    dummy = torch.zeros(16, dtype=torch.float32, device=cuda)
    op = _lib.Operator()
    op.family, op.target_cb = 0, 1
    op.gauge[0] = op.gauge[1] = dummy.data_ptr()
    op.alpha = 4.0
    lat = g.c_struct()
    rc = L.qb200_schur_apply_noalloc(ctypes.byref(lat), ctypes.byref(op), 1, ctypes.c_void_p(dummy.data_ptr()),
                                     ctypes.c_void_p(dummy.data_ptr() + 64), None)
    assert rc == -1
    assert b"scratch" in L.qb200_last_error()
