"""Device-side layout converters (C-ABI qb200_pack_* / qb200_unpack_spinor).

The same conversions as qphix_b200.layout (which states them in torch), run
as CUDA kernels of libqphix_b200.so on canonical complex tensors that are
already on the GPU:

    flat = convert.pack_spinor(g, sp)          # (nt,nz,ny,nxh,4,3) complex -> tiles
    sp = convert.unpack_spinor(g, flat)        # -> complex128
    gauge = convert.pack_gauge(g, U, cb)       # (4,NT,nz,ny,nx,3,3) complex -> tiles of cb
    clov = convert.pack_clover(g, A)           # (nt,nz,ny,nxh,2,6,6) Hermitian -> CloverBlock
    fclov = convert.pack_full_clover(g, F)     # dense blocks -> FullCloverBlock
"""
import ctypes

import torch

from . import _lib, ops
from .lattice import F32, F64, Geometry

_CTYPE = {torch.complex128: F64, torch.complex64: F32}


def _canon(t):
    if t.dtype not in _CTYPE:
        raise ValueError("canonical fields are complex128 or complex64 tensors")
    if not t.is_cuda:
        raise ValueError("canonical fields must be CUDA tensors")
    t = t.resolve_conj().contiguous()
    return t, _CTYPE[t.dtype]


def pack_spinor(g: Geometry, sp, out=None):
    sp, ct = _canon(sp)
    if tuple(sp.shape) != (g.nt, g.nz, g.ny, g.nxh, 4, 3):
        raise ValueError("spinor shape must be (nt, nz, ny, nxh, 4, 3)")
    out = out if out is not None else torch.zeros(g.spinor_elems, dtype=g.dtype, device=sp.device)
    lat = g.c_struct()
    _lib.check(_lib.lib().qb200_pack_spinor(ctypes.byref(lat), ct, sp.data_ptr(), out.data_ptr(), ops._stream(None)))
    return out


def unpack_spinor(g: Geometry, flat, dtype=torch.complex128):
    out = torch.empty((g.nt, g.nz, g.ny, g.nxh, 4, 3), dtype=dtype, device=flat.device)
    lat = g.c_struct()
    _lib.check(_lib.lib().qb200_unpack_spinor(ctypes.byref(lat), _CTYPE[dtype], flat.data_ptr(), out.data_ptr(),
                                              ops._stream(None)))
    return out


def pack_gauge(g: Geometry, U, cb, t0=0, out=None):
    U, ct = _canon(U)
    if U.dim() != 7 or tuple(U.shape[2:]) != (g.nz, g.ny, g.nx, 3, 3) or U.shape[0] != 4:
        raise ValueError("links shape must be (4, nt_global, nz, ny, nx, 3, 3)")
    out = out if out is not None else torch.empty(g.gauge_elems, dtype=g.dtype, device=U.device)
    lat = g.c_struct()
    _lib.check(_lib.lib().qb200_pack_gauge(ctypes.byref(lat), cb, ct, U.data_ptr(), U.shape[1], t0, out.data_ptr(),
                                           ops._stream(None)))
    return out


def _pack_blocks(fn, g, A, n, out):
    A, ct = _canon(A)
    if tuple(A.shape) != (g.nt, g.nz, g.ny, g.nxh, 2, 6, 6):
        raise ValueError("clover shape must be (nt, nz, ny, nxh, 2, 6, 6)")
    out = out if out is not None else torch.empty(n, dtype=g.dtype, device=A.device)
    lat = g.c_struct()
    _lib.check(fn(ctypes.byref(lat), ct, A.data_ptr(), out.data_ptr(), ops._stream(None)))
    return out


def pack_clover(g: Geometry, A, out=None):
    return _pack_blocks(_lib.lib().qb200_pack_clover, g, A, g.clover_elems, out)


def pack_full_clover(g: Geometry, F, out=None):
    return _pack_blocks(_lib.lib().qb200_pack_full_clover, g, F, g.full_clover_elems, out)
