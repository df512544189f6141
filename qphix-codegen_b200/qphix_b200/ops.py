"""Torch-facing calls of the dslash C-ABI.

Each function takes device tensors in the QPhiX layouts of `Geometry`, checks
them, and launches on the current CUDA stream (or `stream`).  The names follow
the reference kernels (codegen/jinja/*_decl.h.j2): family in
{"wilson", "clover", "tm", "tm_clover"}, kernel in {"dslash", "achimbdpsi"},
isign in {+1, -1}.
"""
import ctypes

import torch

from . import _lib
from .lattice import Geometry

FAMILIES = ("wilson", "clover", "tm", "tm_clover")
_PREFIX = {"wilson": "", "clover": "clov_", "tm": "tm_", "tm_clover": "tm_clov_"}


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream(stream):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _check_field(name, t, g: Geometry, numel):
    if t is None:
        raise ValueError("%s is required" % name)
    if not t.is_cuda:
        raise ValueError("%s must be a CUDA tensor" % name)
    if t.dtype != g.dtype:
        raise ValueError("%s has dtype %s, expected %s" % (name, t.dtype, g.dtype))
    if not t.is_contiguous():
        raise ValueError("%s must be contiguous" % name)
    if t.numel() < numel:
        raise ValueError("%s has %d elements, needs %d" % (name, t.numel(), numel))


def dslash(g: Geometry, family, kernel, isign, cb, psi, out, gauge, *, chi=None, clover=None,
           coeff_s=1.0, coeff_t_f=1.0, coeff_t_b=1.0, alpha=1.0, mu=0.0, muinv=1.0, rho=0.0,
           tbc_mask=0, tbc_phases=None, accumulate=None, stream=None):
    """Apply one operator of the family to checkerboard cb: out = op(psi[, chi])."""
    if family not in FAMILIES:
        raise ValueError("unknown family %r" % family)
    if kernel not in ("dslash", "achimbdpsi"):
        raise ValueError("unknown kernel %r" % kernel)
    L = _lib.lib()
    pm = "plus" if isign > 0 else "minus"
    name = "qb200_%sdslash_%s%s_vec" % (_PREFIX[family], "achimbdpsi_" if kernel == "achimbdpsi" else "", pm)
    fn = getattr(L, name)
    _check_field("psi", psi, g, g.spinor_elems)
    _check_field("out", out, g, g.spinor_elems)
    _check_field("gauge", gauge, g, g.gauge_elems)
    if kernel == "achimbdpsi":
        _check_field("chi", chi, g, g.spinor_elems)
    if family in ("clover", "tm_clover"):
        _check_field("clover", clover, g,
                     g.clover_elems if family == "clover" else g.full_clover_elems)
    lat = g.c_struct()
    acc = _lib.uint8(accumulate)
    ph = _lib.phases(tbc_phases)
    m = ctypes.c_uint(int(tbc_mask))
    st = _stream(stream)
    P = _ptr
    if family == "wilson" and kernel == "dslash":
        rc = fn(ctypes.byref(lat), cb, P(psi), P(out), P(gauge), acc, coeff_s, coeff_t_f, coeff_t_b, m, ph, st)
    elif family == "wilson":
        rc = fn(ctypes.byref(lat), cb, P(psi), P(chi), P(out), P(gauge), alpha, coeff_s, coeff_t_f, coeff_t_b,
                m, ph, acc, st)
    elif family in ("clover", "tm_clover") and kernel == "dslash":
        rc = fn(ctypes.byref(lat), cb, P(psi), P(out), P(gauge), P(clover), acc, coeff_s, coeff_t_f,
                coeff_t_b, m, ph, st)
    elif family in ("clover", "tm_clover"):
        rc = fn(ctypes.byref(lat), cb, P(psi), P(chi), P(out), P(gauge), P(clover), coeff_s, coeff_t_f,
                coeff_t_b, m, ph, acc, rho, st)
    elif kernel == "dslash":  # tm
        rc = fn(ctypes.byref(lat), cb, P(psi), P(out), P(gauge), acc, coeff_s, coeff_t_f, coeff_t_b, m, ph,
                mu, muinv, st)
    else:  # tm achimbdpsi
        rc = fn(ctypes.byref(lat), cb, P(psi), P(chi), P(out), P(gauge), alpha, coeff_s, coeff_t_f,
                coeff_t_b, m, ph, mu, acc, st)
    _lib.check(rc)
    return out


def face_pack(g: Geometry, isign, psi_cb, psi, outbuf, dir, stream=None):
    """face_proj_dir: project the face of psi towards dir into outbuf."""
    L = _lib.lib()
    fn = L.qb200_face_proj_dir_plus if isign > 0 else L.qb200_face_proj_dir_minus
    _check_field("psi", psi, g, g.spinor_elems)
    _check_field("outbuf", outbuf, g, g.face_sites(dir) * g.face_elems)
    lat = g.c_struct()
    _lib.check(fn(ctypes.byref(lat), psi_cb, _ptr(psi), _ptr(outbuf), dir, _stream(stream)))
    return outbuf


def face_unpack(g: Geometry, family, isign, cb, inbuf, gauge, out, dir, *, beta=1.0, clover=None,
                mu=0.0, muinv=1.0, tbc=False, tbc_phases=None, stream=None):
    """face_*finish_dir: accumulate the face contribution of dir into out."""
    L = _lib.lib()
    pm = "plus" if isign > 0 else "minus"
    _check_field("inbuf", inbuf, g, g.face_sites(dir) * g.face_elems)
    _check_field("gauge", gauge, g, g.gauge_elems)
    _check_field("out", out, g, g.spinor_elems)
    lat = g.c_struct()
    ph = _lib.phases(tbc_phases)
    st = _stream(stream)
    t = 1 if tbc else 0
    P = _ptr
    if family == "wilson":
        rc = getattr(L, "qb200_face_finish_dir_" + pm)(ctypes.byref(lat), cb, P(inbuf), P(gauge), P(out), beta,
                                                      dir, t, ph, st)
    elif family == "clover":
        _check_field("clover", clover, g, g.clover_elems)
        rc = getattr(L, "qb200_face_clov_finish_dir_" + pm)(ctypes.byref(lat), cb, P(inbuf), P(gauge), P(out),
                                                           P(clover), beta, dir, t, ph, st)
    elif family == "tm":
        rc = getattr(L, "qb200_tm_face_finish_dir_" + pm)(ctypes.byref(lat), cb, P(inbuf), P(gauge), P(out),
                                                         beta, mu, muinv, dir, t, ph, st)
    elif family == "tm_clover":
        _check_field("clover", clover, g, g.full_clover_elems)
        rc = getattr(L, "qb200_tm_clov_face_finish_dir_" + pm)(ctypes.byref(lat), cb, P(inbuf), P(gauge),
                                                              P(out), P(clover), beta, dir, t, ph, st)
    else:
        raise ValueError("unknown family %r" % family)
    _lib.check(rc)
    return out
