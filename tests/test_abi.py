"""The C-ABI library: loads, exports every entry point include/qphix_b200.h
declares, and reports argument errors with status codes (no GPU needed: the
checks run before any device call)."""
import ctypes
import os
import re

import pytest

from qphix_b200 import _lib
from qphix_b200.lattice import BF16, F16N, F32, Geometry

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
HEADERS = [os.path.join(INCLUDE, f) for f in sorted(os.listdir(INCLUDE)) if f.endswith(".h")]


def declared_symbols():
    """every extern "C" entry point of include/*.h (the QPhiX template
    specialisations of qphix_b200_qphix.h are checked by test_qphix_tiles)"""
    syms = set()
    for h in HEADERS:
        src = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        syms.update(re.findall(r"\b(qb200_[a-z0-9_]+)\s*\(", src))
    return sorted(syms)


def test_header_declares_the_reference_kernel_set():
    syms = declared_symbols()
    for fam in ("", "clov_", "tm_", "tm_clov_"):
        for k in ("dslash", "dslash_achimbdpsi"):
            for pm in ("plus", "minus"):
                assert "qb200_%s%s_%s_vec" % (fam, k, pm) in syms
    for pm in ("plus", "minus"):
        for f in ("face_proj_dir", "face_finish_dir", "face_clov_finish_dir", "tm_face_finish_dir",
                  "tm_clov_face_finish_dir"):
            assert "qb200_%s_%s" % (f, pm) in syms


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    assert L.qb200_abi_version() == 1


def test_sizes_match_python_geometry():
    L = _lib.lib()
    for g in (Geometry(8, 8, 4, 4, soalen=4, veclen=8), Geometry(32, 4, 4, 2, soalen=16, compress12=True),
              Geometry(4, 4, 4, 6, soalen=1, pad_xy=3, pad_xyz=1),
              Geometry(16, 8, 4, 4, soalen=8, ftype=F16N, pad_xy=1), Geometry(8, 8, 4, 4, soalen=4, ftype=BF16)):
        lat = g.c_struct()
        assert L.qb200_spinor_elems(ctypes.byref(lat)) == g.spinor_elems
        assert L.qb200_gauge_elems(ctypes.byref(lat)) == g.gauge_elems
        assert L.qb200_clover_elems(ctypes.byref(lat)) == g.clover_elems
        assert L.qb200_full_clover_elems(ctypes.byref(lat)) == g.full_clover_elems
        for d in range(8):
            assert L.qb200_face_sites(ctypes.byref(lat), d) == g.face_sites(d)
    assert L.qb200_face_sites(ctypes.byref(Geometry(8, 8, 4, 4).c_struct()), 8) == -1


def _call_plus(lat, psi=16, out=32, gauge=64, cb=0):
    L = _lib.lib()
    v = lambda x: ctypes.c_void_p(x) if x else None
    return L.qb200_dslash_plus_vec(ctypes.byref(lat), cb, v(psi), v(out), v(gauge), None, 1.0, 1.0, 1.0,
                                   0, None, None)


def test_argument_errors_are_status_codes():
    L = _lib.lib()
    g = Geometry(8, 8, 4, 4, soalen=4, veclen=8, ftype=F32)
    bad = g.c_struct()
    bad.nx = 6  # nx/2 not a multiple of soalen
    assert _call_plus(bad) == -1
    bad = g.c_struct()
    bad.soalen = 3
    assert _call_plus(bad) == -3
    bad = g.c_struct()
    bad.ftype = 9
    assert _call_plus(bad) == -3
    assert L.qb200_layout_supported(3, 2) == 0 and L.qb200_layout_supported(3, 8) == 1
    bad = Geometry(8, 8, 4, 4, soalen=2, ftype=F16N).c_struct()
    assert _call_plus(bad) == -3
    assert _call_plus(g.c_struct(), cb=2) == -1
    assert _call_plus(g.c_struct(), psi=0) == -2
    assert _call_plus(g.c_struct(), out=16) == -1  # out aliases psi
    assert b"alias" in L.qb200_last_error()
    rc = L.qb200_dslash_plus_vec(ctypes.byref(g.c_struct()), 0, ctypes.c_void_p(16), ctypes.c_void_p(32),
                                 ctypes.c_void_p(64), None, 1.0, 1.0, 1.0, 1, None, None)
    assert rc == -2  # tbc mask without phases
    assert L.qb200_face_proj_dir_plus(ctypes.byref(g.c_struct()), 0, ctypes.c_void_p(16), ctypes.c_void_p(32),
                                      9, None) == -4
    assert L.qb200_face_finish_dir_minus(ctypes.byref(g.c_struct()), 0, ctypes.c_void_p(16),
                                         ctypes.c_void_p(32), ctypes.c_void_p(64), 1.0, -1, 0, None, None) == -4
    assert b"invalid dir" in L.qb200_last_error()
    assert L.qb200_clov_dslash_plus_vec(ctypes.byref(g.c_struct()), 0, ctypes.c_void_p(16), ctypes.c_void_p(32),
                                        ctypes.c_void_p(64), None, None, 1.0, 1.0, 1.0, 0, None, None) == -2


def test_python_wrapper_rejects_host_tensors():
    import torch
    from qphix_b200 import ops
    g = Geometry(8, 8, 4, 4, soalen=4, veclen=8)
    t = torch.zeros(g.spinor_elems)
    with pytest.raises(ValueError):
        ops.dslash(g, "wilson", "dslash", 1, 0, t, t.clone(), torch.zeros(g.gauge_elems))
