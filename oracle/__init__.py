"""Python access to the oracle (TEST INFRASTRUCTURE).

Two checkers live here, both CPU-only and used only by tests/, the smoke check
in __graft_entry__.py and bench.py's reference / cpu_baseline legs:

  * liboracle.so  -- qb200_oracle.c, the FP64 C restatement of the operator
                     family (built from source with gcc on first use);
  * oracle/_ref/libqphix_ref_<cfg>.so -- the reference's own generated
                     kernels driven over whole lattices by ref_driver.cpp
                     (built here by ref_build.py from the reference sources;
                     they travel to the GPU box prebuilt).

All fields are numpy arrays in the QPhiX tile layouts of
include/qphix_b200.h, in the storage type of the lattice.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(HERE, "liboracle.so")

FAMILY = {"wilson": 0, "clover": 1, "tm": 2, "tm_clover": 3}
NP_DTYPE = {0: np.float32, 1: np.float64, 2: np.float16}


class Lattice(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("nt", ctypes.c_int),
        ("soalen", ctypes.c_int), ("veclen", ctypes.c_int),
        ("pad_xy", ctypes.c_int), ("pad_xyz", ctypes.c_int),
        ("ftype", ctypes.c_int), ("compress12", ctypes.c_int),
        ("t_boundary", ctypes.c_double),
        ("t_edge_lo", ctypes.c_int), ("t_edge_hi", ctypes.c_int),
    ]


class Params(ctypes.Structure):
    """oracle_params of oracle/oracle.h."""
    _fields_ = [
        ("coeff_s", ctypes.c_double), ("coeff_t_f", ctypes.c_double), ("coeff_t_b", ctypes.c_double),
        ("alpha", ctypes.c_double), ("mu", ctypes.c_double), ("muinv", ctypes.c_double),
        ("rho", ctypes.c_double), ("tbc_mask", ctypes.c_uint),
        ("tbc_phases", (ctypes.c_double * 2) * 4), ("accumulate", ctypes.c_uint * 8),
    ]


def make_params(coeff_s=1.0, coeff_t_f=1.0, coeff_t_b=1.0, alpha=1.0, mu=0.0, muinv=1.0, rho=0.0,
                tbc_mask=0, tbc_phases=None, accumulate=None):
    p = Params()
    p.coeff_s, p.coeff_t_f, p.coeff_t_b = coeff_s, coeff_t_f, coeff_t_b
    p.alpha, p.mu, p.muinv, p.rho = alpha, mu, muinv, rho
    p.tbc_mask = int(tbc_mask)
    ph = tbc_phases if tbc_phases is not None else [[1.0, 0.0]] * 4
    for m in range(4):
        p.tbc_phases[m][0], p.tbc_phases[m][1] = float(ph[m][0]), float(ph[m][1])
    acc = accumulate if accumulate is not None else [1] * 8
    for d in range(8):
        p.accumulate[d] = int(acc[d])
    return p


def lattice_struct(g):
    """Lattice from a qphix_b200.Geometry (or anything with the same fields)."""
    return Lattice(g.nx, g.ny, g.nz, g.nt, g.soalen, g.veclen, g.pad_xy, g.pad_xyz, g.ftype,
                   1 if g.compress12 else 0, float(g.t_boundary), 1 if g.t_edge_lo else 0,
                   1 if g.t_edge_hi else 0)


def aligned(a, align=64, pad=64):
    """Copy of `a` (1-D) in an `align`-byte aligned buffer with `pad` spare elements."""
    a = np.ascontiguousarray(a).reshape(-1)
    n = a.size + pad
    raw = np.zeros(n * a.itemsize + align, dtype=np.uint8)
    off = (-raw.ctypes.data) % align
    out = raw[off: off + n * a.itemsize].view(a.dtype)
    out[: a.size] = a
    return out


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


# --------------------------------------------------------------------------
# the C restatement

_oracle = None


def build_oracle(force=False):
    src = os.path.join(HERE, "qb200_oracle.c")
    hdrs = [os.path.join(HERE, "oracle.h"), os.path.join(os.path.dirname(HERE), "include", "qphix_b200.h")]
    newest = max(os.path.getmtime(p) for p in [src] + hdrs)
    if force or not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < newest:
        subprocess.check_call(["gcc", "-O2", "-std=gnu11", "-fopenmp", "-fPIC", "-shared", "-Wall",
                               src, "-o", ORACLE_SO, "-lm"])
    return ORACLE_SO


def liboracle():
    global _oracle
    if _oracle is None:
        build_oracle()
        L = ctypes.CDLL(ORACLE_SO)
        LP = ctypes.POINTER(Lattice)
        V = ctypes.c_void_p
        I, D = ctypes.c_int, ctypes.c_double
        L.oracle_dslash.argtypes = [LP, I, I, I, I, V, V, V, V, V, ctypes.POINTER(Params)]
        L.oracle_dslash_out.argtypes = [LP, I, I, I, I, I, V, V, V, V, V, ctypes.POINTER(Params)]
        L.oracle_spinor_elems_f64.argtypes = [LP]
        L.oracle_spinor_elems_f64.restype = ctypes.c_longlong
        L.oracle_face_count.argtypes = [LP, I, I]
        L.oracle_face_count.restype = ctypes.c_longlong
        L.oracle_face_pack.argtypes = [LP, I, I, V, V, I, V]
        L.oracle_face_pack_out.argtypes = [LP, I, I, I, V, V, I, V]
        L.oracle_face_unpack.argtypes = [LP, I, I, I, V, V, V, V, D, D, D, I, I, V, V]
        L.oracle_face_unpack_out.argtypes = [LP, I, I, I, I, V, V, V, V, D, D, D, I, I, V, V]
        L.oracle_hop_force.argtypes = [LP, I, I, V, V, V, ctypes.POINTER(Params), V]
        _oracle = L
    return _oracle


def dslash(g, family, kernel, isign, cb, psi, gauge, chi=None, clover=None, params=None, out=None, fp64_out=False):
    """Oracle body kernel; returns out (numpy, storage dtype).  fp64_out: the
    result unrounded, as an FP64 spinor array of the same lattice (layout of
    g with ftype QB200_F64)."""
    L = liboracle()
    lat = lattice_struct(g)
    p = params if params is not None else make_params()
    if out is None:
        if fp64_out:
            n = L.oracle_spinor_elems_f64(ctypes.byref(lat))
            out = np.zeros(n, dtype=np.float64)
        else:
            out = np.zeros(psi.size, dtype=psi.dtype)
    rc = L.oracle_dslash_out(ctypes.byref(lat), 1 if fp64_out else g.ftype, FAMILY[family],
                             1 if kernel == "achimbdpsi" else 0, 1 if isign > 0 else -1, cb, _ptr(psi), _ptr(chi),
                             _ptr(gauge), _ptr(clover), _ptr(out), ctypes.byref(p))
    if rc:
        raise RuntimeError("oracle_dslash failed: %d" % rc)
    return out


def face_pack(g, isign, psi_cb, psi, dir, fp64_out=False):
    """Face records of psi towards dir; fp64_out: unrounded, 12 doubles per site."""
    L = liboracle()
    lat = lattice_struct(g)
    n = L.oracle_face_count(ctypes.byref(lat), psi_cb, dir)
    if fp64_out:
        buf = np.zeros(12 * n, dtype=np.float64)
    else:
        buf = np.zeros((14 if g.ftype == 3 else 12) * n, dtype=psi.dtype)
    scratch = np.zeros(4 * n + 4, dtype=np.int32)
    rc = L.oracle_face_pack_out(ctypes.byref(lat), 1 if fp64_out else g.ftype, 1 if isign > 0 else -1, psi_cb,
                                _ptr(psi), _ptr(buf), dir, _ptr(scratch))
    if rc:
        raise RuntimeError("oracle_face_pack failed: %d" % rc)
    return buf


def face_unpack(g, family, isign, cb, inbuf, gauge, out, dir, beta=1.0, clover=None, mu=0.0, muinv=1.0,
                tbc=False, tbc_phases=None, fp64_out=False):
    """Accumulates into `out` in place (numpy); returns out.  fp64_out: out is
    an FP64 spinor array (layout of g with ftype QB200_F64), kept unrounded."""
    L = liboracle()
    lat = lattice_struct(g)
    n = L.oracle_face_count(ctypes.byref(lat), cb, dir)
    scratch = np.zeros(4 * n + 4, dtype=np.int32)
    ph = np.asarray(tbc_phases if tbc_phases is not None else [[1.0, 0.0]] * 4, dtype=np.float64).reshape(-1)
    rc = L.oracle_face_unpack_out(ctypes.byref(lat), 1 if fp64_out else g.ftype, FAMILY[family],
                                  1 if isign > 0 else -1, cb, _ptr(inbuf), _ptr(gauge), _ptr(out), _ptr(clover),
                                  beta, mu, muinv, dir, 1 if tbc else 0, _ptr(ph), _ptr(scratch))
    if rc:
        raise RuntimeError("oracle_face_unpack failed: %d" % rc)
    return out


def hop_force(g, isign, cb, chi, psi, gauge=None, params=None):
    """FP64 link derivative of Re <chi, H psi> (H: plain Wilson hopping term on
    cb), or its su(3) projection when `gauge` (checkerboard cb) is given.
    Returns a float64 array of 144 * (sites of cb) reals laid out as
    qb200_hop_force's output."""
    L = liboracle()
    lat = lattice_struct(g)
    p = params if params is not None else make_params()
    out = np.zeros(144 * g.nx // 2 * g.ny * g.nz * g.nt, dtype=np.float64)
    rc = L.oracle_hop_force(ctypes.byref(lat), 1 if isign > 0 else -1, cb, _ptr(chi), _ptr(psi), _ptr(gauge),
                            ctypes.byref(p), _ptr(out))
    if rc:
        raise RuntimeError("oracle_hop_force failed: %d" % rc)
    return out


# --------------------------------------------------------------------------
# the reference's generated kernels

_refs = {}


def ref_available(name):
    return os.path.exists(os.path.join(REF_DIR, "libqphix_ref_%s.so" % name))


def reflib(name):
    if name not in _refs:
        path = os.path.join(REF_DIR, "libqphix_ref_%s.so" % name)
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (run python oracle/ref_build.py %s)" % name)
        L = ctypes.CDLL(path)
        LP = ctypes.POINTER(Lattice)
        V, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        IP = ctypes.POINTER(ctypes.c_int)
        L.rd_info.argtypes = [IP, IP, IP, IP]
        L.rd_dslash.argtypes = [LP, I, I, I, I, V, V, V, V, V, ctypes.POINTER(Params), I]
        L.rd_face_pack.argtypes = [LP, I, I, V, V, I]
        L.rd_face_unpack.argtypes = [LP, I, I, I, V, V, V, V, D, D, D, I, I, V]
        _refs[name] = L
    return _refs[name]


def ref_info(name):
    L = reflib(name)
    v, s, b, h = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    L.rd_info(ctypes.byref(v), ctypes.byref(s), ctypes.byref(b), ctypes.byref(h))
    return {"veclen": v.value, "soalen": s.value, "ft_bytes": b.value, "half": bool(h.value)}


def ref_dslash(name, g, family, kernel, isign, cb, psi, gauge, chi=None, clover=None, params=None, out=None,
               nthreads=0):
    """Reference kernels over the whole checkerboard.  Inputs must come from
    `aligned` (64-byte aligned, padded); returns out."""
    L = reflib(name)
    lat = lattice_struct(g)
    p = params if params is not None else make_params()
    if out is None:
        out = aligned(np.zeros(g.spinor_elems, dtype=psi.dtype))
    rc = L.rd_dslash(ctypes.byref(lat), FAMILY[family], 1 if kernel == "achimbdpsi" else 0,
                     1 if isign > 0 else -1, cb, _ptr(psi), _ptr(chi), _ptr(gauge), _ptr(clover), _ptr(out),
                     ctypes.byref(p), nthreads)
    if rc:
        raise RuntimeError("rd_dslash failed: %d" % rc)
    return out


def ref_face_pack(name, g, isign, psi_cb, psi, dir):
    L = reflib(name)
    lat = lattice_struct(g)
    n = liboracle().oracle_face_count(ctypes.byref(lat), psi_cb, dir)
    buf = np.zeros(12 * n + 64, dtype=psi.dtype)
    rc = L.rd_face_pack(ctypes.byref(lat), 1 if isign > 0 else -1, psi_cb, _ptr(psi), _ptr(buf), dir)
    if rc:
        raise RuntimeError("rd_face_pack failed: %d" % rc)
    return buf[: 12 * n]


def ref_face_unpack(name, g, family, isign, cb, inbuf, gauge, out, dir, beta=1.0, clover=None, mu=0.0,
                    muinv=1.0, tbc=False, tbc_phases=None):
    L = reflib(name)
    lat = lattice_struct(g)
    ph = np.asarray(tbc_phases if tbc_phases is not None else [[1.0, 0.0]] * 4, dtype=np.float64).reshape(-1)
    rc = L.rd_face_unpack(ctypes.byref(lat), FAMILY[family], 1 if isign > 0 else -1, cb, _ptr(inbuf),
                          _ptr(gauge), _ptr(out), _ptr(clover), beta, mu, muinv, dir, 1 if tbc else 0, _ptr(ph))
    if rc:
        raise RuntimeError("rd_face_unpack failed: %d" % rc)
    return out
