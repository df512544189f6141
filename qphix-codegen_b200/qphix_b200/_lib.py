"""ctypes binding of libqphix_b200.so (the C-ABI of include/qphix_b200.h).

The library is built in-tree by qphix-codegen_b200/build.py.  There is no
fallback: if the library is missing or a call fails, an exception is raised.
"""
import ctypes
import os

from .lattice import Lattice

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libqphix_b200.so")

_P = ctypes.c_void_p
_I = ctypes.c_int
_U = ctypes.c_uint
_D = ctypes.c_double
_LAT = ctypes.POINTER(Lattice)
_UA = ctypes.POINTER(ctypes.c_uint)
_DA = ctypes.POINTER(ctypes.c_double)

ERRORS = {-1: "QB200_EINVAL", -2: "QB200_ENULL", -3: "QB200_ELAYOUT", -4: "QB200_EDIR",
          -5: "QB200_ECUDA", -6: "QB200_EALIGN", -7: "QB200_ENODEV"}

# argument lists, in the order of include/qphix_b200.h
_BODY = [_LAT, _I, _P, _P, _P, _UA, _D, _D, _D, _U, _DA, _P]
_ACH = [_LAT, _I, _P, _P, _P, _P, _D, _D, _D, _D, _U, _DA, _UA, _P]
_CLOV = [_LAT, _I, _P, _P, _P, _P, _UA, _D, _D, _D, _U, _DA, _P]
_CLOV_ACH = [_LAT, _I, _P, _P, _P, _P, _P, _D, _D, _D, _U, _DA, _UA, _D, _P]
_TM = [_LAT, _I, _P, _P, _P, _UA, _D, _D, _D, _U, _DA, _D, _D, _P]
_TM_ACH = [_LAT, _I, _P, _P, _P, _P, _D, _D, _D, _D, _U, _DA, _D, _UA, _P]
_PACK = [_LAT, _I, _P, _P, _I, _P]
_FIN = [_LAT, _I, _P, _P, _P, _D, _I, _I, _DA, _P]
_FIN_CLOV = [_LAT, _I, _P, _P, _P, _P, _D, _I, _I, _DA, _P]
_FIN_TM = [_LAT, _I, _P, _P, _P, _D, _D, _D, _I, _I, _DA, _P]

SIGNATURES = {}
for _pm in ("plus", "minus"):
    SIGNATURES.update({
        "qb200_dslash_%s_vec" % _pm: _BODY,
        "qb200_dslash_achimbdpsi_%s_vec" % _pm: _ACH,
        "qb200_clov_dslash_%s_vec" % _pm: _CLOV,
        "qb200_clov_dslash_achimbdpsi_%s_vec" % _pm: _CLOV_ACH,
        "qb200_tm_dslash_%s_vec" % _pm: _TM,
        "qb200_tm_dslash_achimbdpsi_%s_vec" % _pm: _TM_ACH,
        "qb200_tm_clov_dslash_%s_vec" % _pm: _CLOV,
        "qb200_tm_clov_dslash_achimbdpsi_%s_vec" % _pm: _CLOV_ACH,
        "qb200_face_proj_dir_%s" % _pm: _PACK,
        "qb200_face_finish_dir_%s" % _pm: _FIN,
        "qb200_face_clov_finish_dir_%s" % _pm: _FIN_CLOV,
        "qb200_tm_face_finish_dir_%s" % _pm: _FIN_TM,
        "qb200_tm_clov_face_finish_dir_%s" % _pm: _FIN_CLOV,
    })
INFO = {
    "qb200_abi_version": ([], _I),
    "qb200_last_error": ([], ctypes.c_char_p),
    "qb200_layout_supported": ([_I, _I], _I),
    "qb200_spinor_elems": ([_LAT], ctypes.c_longlong),
    "qb200_gauge_elems": ([_LAT], ctypes.c_longlong),
    "qb200_clover_elems": ([_LAT], ctypes.c_longlong),
    "qb200_full_clover_elems": ([_LAT], ctypes.c_longlong),
    "qb200_face_sites": ([_LAT, _I], ctypes.c_longlong),
}



class Operator(ctypes.Structure):
    """ctypes mirror of `qb200_operator`."""
    _fields_ = [
        ("family", ctypes.c_int), ("target_cb", ctypes.c_int),
        ("gauge", ctypes.c_void_p * 2), ("clov", ctypes.c_void_p * 2), ("clov_dag", ctypes.c_void_p * 2),
        ("coeff_s", ctypes.c_double), ("coeff_t_f", ctypes.c_double), ("coeff_t_b", ctypes.c_double),
        ("alpha", ctypes.c_double), ("mu", ctypes.c_double), ("muinv", ctypes.c_double), ("rho", ctypes.c_double),
        ("tbc_mask", ctypes.c_uint), ("tbc_phases", (ctypes.c_double * 2) * 4),
    ]


_OP = ctypes.POINTER(Operator)
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)
_LL = ctypes.c_longlong
SIGNATURES.update({
    "qb200_schur_apply": [_LAT, _OP, _I, _P, _P, _P, _P],
    "qb200_schur_apply_noalloc": [_LAT, _OP, _I, _P, _P, _P],
    "qb200_blas_axpby": [_I, _LL, _D, _P, _D, _P, _P],
    "qb200_blas_convert": [_I, _P, _I, _P, _LL, _D, _P],
    "qb200_blas_dot": [_I, _LL, _P, _P, _P, _P, _P],
    "qb200_blas_cdot": [_LAT, _P, _P, _P, _P, _P],
    "qb200_invert_cg": [_LAT, _OP, _P, _P, _D, _I, _P, _IP, _DP, _P],
    "qb200_invert_bicgstab": [_LAT, _OP, _P, _P, _D, _I, _P, _IP, _DP, _P],
    "qb200_invert_cg_normal": [_LAT, _OP, _P, _P, _D, _I, _P, _IP, _DP, _P],
    "qb200_invert_mixed": [_LAT, _OP, _LAT, _OP, _I, _P, _P, _D, _D, _I, _I, _P, _P, _IP, _IP, _DP, _P],
})
INFO.update({
    "qb200_blas_partials_len": ([], _LL),
    "qb200_cg_workspace_bytes": ([_LAT], _LL),
    "qb200_bicgstab_workspace_bytes": ([_LAT], _LL),
    "qb200_mixed_workspace_bytes": ([_LAT, _LAT, ctypes.POINTER(_LL)], _LL),
})



class Coeffs(ctypes.Structure):
    """ctypes mirror of `qb200_coeffs`."""
    _fields_ = [
        ("coeff_s", ctypes.c_double), ("coeff_t_f", ctypes.c_double), ("coeff_t_b", ctypes.c_double),
        ("alpha", ctypes.c_double), ("mu", ctypes.c_double), ("muinv", ctypes.c_double), ("rho", ctypes.c_double),
        ("tbc_mask", ctypes.c_uint), ("tbc_phases", (ctypes.c_double * 2) * 4),
    ]


_PP = ctypes.POINTER(ctypes.c_void_p)
SIGNATURES.update({
    "qb200_spinor_convert": [_LAT, _P, _LAT, _P, _D, _P],
    "qb200_mrhs_pack": [_LAT, _I, _PP, _P, _P],
    "qb200_mrhs_unpack": [_LAT, _I, _P, _PP, _P],
    "qb200_dslash_mrhs": [_LAT, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, ctypes.POINTER(Coeffs), _UA, _P],
    "qb200_schur_apply_mrhs": [_LAT, _I, _OP, _I, _P, _P, _P, _P],
    "qb200_invert_cg_mrhs": [_LAT, _I, _OP, _P, _P, _D, _I, _P, _IP, _DP, _P],
    "qb200_invert_mixed_mrhs": [_LAT, _OP, _LAT, _OP, _I, _PP, _PP, _D, _D, _I, _I, _P, _P, _IP, _IP, _DP, _P],
    "qb200_invert_reliable_mrhs": [_LAT, _OP, _LAT, _OP, _I, _PP, _PP, _D, _D, _I, _I, _P, _P, _IP, _IP, _DP, _P],
})
INFO.update({
    "qb200_mrhs_spinor_elems": ([_LAT, _I], _LL),
    "qb200_cg_mrhs_workspace_bytes": ([_LAT, _I], _LL),
    "qb200_mixed_mrhs_workspace_bytes": ([_LAT, _LAT, _I, ctypes.POINTER(_LL)], _LL),
})
SIGNATURES.update({
    "qb200_hop_force": [_LAT, _I, _I, _P, _P, _P, _D, _D, _D, _U, _DA, _P, _P],
})


class BatchItem(ctypes.Structure):
    """ctypes mirror of `qb200_batch_item`."""
    _fields_ = [
        ("lat", Lattice), ("cb", ctypes.c_int),
        ("psi", ctypes.c_void_p), ("chi", ctypes.c_void_p), ("gauge", ctypes.c_void_p), ("clov", ctypes.c_void_p),
        ("out", ctypes.c_void_p), ("coeffs", Coeffs),
    ]


class LaunchCfg(ctypes.Structure):
    """ctypes mirror of `qb200_launch_cfg`."""
    _fields_ = [("grid", ctypes.c_int), ("block", ctypes.c_int)]


MAX_BATCH = 16
_BIP = ctypes.POINTER(BatchItem)
SIGNATURES.update({
    "qb200_dslash_batched": [_I, _I, _I, _I, _BIP, ctypes.POINTER(LaunchCfg), _P],
    "qb200_tune_batched": [_I, _I, _I, _I, _BIP, ctypes.POINTER(LaunchCfg), _DP, _P],
    "qb200_tune_cache_save": [ctypes.c_char_p],
    "qb200_tune_cache_load": [ctypes.c_char_p],
})
INFO.update({
    "qb200_tune_cache_clear": ([], None),
})
SIGNATURES.update({
    "qb200_pack_spinor": [_LAT, _I, _P, _P, _P],
    "qb200_unpack_spinor": [_LAT, _I, _P, _P, _P],
    "qb200_pack_gauge": [_LAT, _I, _I, _P, _I, _I, _P, _P],
    "qb200_pack_clover": [_LAT, _I, _P, _P, _P],
    "qb200_pack_full_clover": [_LAT, _I, _P, _P, _P],
})
INFO.update({
    "qb200_hop_force_elems": ([_LAT], _LL),
})

_lib = None


class QB200Error(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "error"), code, msg))
        self.code = code


def lib():
    """Load libqphix_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libqphix_b200.so is not built: run python qphix-codegen_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _I
        for name, (args, res) in INFO.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        raise QB200Error(rc, lib().qb200_last_error().decode())
    return rc


def uint8(vals):
    if vals is None:
        return None
    arr = (ctypes.c_uint * 8)(*[int(v) for v in vals])
    return arr


def phases(ph):
    if ph is None:
        return None
    flat = [float(v) for row in ph for v in row]
    return (ctypes.c_double * 8)(*flat)
