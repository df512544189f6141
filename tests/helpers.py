"""Shared fixtures: seeded fields in the QPhiX layouts and comparison metrics."""
import os
import sys

import numpy as np
import torch

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "qphix-codegen_b200")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

from qphix_b200 import fields, layout  # noqa: E402
from qphix_b200.lattice import BF16, F16, F16N, F32, F64, Geometry  # noqa: E402

# numpy carries bfloat16 arrays as their uint16 bit patterns
NP_DTYPE = {F32: np.float32, F64: np.float64, F16: np.float16, F16N: np.float16, BF16: np.uint16}


def to_np(t):
    """storage tensor -> numpy array (bfloat16 as uint16 bits)"""
    t = t.detach().cpu().contiguous()
    if t.dtype == torch.bfloat16:
        return t.view(torch.int16).numpy().view(np.uint16)
    return t.numpy()


def to_torch(a, device=None):
    """numpy storage array -> torch tensor (uint16 bits -> bfloat16)"""
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint16:
        t = torch.from_numpy(a.view(np.int16)).view(torch.bfloat16)
    else:
        t = torch.from_numpy(a)
    return t.to(device) if device is not None else t
FAMILIES = ("wilson", "clover", "tm", "tm_clover")
KERNELS = ("dslash", "achimbdpsi")


def make_fields(g: Geometry, seed=1234, cb=0, inverse_clover=False):
    """Seeded inputs for checkerboard cb (out) / 1-cb (psi), as numpy arrays
    in the storage type of g.  Keys: psi, chi, gauge, clover, fclover."""
    U = fields.random_gauge(g, seed=seed)
    psi = fields.random_spinor(g, seed=seed + 1)
    chi = fields.random_spinor(g, seed=seed + 2)
    A = fields.random_clover(g, seed=seed + 3)
    if inverse_clover:
        A = fields.invert_blocks(A)
    F = fields.random_full_clover(g, seed=seed + 4)
    out = {
        "U": U,
        "psi": to_np(layout.pack_spinor(g, psi)),
        "chi": to_np(layout.pack_spinor(g, chi)),
        "gauge": to_np(layout.pack_gauge(g, U, cb)),
        "clover": to_np(layout.pack_clover(g, A)),
        "fclover": to_np(layout.pack_full_clover(g, F)),
    }
    return out


# Parity tolerances (per site component, relative, floored at the site's rms
# component; see site_rel_err), GPU result against the FP64 oracle's
# unrounded result on the same stored inputs:
#   FP32 1e-6 and FP64 1e-13 (the accuracy the operator must keep);
#   FP16 (IEEE binary16, the reference's `half`) and FP16 + per-site norm
#   1e-3: storing the result rounds each component to 11 significant bits,
#   at most 2^-11 = 4.9e-4 of max(|component|, site rms);
#   BF16 4e-3: the format limit.  8 significant bits give a unit roundoff of
#   2^-8 = 3.9e-3 for the one rounding of the stored result, which no
#   arithmetic can beat; 1e-3 is out of reach for this format.
TOL = {F32: 1e-6, F64: 1e-13, F16: 1e-3, F16N: 1e-3, BF16: 4e-3}

# worst error seen per parity check, printed at the end of the session
PARITY = {}


def record(name, err, tol=None):
    """Keep the worst error of a named parity check (and its bound)."""
    old = PARITY.get(name)
    if old is None or err > old[0]:
        PARITY[name] = (float(err), tol)
    return err


def site_rel_err(g: Geometry, a, b, gb: Geometry = None):
    """max over components of |a-b| / max(|b_i|, |b_site|/sqrt(24)) -- the
    per-component relative error with a floor at the site's rms component.
    a is a spinor array of lattice g, b of lattice gb (default g), so that a
    16-bit result can be compared with an FP64 one."""
    gb = gb if gb is not None else g
    ta = layout.unpack_spinor(g, to_torch(np.asarray(a)[: g.spinor_elems])).numpy().reshape(-1, 12)
    tb = layout.unpack_spinor(gb, to_torch(np.asarray(b)[: gb.spinor_elems])).numpy().reshape(-1, 12)
    ra = np.concatenate([ta.real, ta.imag], axis=1)
    rb = np.concatenate([tb.real, tb.imag], axis=1)
    site = np.sqrt((rb ** 2).sum(axis=1, keepdims=True) / 24.0)
    den = np.maximum(np.abs(rb), site)
    den = np.where(den == 0, 1.0, den)
    return float((np.abs(ra - rb) / den).max())


def as_f64(g: Geometry, a):
    """A stored spinor array of lattice g as an FP64 array of the same layout
    (ftype F64): the values exactly as stored, decoded."""
    t = layout.unpack_spinor(g, to_torch(np.asarray(a)[: g.spinor_elems]))
    return layout.pack_spinor(g.with_(ftype=F64), t, torch.float64).numpy()


def face_rel_err(a, b):
    """face records (n, 12) as float64: max over components of |a-b| /
    max(|b_i|, rms of the record)"""
    a = np.asarray(a, dtype=np.float64).reshape(-1, 12)
    b = np.asarray(b, dtype=np.float64).reshape(-1, 12)
    rms = np.sqrt((b ** 2).mean(axis=1, keepdims=True))
    den = np.maximum(np.abs(b), rms)
    den = np.where(den == 0, 1.0, den)
    return float((np.abs(a - b) / den).max()) if a.size else 0.0


def op_params(family, kernel, seed=0, tbc_mask=0, accumulate=None, coeff=None):
    """Scalar parameters used throughout the parity tests."""
    rng = np.random.default_rng(seed)
    ph = rng.normal(size=(4, 2))
    ph = ph / np.linalg.norm(ph, axis=1, keepdims=True)
    p = dict(coeff_s=0.91 if coeff is None else coeff, coeff_t_f=1.07, coeff_t_b=0.83,
             alpha=1.3 if kernel == "achimbdpsi" else 1.0,
             mu=0.21 if family == "tm" else 0.0,
             muinv=0.77 if family == "tm" else 1.0,
             rho=0.17 if family in ("clover", "tm_clover") and kernel == "achimbdpsi" else 0.0,
             tbc_mask=tbc_mask, tbc_phases=ph.tolist(), accumulate=accumulate)
    return p


def compress_gauge(g18: Geometry, gauge18):
    """12-real gauge array (rows 0,1 of each stored link) from an 18-real one."""
    a = np.asarray(gauge18).reshape(g18.ntiles, 8, 3, 3, 2, g18.veclen)
    return np.ascontiguousarray(a[:, :, :2]).reshape(-1)


def load_golden(ft):
    """The golden vectors produced by tests/golden/make_golden.py."""
    name = {F32: "scalar_f32", F64: "scalar_f64"}[ft]
    path = os.path.join(REPO, "tests", "golden", "ref_%s_4x4x4x4.npz" % name)
    return dict(np.load(path))


def eo_setup(g: Geometry, family, seed=900, target_cb=1, kappa=0.12):
    """Fields and parameters of the even-odd operator of `family` on both
    checkerboards (numpy, storage type of g).  Returns (fields, params):
    fields: gauge[cb], clov[cb] (A on target_cb, A^-1 on the other; dense
    F / F^-1 for tm_clover), clov_dag[cb] (tm_clover), b (source on target_cb)."""
    dt = NP_DTYPE[g.ftype]
    U = fields.random_gauge(g, seed=seed)
    other = 1 - target_cb
    f = {"gauge": [None, None], "clov": [None, None], "clov_dag": [None, None]}
    for cb in (0, 1):
        f["gauge"][cb] = layout.pack_gauge(g, U, cb, torch.float64).numpy().astype(dt)
    if family == "clover":
        A_t = fields.random_clover(g, seed=seed + 1)
        A_o = fields.random_clover(g, seed=seed + 2)
        f["clov"][target_cb] = layout.pack_clover(g, A_t, torch.float64).numpy().astype(dt)
        f["clov"][other] = layout.pack_clover(g, fields.invert_blocks(A_o), torch.float64).numpy().astype(dt)
    if family == "tm_clover":
        F_t = fields.random_full_clover(g, seed=seed + 1)
        F_o = fields.invert_blocks(fields.random_full_clover(g, seed=seed + 2))
        f["clov"][target_cb] = layout.pack_full_clover(g, F_t, torch.float64).numpy().astype(dt)
        f["clov"][other] = layout.pack_full_clover(g, F_o, torch.float64).numpy().astype(dt)
        f["clov_dag"][target_cb] = layout.pack_full_clover(g, F_t.conj().transpose(-1, -2),
                                                           torch.float64).numpy().astype(dt)
        f["clov_dag"][other] = layout.pack_full_clover(g, F_o.conj().transpose(-1, -2),
                                                       torch.float64).numpy().astype(dt)
    f["b"] = layout.pack_spinor(g, fields.random_spinor(g, seed=seed + 3), torch.float64).numpy().astype(dt)
    alpha = 1.0 if family in ("clover", "tm_clover") else 4.2
    mu_t = 0.3
    p = dict(coeff_s=kappa, coeff_t_f=kappa, coeff_t_b=kappa, alpha=alpha,
             mu=mu_t / alpha if family == "tm" else 0.0,
             muinv=alpha / (alpha ** 2 + mu_t ** 2) if family == "tm" else 1.0,
             rho=0.05 if family in ("clover", "tm_clover") else 0.0, tbc_mask=0, tbc_phases=None)
    return f, p


def oracle_schur(g: Geometry, family, f, p, x, isign=1, target_cb=1):
    """Mhat x (or Mhat^dag x) with the oracle: plain kernel on the other
    checkerboard (hops scaled by 1/alpha for Wilson), achimbdpsi on target."""
    import oracle as O
    other = 1 - target_cb
    sc = 1.0 / p["alpha"] if family == "wilson" else 1.0
    clov = f["clov_dag"] if (family == "tm_clover" and isign < 0) else f["clov"]
    q = dict(p)
    q.pop("tbc_phases")
    p1 = O.make_params(**dict(q, coeff_s=p["coeff_s"] * sc, coeff_t_f=p["coeff_t_f"] * sc,
                              coeff_t_b=p["coeff_t_b"] * sc))
    tmp = O.dslash(g, family, "dslash", isign, other, x, f["gauge"][other], clover=clov[other], params=p1)
    p2 = O.make_params(**q)
    return O.dslash(g, family, "achimbdpsi", isign, target_cb, tmp, f["gauge"][target_cb], chi=x,
                    clover=clov[target_cb], params=p2)


def random_algebra(shape, seed):
    """Gaussian traceless anti-Hermitian 3x3 matrices (an su(3) direction per link)."""
    gen = torch.Generator().manual_seed(seed)
    m = torch.complex(torch.randn(tuple(shape) + (3, 3), generator=gen, dtype=torch.float64),
                      torch.randn(tuple(shape) + (3, 3), generator=gen, dtype=torch.float64))
    a = 0.5 * (m - m.conj().transpose(-1, -2))
    tr = torch.diagonal(a, dim1=-2, dim2=-1).sum(-1) / 3.0
    return a - tr[..., None, None] * torch.eye(3, dtype=a.dtype)


def moved_links(U, X, eps):
    """exp(eps X) U, link by link."""
    return torch.linalg.matrix_exp(eps * X.to(U.device)) @ U


def directional(gU, X, U):
    """sum Re <gU, X U>: the derivative along U -> exp(eps X) U of a loss whose
    link gradient (torch convention) is gU."""
    return float((gU.conj() * (X.to(U.device) @ U)).real.sum())
