"""Parity at the benchmark configurations' own sizes, through the C-ABI.

  1. plain Wilson dslash, isign +1 and -1, 8^3 x 16, FP32, 18-real links,
     SOALEN 4: against the reference's own generated kernels (AVX512 SOALEN 4
     and scalar SOALEN 1, oracle/_ref) and the FP64 oracle;
  2. clover A.chi - b.D.psi and the plain clover dslash with A^-1 (the
     inverse-clover variant), 32^3 x 64, FP32, 12-real links, SOALEN 16,
     b = kappa = 0.125: against the reference's AVX512 SOALEN 16 kernels (on
     the very same arrays) and the FP64 oracle;
  3. twisted mass and twisted-mass clover, 48^3 x 96, FP16 + per-site norm,
     SOALEN 8, mu = 0.01, kappa = 0.16: against the FP64 oracle (no reference
     kernel stores this format).

Metric: per site component, relative, floored at the site rms
(helpers.site_rel_err); bounds helpers.TOL (FP32 1e-6, FP16 + norm 1e-3)
against the FP64 oracle.  A reference kernel computes in FP32 too and
carries its own rounding error, which at 32^3 x 64 reaches 1e-6 of a
component by itself; the GPU result is held to within 1e-6 of it beyond that
error, component by component (ref_bound), and both errors are recorded.
Fields are generated on the GPU (seeded) and copied to the host for the
CPU checkers."""
import numpy as np
import pytest
import torch

import helpers as H
import oracle as O
from qphix_b200 import fields, layout, ops
from qphix_b200.lattice import F16N, F32, F64, Geometry

pytestmark = pytest.mark.gpu


def _canon_fields(g, dev, seed, clover=None):
    """seeded canonical fields on the GPU; clover: None, "A" (I + 0.1 H),
    "Ainv" (its block inverse) or "F" (dense FullCloverBlock)"""
    f = {"U": fields.random_gauge(g, seed=seed, device=dev),
         "psi": fields.random_spinor(g, seed=seed + 1, device=dev),
         "chi": fields.random_spinor(g, seed=seed + 2, device=dev)}
    if clover == "F":
        f["fclover"] = fields.random_full_clover(g, seed=seed + 3, device=dev)
    elif clover is not None:
        A = fields.random_clover(g, seed=seed + 3, device=dev)
        f["clover"] = fields.invert_blocks(A) if clover == "Ainv" else A
    return f


def _packed(g, c, cb):
    """the canonical fields in the tile layouts of g (torch, on c's device)"""
    d = {"psi": layout.pack_spinor(g, c["psi"]), "chi": layout.pack_spinor(g, c["chi"]),
         "gauge": layout.pack_gauge(g, c["U"], cb), "clover": None}
    if "clover" in c:
        d["clover"] = layout.pack_clover(g, c["clover"])
    if "fclover" in c:
        d["clover"] = layout.pack_full_clover(g, c["fclover"])
    return d


def _host(t):
    return None if t is None else O.aligned(H.to_np(t))


def _components(g, a):
    """the spinor array a of lattice g as (sites, 24) float64 components"""
    t = layout.unpack_spinor(g, H.to_torch(np.asarray(a)[: g.spinor_elems])).numpy().reshape(-1, 12)
    return np.concatenate([t.real, t.imag], axis=1).astype(np.float64)


def ref_bound(g, gpu, gr, ref, g64, exact, tol):
    """per component: |gpu - ref| <= tol * max(|exact_i|, site rms) + |ref - exact|.
    Returns (worst |gpu - ref| / den, worst |ref - exact| / den, holds)."""
    a, r, x = _components(g, gpu), _components(gr, ref), _components(g64, exact)
    den = np.maximum(np.abs(x), np.sqrt((x ** 2).sum(axis=1, keepdims=True) / 24.0))
    den = np.where(den == 0, 1.0, den)
    d_gr = np.abs(a - r) / den
    d_rx = np.abs(r - x) / den
    return float(d_gr.max()), float(d_rx.max()), bool((d_gr <= tol + d_rx).all())


def _gpu(g, fam, kernel, isign, cb, d, pp):
    out = torch.zeros_like(d["psi"])
    ops.dslash(g, fam, kernel, isign, cb, d["psi"], out, d["gauge"], chi=d["chi"], clover=d["clover"], **pp)
    torch.cuda.synchronize()
    return H.to_np(out)


@pytest.mark.parametrize("veclen", [4, 16])
def test_config1_wilson_8c16_vs_reference(cuda, veclen):
    if not (O.ref_available("avx512_f32_s4") and O.ref_available("scalar_f32")):
        pytest.fail("reference kernels missing from oracle/_ref (python oracle/ref_build.py)")
    dims = (8, 8, 8, 16)
    g = Geometry(*dims, soalen=4, veclen=veclen, ftype=F32, compress12=False, t_boundary=-1.0)
    c = _canon_fields(g, cuda, seed=2100)
    refs = {}
    for name in ("avx512_f32_s4", "scalar_f32"):
        info = O.ref_info(name)
        refs[name] = g.with_(soalen=info["soalen"], veclen=info["veclen"])
    pp = dict(coeff_s=1.0, coeff_t_f=1.0, coeff_t_b=1.0)
    prm = O.make_params(**pp)
    for cb in (0, 1):
        d = _packed(g, c, cb)
        h = {k: None if v is None else H.to_np(v) for k, v in d.items()}
        for isign in (1, -1):
            a = _gpu(g, "wilson", "dslash", isign, cb, d, pp)
            b = O.dslash(g, "wilson", "dslash", isign, cb, h["psi"], h["gauge"], params=prm, fp64_out=True)
            e = H.record("config1 wilson 8^3x16 s4 v%d vs fp64 oracle" % veclen,
                         H.site_rel_err(g, a, b, g.with_(ftype=F64)), H.TOL[F32])
            assert e < H.TOL[F32], (cb, isign, e)
            for name, gr in refs.items():
                dr = {k: _host(v) for k, v in _packed(gr, c, cb).items()}
                r = O.ref_dslash(name, gr, "wilson", "dslash", isign, cb, dr["psi"], dr["gauge"], params=prm)
                d_gr, d_rx, ok = ref_bound(g, a, gr, r, g.with_(ftype=F64), b, H.TOL[F32])
                H.record("config1 wilson 8^3x16 s4 v%d vs reference %s" % (veclen, name), d_gr, H.TOL[F32])
                H.record("config1 wilson 8^3x16 reference %s vs fp64 oracle" % name, d_rx)
                assert ok, (name, cb, isign, d_gr, d_rx)


@pytest.mark.parametrize("variant", ["achimbdpsi", "inverse_clover"])
def test_config2_clover_32c64_vs_reference(cuda, variant):
    name = "avx512_f32_s16"
    if not O.ref_available(name):
        pytest.fail("reference kernels missing from oracle/_ref (python oracle/ref_build.py)")
    info = O.ref_info(name)
    assert info["soalen"] == 16 and info["veclen"] == 16
    g = Geometry(32, 32, 32, 64, soalen=16, veclen=16, ftype=F32, compress12=True, t_boundary=-1.0)
    c = _canon_fields(g, cuda, seed=2200, clover="Ainv" if variant == "inverse_clover" else "A")
    kernel = "achimbdpsi" if variant == "achimbdpsi" else "dslash"
    pp = dict(coeff_s=0.125, coeff_t_f=0.125, coeff_t_b=0.125, rho=0.0)
    prm = O.make_params(**pp)
    cb = 0
    d = _packed(g, c, cb)
    del c
    h = {k: _host(v) for k, v in d.items()}
    for isign in (1, -1):
        a = _gpu(g, "clover", kernel, isign, cb, d, pp)
        b = O.dslash(g, "clover", kernel, isign, cb, h["psi"], h["gauge"], chi=h["chi"], clover=h["clover"],
                     params=prm, fp64_out=True)
        e = H.record("config2 clover %s 32^3x64 s16 vs fp64 oracle" % variant,
                     H.site_rel_err(g, a, b, g.with_(ftype=F64)), H.TOL[F32])
        assert e < H.TOL[F32], (isign, e)
        # the reference kernels on the very same arrays (same layout)
        r = O.ref_dslash(name, g, "clover", kernel, isign, cb, h["psi"], h["gauge"], chi=h["chi"],
                         clover=h["clover"], params=prm)
        d_gr, d_rx, ok = ref_bound(g, a, g, r, g.with_(ftype=F64), b, H.TOL[F32])
        H.record("config2 clover %s 32^3x64 s16 vs reference %s" % (variant, name), d_gr, H.TOL[F32])
        H.record("config2 clover %s 32^3x64 reference %s vs fp64 oracle" % (variant, name), d_rx)
        assert ok, (isign, d_gr, d_rx)


@pytest.mark.parametrize("family", ["tm", "tm_clover"])
def test_config3_twisted_48c96_f16n_vs_fp64_oracle(cuda, family):
    g = Geometry(48, 48, 48, 96, soalen=8, veclen=8, ftype=F16N, compress12=True, t_boundary=-1.0)
    c = _canon_fields(g, cuda, seed=2300, clover="F" if family == "tm_clover" else None)
    kappa, mu = 0.16, 0.01
    alpha = 1.0 / (2 * kappa)
    cb = 1
    d = _packed(g, c, cb)
    del c
    h = {k: None if v is None else H.to_np(v) for k, v in d.items()}
    g64 = g.with_(ftype=F64)
    for kernel, isign in (("dslash", 1), ("achimbdpsi", -1)):
        if family == "tm":
            pp = dict(coeff_s=0.5, coeff_t_f=0.5, coeff_t_b=0.5, alpha=alpha, mu=mu / alpha,
                      muinv=alpha / (alpha ** 2 + mu ** 2))
        else:
            pp = dict(coeff_s=0.5, coeff_t_f=0.5, coeff_t_b=0.5, rho=0.0)
        a = _gpu(g, family, kernel, isign, cb, d, pp)
        b = O.dslash(g, family, kernel, isign, cb, h["psi"], h["gauge"], chi=h["chi"], clover=h["clover"],
                     params=O.make_params(**pp), fp64_out=True)
        e = H.record("config3 %s 48^3x96 f16n s8 vs fp64 oracle" % family, H.site_rel_err(g, a, b, g64),
                     H.TOL[F16N])
        assert e < H.TOL[F16N], (kernel, isign, e)
