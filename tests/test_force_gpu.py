"""Backward kernels on the GPU: the link force of the hopping term against the
oracle, and the autograd bindings (hopping term, pseudofermion action)
against central finite differences along random su(3) directions."""
import numpy as np
import pytest
import torch

import helpers as H
import oracle as O
from qphix_b200 import autograd as AG
from qphix_b200 import fields, layout
from qphix_b200.lattice import F32, F64, Geometry

pytestmark = pytest.mark.gpu

EPS = 1e-4
NDIR = 8
FD_TOL = 1e-6


def _coeffs(p, tbc_mask):
    return dict(coeff_s=p["coeff_s"], coeff_t_f=p["coeff_t_f"], coeff_t_b=p["coeff_t_b"], tbc_mask=tbc_mask,
                tbc_phases=p["tbc_phases"])


@pytest.mark.parametrize("ft,S,V,comp12,proj", [
    (F64, 4, 4, False, False), (F64, 8, 16, True, True), (F64, 2, 2, False, True),
    (F32, 4, 8, False, False), (F32, 16, 16, True, True), (F32, 8, 8, False, True)])
@pytest.mark.parametrize("isign", [1, -1])
def test_force_vs_oracle(cuda, ft, S, V, comp12, proj, isign):
    g = Geometry(2 * max(S, 4), 8, 4, 4, soalen=S, veclen=V, ftype=ft, compress12=comp12, t_boundary=-1.0)
    f = H.make_fields(g, seed=610 + S, cb=1)
    p = H.op_params("wilson", "dslash", seed=3, tbc_mask=0b1101)
    kw = _coeffs(p, 0b1101)
    prm = O.make_params(**kw)
    want = O.hop_force(g, isign, 1, f["chi"], f["psi"], gauge=f["gauge"] if proj else None, params=prm)
    d = {k: H.to_torch(f[k], cuda) for k in ("chi", "psi", "gauge")}
    got = AG.hop_force(g, 1, isign, d["chi"], d["psi"], d["gauge"] if proj else None, **kw)
    torch.cuda.synchronize()
    got = got.cpu().double().numpy()
    scale = np.abs(want).max()
    # max error relative to the largest force component: FP32 1e-6, FP64 1e-12
    tol = 1e-12 if ft == F64 else 1e-6
    e = H.record("force vs oracle %s" % ("f64" if ft == F64 else "f32"), np.abs(got - want).max() / scale, tol)
    assert e <= tol, e


def _hop_loss(g, cb, isign, psi, U, chi, kw):
    out = AG.WilsonHop.apply(psi, U, g, cb, isign, kw)
    return (chi * out).sum()


@pytest.mark.parametrize("isign", [1, -1])
def test_wilson_hop_autograd_fd(cuda, isign):
    """FP64: dL/dU along 8 random su(3) directions and dL/dpsi against
    central differences of L = Re <chi, H(U) psi>."""
    g = Geometry(8, 8, 4, 4, soalen=4, ftype=F64, t_boundary=-1.0)
    cb = 0
    U = fields.random_gauge(g, seed=620).to(cuda).requires_grad_(True)
    psi = layout.pack_spinor(g, fields.random_spinor(g, seed=621)).to(cuda).requires_grad_(True)
    chi = layout.pack_spinor(g, fields.random_spinor(g, seed=622)).to(cuda)
    p = H.op_params("wilson", "dslash", seed=5, tbc_mask=0b1010)
    kw = _coeffs(p, 0b1010)
    L = _hop_loss(g, cb, isign, psi, U, chi, kw)
    L.backward()
    Ud = U.detach()
    with torch.no_grad():
        for k in range(NDIR):
            X = H.random_algebra(Ud.shape[:-2], seed=700 + k)
            lp = float(_hop_loss(g, cb, isign, psi, H.moved_links(Ud, X, EPS), chi, kw))
            lm = float(_hop_loss(g, cb, isign, psi, H.moved_links(Ud, X, -EPS), chi, kw))
            fd = (lp - lm) / (2 * EPS)
            an = H.directional(U.grad, X, Ud)
            assert abs(an - fd) <= FD_TOL * max(1.0, abs(fd)), (k, an, fd)
        # L is linear in psi: <grad, v> = L(psi + v) - L(psi) for any v
        v = layout.pack_spinor(g, fields.random_spinor(g, seed=623)).to(cuda)
        dl = float(_hop_loss(g, cb, isign, psi + v, Ud, chi, kw)) - float(L)
        assert abs(float((psi.grad * v).sum()) - dl) <= 1e-10 * max(1.0, abs(dl))


def test_wilson_hop_fp32_forward_fp64_check(cuda):
    """FP32 forward and backward agree with the FP64 path to FP32 precision."""
    g64 = Geometry(16, 8, 4, 4, soalen=8, ftype=F64)
    g32 = g64.with_(ftype=F32)
    U = fields.random_gauge(g64, seed=630).to(cuda)
    sp = fields.random_spinor(g64, seed=631)
    ch = fields.random_spinor(g64, seed=632)
    grads = {}
    for g in (g64, g32):
        Ux = U.to(torch.complex128 if g.ftype == F64 else torch.complex64).clone().requires_grad_(True)
        psi = layout.pack_spinor(g, sp).to(cuda).requires_grad_(True)
        chi = layout.pack_spinor(g, ch).to(cuda)
        _hop_loss(g, 1, 1, psi, Ux, chi, {"coeff_s": 0.9}).backward()
        grads[g.ftype] = (Ux.grad.to(torch.complex128), psi.grad.double())
    for a, b in zip(grads[F32], grads[F64]):
        assert float((a - b).abs().max()) <= 2e-5 * float(b.abs().max())


def _pseudofermion_fd(cuda, g, family, seed, tol=1e-14):
    """dS/dU of S = phi^dag (Mhat^dag Mhat)^-1 phi along NDIR random su(3)
    directions against central differences (FP64, CG to tol); returns the
    worst |analytic - fd| / max(1, |fd|)."""
    f, p = H.eo_setup(g, family, seed=seed, kappa=0.11)
    U = fields.random_gauge(g, seed=seed, device=cuda).requires_grad_(True)
    phi = H.to_torch(f["b"], cuda)
    T = lambda cs: tuple(H.to_torch(c, cuda) if c is not None else None for c in cs)
    clov, clov_dag = T(f["clov"]), T(f["clov_dag"])
    kw = dict(p, target_cb=1)
    S = AG.PseudofermionAction.apply(U, phi, g, family, kw, clov, clov_dag, tol)
    S.backward()
    Ud = U.detach()
    worst = 0.0
    with torch.no_grad():
        for k in range(NDIR):
            X = H.random_algebra(Ud.shape[:-2], seed=720 + k)
            sp = float(AG.PseudofermionAction.apply(H.moved_links(Ud, X, EPS), phi, g, family, kw, clov, clov_dag,
                                                    tol))
            sm = float(AG.PseudofermionAction.apply(H.moved_links(Ud, X, -EPS), phi, g, family, kw, clov, clov_dag,
                                                    tol))
            fd = (sp - sm) / (2 * EPS)
            an = H.directional(U.grad, X, Ud)
            worst = max(worst, abs(an - fd) / max(1.0, abs(fd)))
    return worst


@pytest.mark.parametrize("family", ["clover", "wilson", "tm", "tm_clover"])
def test_pseudofermion_action_fd(cuda, family):
    """S = phi^dag (Mhat^dag Mhat)^-1 phi: dS/dU along 8 random su(3)
    directions against central differences (FP64, CG to 1e-14)."""
    g = Geometry(8, 4, 4, 4, soalen=4, ftype=F64, t_boundary=-1.0)
    e = H.record("pseudofermion dS/dU vs central differences (8^3x4 family mix)",
                 _pseudofermion_fd(cuda, g, family, 640), FD_TOL)
    assert e <= FD_TOL, (family, e)


def test_pseudofermion_phi_grad(cuda):
    """dS/dphi = 2 (Mhat^dag Mhat)^-1 phi: S is quadratic in phi, so
    S(phi + v) - S(phi - v) = 2 <grad, v> exactly."""
    g = Geometry(8, 4, 4, 4, soalen=4, ftype=F64)
    f, p = H.eo_setup(g, "clover", seed=650, kappa=0.11)
    U = fields.random_gauge(g, seed=650).to(cuda)
    phi = H.to_torch(f["b"], cuda).requires_grad_(True)
    clov = tuple(H.to_torch(c, cuda) for c in f["clov"])
    kw = dict(p, target_cb=1)
    AG.PseudofermionAction.apply(U, phi, g, "clover", kw, clov, (None, None), 1e-14).backward()
    v = layout.pack_spinor(g, fields.random_spinor(g, seed=651)).to(cuda)
    with torch.no_grad():
        sp = float(AG.PseudofermionAction.apply(U, phi + v, g, "clover", kw, clov, (None, None), 1e-14))
        sm = float(AG.PseudofermionAction.apply(U, phi - v, g, "clover", kw, clov, (None, None), 1e-14))
    assert abs((sp - sm) - 2 * float((phi.grad * v).sum())) <= 1e-8 * max(1.0, abs(sp - sm))
