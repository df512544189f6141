"""The oracle's link force (the backward of the hopping term, which the
reference does not have) against central finite differences of the forward
operator: of the oracle's own FP64 dslash and, where the library is built, of
the reference's scalar FP64 kernels.  Eight random su(3) directions, eps 1e-4."""
import numpy as np
import pytest
import torch

import helpers as H
import oracle as O
from qphix_b200 import autograd as AG
from qphix_b200 import layout
from qphix_b200.lattice import F64, Geometry

EPS = 1e-4
NDIR = 8


def _loss(g, cb, isign, U, psi, chi, prm, ref=None):
    gauge = layout.pack_gauge(g, U, cb, torch.float64).numpy()
    if ref is None:
        out = O.dslash(g, "wilson", "dslash", isign, cb, psi, gauge, params=prm)
    else:
        out = O.ref_dslash(ref, g, "wilson", "dslash", isign, cb, O.aligned(psi), O.aligned(gauge), params=prm)
    return float(np.dot(chi, out[: g.spinor_elems]))


def _setup(g, seed, tbc_mask):
    f = H.make_fields(g, seed=seed)
    p = H.op_params("wilson", "dslash", seed=seed, tbc_mask=tbc_mask)
    prm = O.make_params(coeff_s=p["coeff_s"], coeff_t_f=p["coeff_t_f"], coeff_t_b=p["coeff_t_b"],
                        tbc_mask=tbc_mask, tbc_phases=p["tbc_phases"])
    return f, p, prm


@pytest.mark.parametrize("isign", [1, -1])
@pytest.mark.parametrize("cb", [0, 1])
@pytest.mark.parametrize("tbc_mask", [0, 0b1011])
def test_oracle_force_vs_fd(isign, cb, tbc_mask):
    g = Geometry(4, 4, 4, 4, soalen=2, ftype=F64, t_boundary=-1.0)
    f, p, prm = _setup(g, 500 + cb, tbc_mask)
    U = f["U"]
    F = O.hop_force(g, isign, cb, f["chi"], f["psi"], params=prm)
    gU = AG.links_grad(g, cb, torch.from_numpy(F))
    for k in range(NDIR):
        X = H.random_algebra(U.shape[:-2], seed=900 + k)
        fd = (_loss(g, cb, isign, H.moved_links(U, X, EPS), f["psi"], f["chi"], prm)
              - _loss(g, cb, isign, H.moved_links(U, X, -EPS), f["psi"], f["chi"], prm)) / (2 * EPS)
        an = H.directional(gU, X, U)
        assert abs(an - fd) <= 1e-6 * max(1.0, abs(fd)), (k, an, fd)


@pytest.mark.parametrize("comp12", [False, True])
def test_oracle_projected_force(comp12):
    """gauge given -> TA(F U^dag) per stored link, 12-real links reconstructed."""
    g = Geometry(4, 4, 4, 4, soalen=2, ftype=F64, compress12=comp12)
    f, p, prm = _setup(g, 510, 0)
    gauge = f["gauge"]                                            # 12 reals per link when comp12
    F = torch.from_numpy(O.hop_force(g, 1, 0, f["chi"], f["psi"], params=prm))
    P = torch.from_numpy(O.hop_force(g, 1, 0, f["chi"], f["psi"], gauge=gauge, params=prm))
    links = layout.site_links(g, f["U"], 0)                       # (nt,nz,ny,nxh,8,3,3)
    want = AG.link_force(links, AG.force_sites(g, F))
    got = AG.force_sites(g, P)
    assert torch.allclose(got, want, atol=1e-12, rtol=0)
    # su(3): traceless and anti-Hermitian
    assert torch.allclose(got, -got.conj().transpose(-1, -2), atol=1e-13)
    assert float(torch.diagonal(got, dim1=-2, dim2=-1).sum(-1).abs().max()) < 1e-13


def test_projected_force_directional():
    """sum Re tr(X^dag P) of the folded projected force equals the directional
    derivative of the unprojected one."""
    g = Geometry(4, 4, 4, 4, soalen=1, ftype=F64)
    f, p, prm = _setup(g, 520, 0)
    U = f["U"]
    gU = AG.links_grad(g, 1, torch.from_numpy(O.hop_force(g, -1, 1, f["chi"], f["psi"], params=prm)))
    gauge1 = layout.pack_gauge(g, U, 1, torch.float64).numpy()
    Pf = AG.links_grad(g, 1, torch.from_numpy(O.hop_force(g, -1, 1, f["chi"], f["psi"], gauge=gauge1,
                                                          params=prm)))
    for k in range(3):
        X = H.random_algebra(U.shape[:-2], seed=930 + k)
        a = H.directional(gU, X, U)
        b = float((X.conj() * Pf).real.sum())
        assert abs(a - b) <= 1e-12 * max(1.0, abs(a))


@pytest.mark.parametrize("isign", [1, -1])
def test_oracle_force_vs_reference_fd(isign):
    """The FP64 gradient from the reference's scalar kernels by central
    differences agrees with the oracle's analytic force."""
    name = "scalar_f64"
    if not O.ref_available(name):
        pytest.skip("reference kernels %s not built" % name)
    g = Geometry(4, 4, 4, 4, soalen=1, veclen=1, ftype=F64, t_boundary=-1.0)
    f, p, prm = _setup(g, 530, 0b0101)
    U = f["U"]
    gU = AG.links_grad(g, 1, torch.from_numpy(O.hop_force(g, isign, 1, f["chi"], f["psi"], params=prm)))
    for k in range(NDIR):
        X = H.random_algebra(U.shape[:-2], seed=940 + k)
        fd = (_loss(g, 1, isign, H.moved_links(U, X, EPS), f["psi"], f["chi"], prm, ref=name)
              - _loss(g, 1, isign, H.moved_links(U, X, -EPS), f["psi"], f["chi"], prm, ref=name)) / (2 * EPS)
        an = H.directional(gU, X, U)
        assert abs(an - fd) <= 1e-6 * max(1.0, abs(fd)), (k, an, fd)
