"""The differentiable Wilson-clover configuration at its own size, 24^3 x 48.

  1. the link force of the hopping term, FP32 (the forward precision) and
     FP64, plain and su(3)-projected, against the FP64 oracle's force, whose
     derivative is pinned by tests/test_force_oracle.py to central
     differences of the reference's scalar kernels;
  2. L = Re <chi, D(U) psi>: dL/dU along 8 random su(3) directions against
     central differences (eps = 1e-4, FP64 check path), dL/dpsi (the dagger
     dslash) against the exact linear change, and the FP32 forward and
     backward against the FP64 ones;
  3. the pseudofermion action S = phi^dag (Mhat^dag Mhat)^-1 phi of the
     Wilson-clover even-odd operator (Gaussian phi): dS/dU along 8 random
     su(3) directions against central differences (FP64, CG to 1e-14)."""
import numpy as np
import pytest
import torch

import helpers as H
import oracle as O
from qphix_b200 import autograd as AG
from qphix_b200 import fields, layout
from qphix_b200.lattice import F32, F64, Geometry
from test_force_gpu import EPS, FD_TOL, NDIR, _coeffs, _hop_loss, _pseudofermion_fd

pytestmark = pytest.mark.gpu
DIMS = (24, 24, 24, 48)


@pytest.mark.parametrize("ft", [F32, F64])
def test_config5_force_24c48_vs_fp64_oracle(cuda, ft):
    g = Geometry(*DIMS, soalen=4, ftype=ft, compress12=False, t_boundary=-1.0)
    f = H.make_fields(g, seed=5100, cb=0)
    p = H.op_params("wilson", "dslash", seed=7, tbc_mask=0)
    kw = _coeffs(p, 0)
    prm = O.make_params(**kw)
    d = {k: H.to_torch(f[k], cuda) for k in ("chi", "psi", "gauge")}
    tol = 1e-12 if ft == F64 else 1e-6
    for proj in (False, True):
        for isign in (1, -1):
            want = O.hop_force(g, isign, 0, f["chi"], f["psi"], gauge=f["gauge"] if proj else None, params=prm)
            got = AG.hop_force(g, 0, isign, d["chi"], d["psi"], d["gauge"] if proj else None, **kw)
            torch.cuda.synchronize()
            got = got.cpu().double().numpy()
            e = H.record("config5 24^3x48 force %s vs fp64 oracle" % ("f64" if ft == F64 else "f32"),
                         np.abs(got - want).max() / np.abs(want).max(), tol)
            assert e <= tol, (proj, isign, e)


def test_config5_hop_autograd_24c48(cuda):
    g = Geometry(*DIMS, soalen=4, ftype=F64, t_boundary=-1.0)
    cb = 0
    U = fields.random_gauge(g, seed=5200, device=cuda).requires_grad_(True)
    sp = fields.random_spinor(g, seed=5201, device=cuda)
    ch = fields.random_spinor(g, seed=5202, device=cuda)
    psi = layout.pack_spinor(g, sp).requires_grad_(True)
    chi = layout.pack_spinor(g, ch)
    kw = {"coeff_s": 0.125, "coeff_t_f": 0.125, "coeff_t_b": 0.125}
    L = _hop_loss(g, cb, 1, psi, U, chi, kw)
    L.backward()
    Ud = U.detach()
    worst = 0.0
    with torch.no_grad():
        for k in range(NDIR):
            X = H.random_algebra(Ud.shape[:-2], seed=5300 + k).to(cuda)
            lp = float(_hop_loss(g, cb, 1, psi, H.moved_links(Ud, X, EPS), chi, kw))
            lm = float(_hop_loss(g, cb, 1, psi, H.moved_links(Ud, X, -EPS), chi, kw))
            fd = (lp - lm) / (2 * EPS)
            an = H.directional(U.grad, X, Ud)
            worst = max(worst, abs(an - fd) / max(1.0, abs(fd)))
        v = layout.pack_spinor(g, fields.random_spinor(g, seed=5203, device=cuda))
        dl = float(_hop_loss(g, cb, 1, psi + v, Ud, chi, kw)) - float(L)
        lin = abs(float((psi.grad * v).sum()) - dl) / max(1.0, abs(dl))
    H.record("config5 24^3x48 dL/dU vs central differences", worst, FD_TOL)
    H.record("config5 24^3x48 dL/dpsi vs the exact linear change", lin, 1e-10)
    assert worst <= FD_TOL, worst
    assert lin <= 1e-10, lin
    # FP32 forward and backward against the FP64 path
    g32 = g.with_(ftype=F32)
    U32 = Ud.to(torch.complex64).clone().requires_grad_(True)
    psi32 = layout.pack_spinor(g32, sp).requires_grad_(True)
    _hop_loss(g32, cb, 1, psi32, U32, layout.pack_spinor(g32, ch), kw).backward()
    eu = float((U32.grad.to(torch.complex128) - U.grad).abs().max() / U.grad.abs().max())
    ep = float((psi32.grad.double() - psi.grad).abs().max() / psi.grad.abs().max())
    H.record("config5 24^3x48 fp32 backward vs fp64", max(eu, ep), 2e-5)
    assert eu <= 2e-5 and ep <= 2e-5, (eu, ep)


def test_config5_pseudofermion_24c48_fd(cuda):
    g = Geometry(*DIMS, soalen=4, ftype=F64, t_boundary=-1.0)
    e = H.record("config5 24^3x48 pseudofermion dS/dU vs central differences", _pseudofermion_fd(cuda, g, "clover",
                                                                                                  5400), FD_TOL)
    assert e <= FD_TOL, e
