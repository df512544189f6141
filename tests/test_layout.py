"""Layout converters and synthetic fields (host logic)."""
import numpy as np
import torch

from qphix_b200 import fields, layout
from qphix_b200.lattice import F32, Geometry


def test_spinor_roundtrip_with_padding():
    for g in (Geometry(8, 8, 4, 4, soalen=4, veclen=8, pad_xy=3, pad_xyz=7), Geometry(4, 4, 2, 2, soalen=1),
              Geometry(32, 2, 2, 2, soalen=16)):
        sp = fields.random_spinor(g, seed=3)
        flat = layout.pack_spinor(g, sp, torch.float64)
        assert flat.numel() == g.spinor_elems
        assert torch.equal(layout.unpack_spinor(g, flat), sp)


def test_spinor_element_addressing():
    """Component (c, s, ri) of site xcb sits at block*24S + ((c*4+s)*2+ri)*S + xcb%S."""
    g = Geometry(8, 4, 2, 2, soalen=2, veclen=2, pad_xy=1, pad_xyz=2)
    sp = fields.random_spinor(g, seed=9)
    flat = layout.pack_spinor(g, sp, torch.float64).numpy()
    t, z, y, xcb, s, c = 1, 1, 2, 3, 2, 1
    blk = t * g.Pxyz + z * g.Pxy + y * g.nvecs + xcb // g.soalen
    e = blk * 24 * g.soalen + ((c * 4 + s) * 2) * g.soalen + xcb % g.soalen
    assert flat[e] == sp[t, z, y, xcb, s, c].real
    assert flat[e + g.soalen] == sp[t, z, y, xcb, s, c].imag


def test_su3_and_twelve_real_reconstruction():
    g = Geometry(4, 4, 4, 4, soalen=2, veclen=4, compress12=True)
    U = fields.random_gauge(g, seed=1)
    eye = torch.eye(3, dtype=U.dtype)
    assert torch.allclose(U @ U.conj().transpose(-1, -2), eye, atol=1e-12)
    assert torch.allclose(torch.linalg.det(U), torch.ones((), dtype=U.dtype), atol=1e-12)
    G = layout.unpack_gauge(g, layout.pack_gauge(g, U, 0, torch.float64))
    full = layout.site_links(g, U, 0).transpose(-1, -2)
    assert torch.allclose(G, full[..., :2, :])
    # row 2 = conj(row0 x row1), the reconstruction the kernels use
    r2 = torch.linalg.cross(full[..., 0, :], full[..., 1, :], dim=-1).conj()
    assert torch.allclose(r2, full[..., 2, :], atol=1e-12)


def test_backward_link_is_forward_link_of_neighbour():
    g = Geometry(4, 4, 4, 4, soalen=1)
    U = fields.random_gauge(g, seed=2)
    L0 = layout.site_links(g, U, 0)
    # site (xcb=0, y=0, z=0, t=1) on cb 0: x = (0+0+1+0)&1 = 1; its t-back link is U_t(x=1,y=0,z=0,t=0)
    assert torch.equal(L0[1, 0, 0, 0, 6], U[3, 0, 0, 0, 1])
    assert torch.equal(L0[1, 0, 0, 0, 7], U[3, 1, 0, 0, 1])


def test_clover_roundtrip_and_positivity():
    g = Geometry(8, 4, 2, 2, soalen=4, veclen=8)
    A = fields.random_clover(g, seed=4)
    assert torch.allclose(A, A.conj().transpose(-1, -2))
    assert float(torch.linalg.eigvalsh(A).min()) > 0.85
    assert torch.allclose(layout.unpack_clover(g, layout.pack_clover(g, A, torch.float64)), A)
    F = fields.random_full_clover(g, seed=5)
    assert torch.equal(layout.unpack_full_clover(g, layout.pack_full_clover(g, F, torch.float64)), F)


def test_slab_gauge_matches_global():
    G = Geometry(4, 4, 4, 8, soalen=1)
    g = G.with_(nt=4)
    U = fields.random_gauge(G, seed=6)
    full = layout.pack_gauge(G, U, 1, torch.float64).reshape(G.nt, -1)
    slab = layout.pack_gauge(g, U, 1, torch.float64, t0=4).reshape(g.nt, -1)
    assert torch.equal(full[4:], slab)
