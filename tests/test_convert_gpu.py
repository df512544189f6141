"""Device converters against the torch statement of the layouts
(qphix_b200.layout), bit for bit, for every storage type."""
import pytest
import torch

from qphix_b200 import convert, fields, layout
from qphix_b200.lattice import BF16, F16, F16N, F32, F64, Geometry

pytestmark = pytest.mark.gpu

CASES = [(4, 4, F32, True), (8, 16, F32, False), (2, 2, F64, False), (4, 8, F16, True), (4, 4, F16N, True),
         (8, 8, BF16, False), (16, 16, F32, True)]


@pytest.mark.parametrize("soa,vec,ft,comp", CASES)
def test_converters_match_torch(cuda, soa, vec, ft, comp):
    g = Geometry(max(8, 2 * soa), 4, 6, 4, soalen=soa, veclen=vec, ftype=ft, compress12=comp, pad_xy=1, pad_xyz=2)
    sp = fields.random_spinor(g, seed=41).to(cuda)
    U = fields.random_gauge(g, seed=42).to(cuda)
    A = fields.random_clover(g, seed=43).to(cuda)
    F = fields.random_full_clover(g, seed=44).to(cuda)
    for cdt in (torch.complex128, torch.complex64):
        want = layout.pack_spinor(g, sp.to(cdt))
        got = convert.pack_spinor(g, sp.to(cdt))
        assert torch.equal(got.view(torch.int16) if got.element_size() == 2 else got,
                           want.view(torch.int16) if want.element_size() == 2 else want), cdt
    back = convert.unpack_spinor(g, got)
    assert torch.equal(back, layout.unpack_spinor(g, got))
    for cb in (0, 1):
        assert torch.equal(convert.pack_gauge(g, U, cb), layout.pack_gauge(g, U, cb))
    assert torch.equal(convert.pack_clover(g, A), layout.pack_clover(g, A))
    assert torch.equal(convert.pack_full_clover(g, F), layout.pack_full_clover(g, F))


def test_gauge_slab(cuda):
    """links of a t slab of a longer lattice (multi-GPU packing)"""
    g = Geometry(8, 4, 4, 4, soalen=4, ftype=F32, compress12=True, t_edge_lo=False, t_edge_hi=False)
    G = g.with_(nt=12)
    U = fields.random_gauge(G, seed=45).to(cuda)
    for t0 in (0, 4, 8):
        for cb in (0, 1):
            assert torch.equal(convert.pack_gauge(g, U, cb, t0=t0), layout.pack_gauge(g, U, cb, t0=t0))
