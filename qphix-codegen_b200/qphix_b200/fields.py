"""Seeded synthetic fields in canonical form (torch, any device).

  gauge    random SU(3) per link: complex Gaussian 3x3, rows Gram-Schmidt
           orthonormalised, third row conj(row0 x row1) (det = 1)
  spinor   complex Gaussian, N(0,1) real and imaginary parts
  clover   A = I + scale*H per 6x6 block, H Hermitian with |H|_2 <= 1, so A is
           Hermitian positive definite for scale < 1
  fclover  F = I + scale*M, M a complex Gaussian 6x6 with |M|_F = 1 (dense,
           non-Hermitian: the FullCloverBlock of twisted-mass clover)
"""
import torch

from .lattice import Geometry


def _gen(seed, device):
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    return gen


def _cgauss(shape, gen, device):
    re = torch.randn(*shape, generator=gen, device=device, dtype=torch.float64)
    im = torch.randn(*shape, generator=gen, device=device, dtype=torch.float64)
    return torch.complex(re, im)


def random_su3(shape, seed=1234, device="cpu"):
    gen = _gen(seed, device)
    m = _cgauss(tuple(shape) + (3, 3), gen, device)
    r0 = m[..., 0, :]
    r0 = r0 / torch.linalg.vector_norm(r0, dim=-1, keepdim=True)
    r1 = m[..., 1, :]
    r1 = r1 - (r0.conj() * r1).sum(-1, keepdim=True) * r0
    r1 = r1 / torch.linalg.vector_norm(r1, dim=-1, keepdim=True)
    r2 = torch.linalg.cross(r0, r1, dim=-1).conj()
    return torch.stack([r0, r1, r2], dim=-2)


def random_gauge(g: Geometry, seed=1234, device="cpu"):
    """Full-lattice links U[mu][t][z][y][x] (4, nt, nz, ny, nx, 3, 3)."""
    return random_su3((4, g.nt, g.nz, g.ny, g.nx), seed=seed, device=device)


def random_spinor(g: Geometry, seed=1235, device="cpu"):
    """Checkerboard spinor (nt, nz, ny, nxh, 4, 3)."""
    return _cgauss((g.nt, g.nz, g.ny, g.nxh, 4, 3), _gen(seed, device), device)


def random_clover(g: Geometry, seed=1236, scale=0.1, device="cpu"):
    """Hermitian positive-definite blocks (nt, nz, ny, nxh, 2, 6, 6)."""
    m = _cgauss((g.nt, g.nz, g.ny, g.nxh, 2, 6, 6), _gen(seed, device), device)
    h = 0.5 * (m + m.conj().transpose(-1, -2))
    h = h / torch.linalg.matrix_norm(h, dim=(-2, -1), keepdim=True)  # Frobenius >= spectral
    eye = torch.eye(6, dtype=h.dtype, device=device)
    return eye + scale * h


def random_full_clover(g: Geometry, seed=1237, scale=0.1, device="cpu"):
    """Dense complex blocks (nt, nz, ny, nxh, 2, 6, 6)."""
    m = _cgauss((g.nt, g.nz, g.ny, g.nxh, 2, 6, 6), _gen(seed, device), device)
    m = m / torch.linalg.matrix_norm(m, dim=(-2, -1), keepdim=True)
    eye = torch.eye(6, dtype=m.dtype, device=device)
    return eye + scale * m


def invert_blocks(A):
    """Block-wise inverse (FP64), e.g. A^-1 for the inverse-clover variant."""
    return torch.linalg.inv(A.to(torch.complex128))
