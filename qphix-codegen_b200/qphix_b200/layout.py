"""Converters between canonical fields and the QPhiX tile layouts.

Canonical forms (complex torch tensors, any device):
  full-lattice links   U[mu][t][z][y][x][a][b]        (4, nt, nz, ny, nx, 3, 3)
  checkerboard spinor  sp[t][z][y][xcb][spin][colour] (nt, nz, ny, nxh, 4, 3)
  clover blocks        A[t][z][y][xcb][block][r][c]   (nt, nz, ny, nxh, 2, 6, 6)
Site (xcb, y, z, t) of checkerboard cb sits at x = 2*xcb + ((y+z+t+cb) & 1).

The packed gauge of checkerboard cb stores, per output site, the eight links
its hops use (codegen/dslash_common.cc:1678-1727): direction 2*mu+1 (forward)
U_mu(x), direction 2*mu (backward) U_mu(x - mu), each as G = U^T; a 12-real
gauge keeps rows 0 and 1 of G (codegen/dslash_common.cc:1657-1676).  The
clover block b covers spins 2b, 2b+1 with combined index 3*(spin-2b)+colour;
off_diag[r(r-1)/2+c] holds element (r, c), r > c
(codegen/dslash_common.cc:1098-1186, codegen/include/decl_common.h:15-32).
"""
import torch

from .lattice import F16N, Geometry


def cb_coords(g: Geometry, cb: int, device=None):
    """Coordinates (x, y, z, t) of the checkerboard sites, shape (nt,nz,ny,nxh)."""
    t = torch.arange(g.nt, device=device).view(-1, 1, 1, 1)
    z = torch.arange(g.nz, device=device).view(1, -1, 1, 1)
    y = torch.arange(g.ny, device=device).view(1, 1, -1, 1)
    xcb = torch.arange(g.nxh, device=device).view(1, 1, 1, -1)
    par = (y + z + t + cb) & 1
    x = 2 * xcb + par
    shape = (g.nt, g.nz, g.ny, g.nxh)
    return (x.expand(shape), y.expand(shape), z.expand(shape), t.expand(shape))


def _blocks_to_flat(g: Geometry, blocks: torch.Tensor) -> torch.Tensor:
    """blocks (nt, nz, ny, nvecs, B) -> flat spinor field with padding
    (B = spb*S storage elements per block)."""
    B = blocks.shape[-1]
    nt = g.nt
    out = torch.zeros(nt, g.Pxyz * B, dtype=blocks.dtype, device=blocks.device)
    body = out[:, : g.nz * g.Pxy * B].view(nt, g.nz, g.Pxy * B)
    body[:, :, : g.ny * g.nvecs * B] = blocks.reshape(nt, g.nz, g.ny * g.nvecs * B)
    return out.reshape(-1)


def _flat_to_blocks(g: Geometry, flat: torch.Tensor, B: int) -> torch.Tensor:
    v = flat.reshape(g.nt, g.Pxyz * B)[:, : g.nz * g.Pxy * B]
    v = v.reshape(g.nt, g.nz, g.Pxy * B)[:, :, : g.ny * g.nvecs * B]
    return v.reshape(g.nt, g.nz, g.ny, g.nvecs, B)


def _encode_f16n(g: Geometry, blocks: torch.Tensor) -> torch.Tensor:
    """(..., 24*S) values -> (..., 26*S) halves: values / site norm, then the
    FP32 norms of the S lanes as pairs of halves."""
    S = g.soalen
    v = blocks.reshape(*blocks.shape[:-1], 24, S)
    nrm = v.abs().amax(dim=-2)                                   # (..., S)
    nrm = torch.where(nrm > 0, nrm, torch.ones_like(nrm)).to(torch.float32)
    h = (v / nrm.to(v.dtype).unsqueeze(-2)).to(torch.float16).reshape(*blocks.shape[:-1], 24 * S)
    n16 = nrm.contiguous().view(torch.float16)                   # (..., 2*S)
    return torch.cat([h, n16], dim=-1)


def _decode_f16n(g: Geometry, blocks: torch.Tensor) -> torch.Tensor:
    S = g.soalen
    h = blocks[..., : 24 * S].to(torch.float64).reshape(*blocks.shape[:-1], 24, S)
    nrm = blocks[..., 24 * S:].contiguous().view(torch.float32).to(torch.float64)
    return (h * nrm.unsqueeze(-2)).reshape(*blocks.shape[:-1], 24 * S)


def pack_spinor(g: Geometry, sp: torch.Tensor, dtype=None) -> torch.Tensor:
    """Canonical checkerboard spinor -> FourSpinorBlock array (flat)."""
    dtype = dtype or g.dtype
    S = g.soalen
    r = torch.view_as_real(sp.to(torch.complex128).resolve_conj())        # nt nz ny nxh 4 3 2
    r = r.reshape(g.nt, g.nz, g.ny, g.nvecs, S, 4, 3, 2)
    r = r.permute(0, 1, 2, 3, 6, 5, 7, 4)                    # .. nvecs c s ri S
    r = r.reshape(g.nt, g.nz, g.ny, g.nvecs, 24 * S)
    if g.ftype == F16N and dtype == torch.float16:
        return _blocks_to_flat(g, _encode_f16n(g, r))
    return _blocks_to_flat(g, r.to(dtype))


def unpack_spinor(g: Geometry, flat: torch.Tensor) -> torch.Tensor:
    """FourSpinorBlock array -> canonical complex128 checkerboard spinor."""
    S = g.soalen
    if g.ftype == F16N and flat.dtype == torch.float16:
        b = _decode_f16n(g, _flat_to_blocks(g, flat, 26 * S))
    else:
        b = _flat_to_blocks(g, flat.to(torch.float64), 24 * S)
    b = b.reshape(g.nt, g.nz, g.ny, g.nvecs, 3, 4, 2, S).permute(0, 1, 2, 3, 7, 5, 4, 6)
    b = b.reshape(g.nt, g.nz, g.ny, g.nxh, 4, 3, 2).contiguous()
    return torch.view_as_complex(b)


def site_links(g: Geometry, U: torch.Tensor, cb: int, t0: int = 0, z0: int = 0) -> torch.Tensor:
    """The eight links each site of cb uses, as U (not transposed):
    (nt, nz, ny, nxh, 8, 3, 3).  U may cover longer z and t extents than g
    (a global lattice of which g is the block starting at slices z0, t0;
    both even, so that local and global checkerboards agree)."""
    x, y, z, t = cb_coords(g, cb, U.device)
    NZ, NT = U.shape[2], U.shape[1]
    t = (t + t0) % NT
    z = (z + z0) % NZ
    L = [g.nx, g.ny, NZ, NT]
    links = []
    for mu in range(4):
        c = [x, y, z, t]
        cm = list(c)
        cm[mu] = (c[mu] - 1) % L[mu]
        back = U[mu][cm[3], cm[2], cm[1], cm[0]]
        fwd = U[mu][t, z, y, x]
        links += [back, fwd]
    return torch.stack(links, dim=4)


def _to_tiles(g: Geometry, per_site: torch.Tensor) -> torch.Tensor:
    """per-site reals (nt, nz, ny, nxh, K) -> tile layout (ntiles, K, V) flat."""
    K = per_site.shape[-1]
    v = per_site.reshape(g.nt, g.nz, g.nyg, g.ngy, g.nvecs, g.soalen, K)
    v = v.permute(0, 1, 2, 4, 6, 3, 5)                     # nt nz nyg nvecs K ngy S
    return v.reshape(-1)


def _from_tiles(g: Geometry, flat: torch.Tensor, K: int) -> torch.Tensor:
    v = flat.reshape(g.nt, g.nz, g.nyg, g.nvecs, K, g.ngy, g.soalen)
    v = v.permute(0, 1, 2, 5, 3, 6, 4)                     # nt nz nyg ngy nvecs S K
    return v.reshape(g.nt, g.nz, g.ny, g.nxh, K)


def pack_gauge(g: Geometry, U: torch.Tensor, cb: int, dtype=None, t0: int = 0, z0: int = 0) -> torch.Tensor:
    """Full-lattice links -> SU3MatrixBlock array of checkerboard cb (of the
    block of g that starts at global slices z0 and t0)."""
    dtype = dtype or g.dtype
    G = site_links(g, U.to(torch.complex128), cb, t0, z0).transpose(-1, -2)   # G = U^T
    G = G[..., : g.rows, :]
    r = torch.view_as_real(G.resolve_conj()).reshape(g.nt, g.nz, g.ny, g.nxh, 8 * g.rows * 6)
    return _to_tiles(g, r).to(dtype).contiguous()


def unpack_gauge(g: Geometry, flat: torch.Tensor) -> torch.Tensor:
    """SU3MatrixBlock array -> stored rows of G per site (..., 8, rows, 3) complex."""
    r = _from_tiles(g, flat.to(torch.float64), 8 * g.rows * 6)
    r = r.reshape(g.nt, g.nz, g.ny, g.nxh, 8, g.rows, 3, 2).contiguous()
    return torch.view_as_complex(r)


def _tril_index():
    rows, cols = [], []
    for r in range(6):
        for c in range(r):
            rows.append(r)
            cols.append(c)
    # od index r(r-1)/2 + c enumerates exactly this order
    return rows, cols


def pack_clover(g: Geometry, A: torch.Tensor, dtype=None) -> torch.Tensor:
    """Hermitian blocks (nt,nz,ny,nxh,2,6,6) -> CloverBlock array."""
    dtype = dtype or g.dtype
    A = A.to(torch.complex128)
    rows, cols = _tril_index()
    diag = torch.diagonal(A, dim1=-2, dim2=-1).real              # ... 2 6
    off = A[..., rows, cols]                                      # ... 2 15
    off = torch.view_as_real(off.resolve_conj()).reshape(*off.shape[:-1], 30)    # ... 2 30
    per = torch.cat([diag, off], dim=-1).reshape(g.nt, g.nz, g.ny, g.nxh, 72)
    return _to_tiles(g, per).to(dtype).contiguous()


def unpack_clover(g: Geometry, flat: torch.Tensor) -> torch.Tensor:
    per = _from_tiles(g, flat.to(torch.float64), 72).reshape(g.nt, g.nz, g.ny, g.nxh, 2, 36)
    A = torch.zeros(g.nt, g.nz, g.ny, g.nxh, 2, 6, 6, dtype=torch.complex128, device=flat.device)
    idx = torch.arange(6, device=flat.device)
    A[..., idx, idx] = per[..., :6].to(torch.complex128)
    rows, cols = _tril_index()
    off = torch.view_as_complex(per[..., 6:].reshape(*per.shape[:-1], 15, 2).contiguous())
    A[..., rows, cols] = off
    A[..., cols, rows] = off.conj()
    return A


def pack_full_clover(g: Geometry, F: torch.Tensor, dtype=None) -> torch.Tensor:
    """Dense complex blocks (nt,nz,ny,nxh,2,6,6) -> FullCloverBlock array."""
    dtype = dtype or g.dtype
    r = torch.view_as_real(F.to(torch.complex128).resolve_conj()).reshape(g.nt, g.nz, g.ny, g.nxh, 144)
    return _to_tiles(g, r).to(dtype).contiguous()


def unpack_full_clover(g: Geometry, flat: torch.Tensor) -> torch.Tensor:
    r = _from_tiles(g, flat.to(torch.float64), 144).reshape(g.nt, g.nz, g.ny, g.nxh, 2, 6, 6, 2)
    return torch.view_as_complex(r.contiguous())
