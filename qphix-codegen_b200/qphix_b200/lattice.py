"""Lattice description and QPhiX tile-layout geometry.

`Lattice` is the ctypes image of `qb200_lattice` (include/qphix_b200.h).
`Geometry` adds the derived sizes of the QPhiX layouts of
codegen/include/decl_common.h:9-62 (Types<FT,V,S,compress12>):

  spinor  FourSpinorBlock FT[3][4][2][S]           one per S x-sites
  gauge   SU3MatrixBlock  FT[8][2|3][3][2][V]       one per tile of V sites
  clover  CloverBlock     diag1[6][V], off_diag1[15][2][V], diag2, off_diag2
  tmclov  FullCloverBlock block1[6][6][2][V], block2[6][6][2][V]

A tile covers V/S consecutive y rows of S x-sites of one checkerboard.
"""
import ctypes
from dataclasses import dataclass

import torch

F32, F64, F16, F16N, BF16 = 0, 1, 2, 3, 4
FTYPE_NAMES = {F32: "f32", F64: "f64", F16: "f16", F16N: "f16n", BF16: "bf16"}
# F16N: FP16 spinors with a per-site FP32 norm after each block; links and
# clover plain FP16.  BF16: bfloat16 everywhere.
TORCH_DTYPE = {F32: torch.float32, F64: torch.float64, F16: torch.float16, F16N: torch.float16,
               BF16: torch.bfloat16}
FT_BYTES = {F32: 4, F64: 8, F16: 2, F16N: 2, BF16: 2}


class Lattice(ctypes.Structure):
    """ctypes mirror of `qb200_lattice`."""

    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("nt", ctypes.c_int),
        ("soalen", ctypes.c_int), ("veclen", ctypes.c_int),
        ("pad_xy", ctypes.c_int), ("pad_xyz", ctypes.c_int),
        ("ftype", ctypes.c_int), ("compress12", ctypes.c_int),
        ("t_boundary", ctypes.c_double),
        ("t_edge_lo", ctypes.c_int), ("t_edge_hi", ctypes.c_int),
    ]


@dataclass(frozen=True)
class Geometry:
    """Local lattice plus layout parameters (mirrors qb200_lattice)."""

    nx: int
    ny: int
    nz: int
    nt: int
    soalen: int = 4
    veclen: int = 0          # 0 -> soalen
    ftype: int = F32
    compress12: bool = False
    pad_xy: int = 0
    pad_xyz: int = 0
    t_boundary: float = 1.0
    t_edge_lo: bool = True
    t_edge_hi: bool = True

    def __post_init__(self):
        if self.veclen == 0:
            object.__setattr__(self, "veclen", self.soalen)
        for n in (self.nx, self.ny, self.nz, self.nt):
            if n <= 0 or n % 2:
                raise ValueError("lattice extents must be positive and even: %r" % (self.dims,))
        if self.veclen % self.soalen:
            raise ValueError("veclen must be a multiple of soalen")
        if (self.nx // 2) % self.soalen:
            raise ValueError("nx/2 must be a multiple of soalen")
        if self.ny % self.ngy:
            raise ValueError("ny must be a multiple of veclen/soalen")

    # -- derived sizes
    @property
    def dims(self):
        return (self.nx, self.ny, self.nz, self.nt)

    @property
    def nxh(self):
        return self.nx // 2

    @property
    def ngy(self):
        return self.veclen // self.soalen

    @property
    def nyg(self):
        return self.ny // self.ngy

    @property
    def nvecs(self):
        return self.nxh // self.soalen

    @property
    def Pxy(self):
        return self.ny * self.nvecs + self.pad_xy

    @property
    def Pxyz(self):
        return self.nz * self.Pxy + self.pad_xyz

    @property
    def vol_cb(self):
        return self.nxh * self.ny * self.nz * self.nt

    @property
    def ntiles(self):
        return self.nt * self.nz * self.nyg * self.nvecs

    @property
    def rows(self):
        return 2 if self.compress12 else 3

    @property
    def spb(self):
        """storage elements per lane of a spinor block"""
        return 26 if self.ftype == F16N else 24

    @property
    def face_elems(self):
        """storage elements per face site"""
        return 14 if self.ftype == F16N else 12

    @property
    def spinor_elems(self):
        return self.nt * self.Pxyz * self.spb * self.soalen

    @property
    def gauge_elems(self):
        return self.ntiles * 8 * self.rows * 6 * self.veclen

    @property
    def clover_elems(self):
        return self.ntiles * 72 * self.veclen

    @property
    def full_clover_elems(self):
        return self.ntiles * 144 * self.veclen

    @property
    def dtype(self):
        return TORCH_DTYPE[self.ftype]

    def face_sites(self, dir):
        mu = dir // 2
        return [self.nt * self.nz * self.ny // 2, self.nt * self.nz * self.nxh,
                self.nt * self.ny * self.nxh, self.nz * self.ny * self.nxh][mu]

    def with_(self, **kw):
        d = dict(self.__dict__)
        d.update(kw)
        return Geometry(**d)

    def c_struct(self):
        return Lattice(self.nx, self.ny, self.nz, self.nt, self.soalen, self.veclen,
                       self.pad_xy, self.pad_xyz, self.ftype, 1 if self.compress12 else 0,
                       float(self.t_boundary), 1 if self.t_edge_lo else 0, 1 if self.t_edge_hi else 0)
