"""qphix_b200: host side of the B200 dslash library.

The CUDA kernels live in libqphix_b200.so (C-ABI: include/qphix_b200.h);
this package holds the lattice description, the QPhiX layout converters,
seeded synthetic fields and thin torch wrappers of the C entry points.
"""
from .lattice import F16, F32, F64, Geometry, Lattice  # noqa: F401
from . import fields, layout  # noqa: F401

