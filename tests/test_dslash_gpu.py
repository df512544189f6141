"""GPU parity of the body kernels against the FP64 oracle, through the
C-ABI.  Tolerances (per site component, relative, floored at the site rms;
helpers.TOL): 1e-6 FP32, 1e-13 FP64, 1e-3 FP16 and FP16 + per-site norm,
4e-3 BF16 (its 8-bit significand alone costs up to 2^-8 = 3.9e-3)."""
import numpy as np
import pytest
import torch

import helpers as H
import oracle as O
from qphix_b200 import ops
from qphix_b200.lattice import BF16, F16, F16N, F32, F64, FTYPE_NAMES, Geometry

TOL = H.TOL

pytestmark = pytest.mark.gpu


def _run_gpu(g, f, fam, kernel, isign, cb, pp, dev):
    T = lambda a: H.to_torch(a, dev)
    psi, chi, gauge = T(f["psi"]), T(f["chi"]), T(f["gauge"])
    cl = T(f["fclover"] if fam == "tm_clover" else f["clover"])
    out = torch.zeros_like(psi)
    ops.dslash(g, fam, kernel, isign, cb, psi, out, gauge, chi=chi, clover=cl, **pp)
    torch.cuda.synchronize()
    return H.to_np(out)


def _run_oracle(g, f, fam, kernel, isign, cb, pp):
    """the oracle's FP64 result (unrounded) on the same stored inputs"""
    prm = O.make_params(**pp)
    cl = f["fclover"] if fam == "tm_clover" else f["clover"]
    return O.dslash(g, fam, kernel, isign, cb, f["psi"], f["gauge"], chi=f["chi"], clover=cl, params=prm,
                    fp64_out=True)


def _err(g, a, b, name):
    return H.record(name, H.site_rel_err(g, a, b, g.with_(ftype=F64)), TOL[g.ftype])


LAYOUTS = [
    (1, 1, F32), (2, 2, F32), (4, 4, F32), (4, 16, F32), (8, 8, F32), (16, 16, F32),
    (4, 8, F64), (8, 8, F64), (4, 16, F16), (8, 8, F16), (16, 16, F16),
    (4, 8, F16N), (16, 16, F16N), (8, 16, BF16), (16, 16, BF16),
    (4, 4, F64), (4, 4, F16), (8, 8, F16N), (4, 4, BF16),
]


@pytest.mark.parametrize("soa,vec,ft", LAYOUTS)
@pytest.mark.parametrize("comp", [False, True])
def test_all_variants_vs_oracle(cuda, soa, vec, ft, comp):
    nx = max(4, 2 * soa)
    g = Geometry(nx, 8, 4, 4, soalen=soa, veclen=vec, ftype=ft, compress12=comp, t_boundary=-1.0)
    name = "dslash %s soa%d vec%d c%d" % (FTYPE_NAMES[ft], soa, vec, comp)
    for cb in (0, 1):
        f = H.make_fields(g, cb=cb, seed=100 + cb)
        for fam in H.FAMILIES:
            for kernel in H.KERNELS:
                for isign in (1, -1):
                    for tbc in (0, 11):
                        pp = H.op_params(fam, kernel, tbc_mask=tbc)
                        a = _run_gpu(g, f, fam, kernel, isign, cb, pp, cuda)
                        b = _run_oracle(g, f, fam, kernel, isign, cb, pp)
                        e = _err(g, a, b, name)
                        assert e < TOL[ft], (fam, kernel, isign, cb, tbc, e)


@pytest.mark.parametrize("acc", [[0, 1, 1, 1, 1, 1, 1, 1], [1, 0, 0, 1, 1, 0, 0, 1], [0] * 8])
def test_accumulate_flags(cuda, acc):
    g = Geometry(8, 8, 4, 4, soalen=4, veclen=8, ftype=F32, compress12=True, t_boundary=-1.0)
    f = H.make_fields(g, cb=0)
    for fam in H.FAMILIES:
        for kernel in H.KERNELS:
            pp = H.op_params(fam, kernel, tbc_mask=3, accumulate=acc)
            a = _run_gpu(g, f, fam, kernel, -1, 0, pp, cuda)
            b = _run_oracle(g, f, fam, kernel, -1, 0, pp)
            assert _err(g, a, b, "dslash accumulate flags f32") < TOL[F32]


def test_padding_and_time_edges(cuda):
    g = Geometry(8, 4, 4, 6, soalen=2, veclen=4, ftype=F32, pad_xy=3, pad_xyz=5, t_boundary=-1.0,
                 t_edge_lo=True, t_edge_hi=False)
    f = H.make_fields(g, cb=1)
    for fam in H.FAMILIES:
        pp = H.op_params(fam, "dslash")
        a = _run_gpu(g, f, fam, "dslash", 1, 1, pp, cuda)
        b = _run_oracle(g, f, fam, "dslash", 1, 1, pp)
        assert _err(g, a, b, "dslash padding and time edges f32") < TOL[F32]


@pytest.mark.parametrize("dims,soa,ft", [((8, 6, 4, 4), 4, F32), ((24, 6, 4, 4), 4, F32), ((16, 6, 4, 4), 8, F64),
                                         ((24, 10, 4, 4), 4, F16N), ((48, 2, 4, 4), 8, BF16)])
def test_staged_layouts_ragged_planes(cuda, dims, soa, ft):
    """SOALEN 4/8 with VECLEN == SOALEN (the kernels that stage every field
    through shared memory: async for 32-bit, twin for 16-bit storage; FP64
    takes the thread-per-site kernel), including planes whose site count is
    not a multiple of 32 (idle lanes), padding, and the skipped t hops of a
    communicated boundary."""
    for pad, acc in (((0, 0), None), ((3, 5), [1, 1, 1, 1, 1, 1, 0, 0])):
        g = Geometry(*dims, soalen=soa, veclen=soa, ftype=ft, compress12=True, t_boundary=-1.0,
                     pad_xy=pad[0], pad_xyz=pad[1])
        f = H.make_fields(g, cb=1, seed=140)
        for fam in H.FAMILIES:
            for kernel in H.KERNELS:
                pp = H.op_params(fam, kernel, tbc_mask=13, accumulate=acc)
                a = _run_gpu(g, f, fam, kernel, 1, 1, pp, cuda)
                b = _run_oracle(g, f, fam, kernel, 1, 1, pp)
                e = _err(g, a, b, "dslash ragged planes %s soa%d" % (FTYPE_NAMES[ft], soa))
                assert e < TOL[ft], (fam, kernel, pad, e)

