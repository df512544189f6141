"""GPU parity of the body kernels against the oracle (and the reference's
golden vectors), through the C-ABI.  Tolerances (per site component,
relative, floored at the site rms): 1e-6 FP32 (the reference computes in FP32
too, so 2e-6 is allowed for accumulated rounding), 1e-13 FP64, 1e-3 half."""
import numpy as np
import pytest
import torch

import helpers as H
import oracle as O
from qphix_b200 import ops
from qphix_b200.lattice import BF16, F16, F16N, F32, F64, Geometry

# FP16 with a per-site norm quantises every component to 2^-11 of the site's
# largest one, bfloat16 to 2^-8 of each value
TOL = {F32: 2e-6, F64: 1e-13, F16: 1e-3, F16N: 2e-3, BF16: 1e-2}

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
    prm = O.make_params(**pp)
    cl = f["fclover"] if fam == "tm_clover" else f["clover"]
    return O.dslash(g, fam, kernel, isign, cb, f["psi"], f["gauge"], chi=f["chi"], clover=cl, params=prm)


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
    worst = 0.0
    for cb in (0, 1):
        f = H.make_fields(g, cb=cb, seed=100 + cb)
        for fam in H.FAMILIES:
            for kernel in H.KERNELS:
                for isign in (1, -1):
                    for tbc in (0, 11):
                        pp = H.op_params(fam, kernel, tbc_mask=tbc)
                        a = _run_gpu(g, f, fam, kernel, isign, cb, pp, cuda)
                        b = _run_oracle(g, f, fam, kernel, isign, cb, pp)
                        e = H.site_rel_err(g, a, b)
                        worst = max(worst, e)
                        assert e < TOL[ft], (fam, kernel, isign, cb, tbc, e)
    print("worst", worst)


@pytest.mark.parametrize("acc", [[0, 1, 1, 1, 1, 1, 1, 1], [1, 0, 0, 1, 1, 0, 0, 1], [0] * 8])
def test_accumulate_flags(cuda, acc):
    g = Geometry(8, 8, 4, 4, soalen=4, veclen=8, ftype=F32, compress12=True, t_boundary=-1.0)
    f = H.make_fields(g, cb=0)
    for fam in H.FAMILIES:
        for kernel in H.KERNELS:
            pp = H.op_params(fam, kernel, tbc_mask=3, accumulate=acc)
            a = _run_gpu(g, f, fam, kernel, -1, 0, pp, cuda)
            b = _run_oracle(g, f, fam, kernel, -1, 0, pp)
            assert H.site_rel_err(g, a, b) < TOL[F32]


def test_padding_and_time_edges(cuda):
    g = Geometry(8, 4, 4, 6, soalen=2, veclen=4, ftype=F32, pad_xy=3, pad_xyz=5, t_boundary=-1.0,
                 t_edge_lo=True, t_edge_hi=False)
    f = H.make_fields(g, cb=1)
    for fam in H.FAMILIES:
        pp = H.op_params(fam, "dslash")
        a = _run_gpu(g, f, fam, "dslash", 1, 1, pp, cuda)
        b = _run_oracle(g, f, fam, "dslash", 1, 1, pp)
        assert H.site_rel_err(g, a, b) < TOL[F32]


@pytest.mark.parametrize("dims,soa,ft", [((8, 6, 4, 4), 4, F32), ((24, 6, 4, 4), 4, F32), ((16, 6, 4, 4), 8, F64),
                                         ((24, 10, 4, 4), 4, F16N), ((48, 2, 4, 4), 8, BF16)])
def test_staged_layouts_ragged_planes(cuda, dims, soa, ft):
    """SOALEN 4/8 with VECLEN == SOALEN (the shared-memory staged kernel),
    including planes whose site count is not a multiple of 32 (idle lanes),
    padding, and the skipped t hops of a communicated boundary."""
    for pad, acc in (((0, 0), None), ((3, 5), [1, 1, 1, 1, 1, 1, 0, 0])):
        g = Geometry(*dims, soalen=soa, veclen=soa, ftype=ft, compress12=True, t_boundary=-1.0,
                     pad_xy=pad[0], pad_xyz=pad[1])
        f = H.make_fields(g, cb=1, seed=140)
        for fam in H.FAMILIES:
            for kernel in H.KERNELS:
                pp = H.op_params(fam, kernel, tbc_mask=13, accumulate=acc)
                a = _run_gpu(g, f, fam, kernel, 1, 1, pp, cuda)
                b = _run_oracle(g, f, fam, kernel, 1, 1, pp)
                assert H.site_rel_err(g, a, b) < TOL[ft], (fam, kernel, pad)
