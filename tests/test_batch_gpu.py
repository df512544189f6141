"""Batched launch over lattices of different sizes: every lattice's result
equals the single-lattice entry point's, bit for bit, for any launch shape,
after tuning, and when replayed from a CUDA graph."""
import os

import pytest
import torch

import helpers as H
from qphix_b200 import _lib, batch, ops
from qphix_b200.lattice import F16, F32, F64, Geometry

pytestmark = pytest.mark.gpu

DIMS = [(16, 4, 4, 4), (16, 8, 4, 4), (32, 4, 8, 4)]


def _problems(ft, S, family, kernel, comp12, cuda, seed=300):
    probs, refs = [], []
    for k, d in enumerate(DIMS):
        g = Geometry(*d, soalen=S, veclen=S, ftype=ft, compress12=comp12, t_boundary=-1.0)
        f = H.make_fields(g, cb=k % 2, seed=seed + k)
        T = lambda a: H.to_torch(a, cuda)
        cl = T(f["fclover" if family == "tm_clover" else "clover"])
        pp = H.op_params(family, kernel, seed=k, tbc_mask=0b0110 if k == 1 else 0)
        pp.pop("accumulate")
        psi, chi, gauge = T(f["psi"]), T(f["chi"]), T(f["gauge"])
        out = torch.zeros_like(psi)
        probs.append(batch.Problem(g, k % 2, psi, out, gauge, chi=chi if kernel == "achimbdpsi" else None,
                                   clover=cl if family in ("clover", "tm_clover") else None, **pp))
        ref = torch.zeros_like(psi)
        ops.dslash(g, family, kernel, 1, k % 2, psi, ref, gauge, chi=chi, clover=cl, **pp)
        refs.append(ref)
    return probs, refs


@pytest.mark.parametrize("ft,S", [(F32, 4), (F64, 2), (F16, 8)])
@pytest.mark.parametrize("family", H.FAMILIES)
def test_batched_matches_single(cuda, ft, S, family):
    for kernel in H.KERNELS:
        probs, refs = _problems(ft, S, family, kernel, ft != F64, cuda)
        op = batch.BatchedDslash(family, kernel, 1, probs)
        for grid, block in ((0, 128), (3, 64), (1, 128)):
            for p in probs:
                p.out.zero_()
            op(grid=grid, block=block)
            torch.cuda.synchronize()
            for p, r in zip(probs, refs):
                assert torch.equal(p.out, r), (family, kernel, grid, block)


def test_tune_and_graph(cuda, tmp_path):
    probs, refs = _problems(F32, 4, "clover", "achimbdpsi", True, cuda, seed=310)
    op = batch.BatchedDslash("clover", "achimbdpsi", 1, probs)
    grid, block, ms = op.tune()
    assert block in (64, 128) and grid > 0 and ms > 0
    for p, r in zip(probs, refs):
        assert torch.equal(p.out, r)
    # the table round-trips through a file
    path = str(tmp_path / "tune.txt")
    L = _lib.lib()
    _lib.check(L.qb200_tune_cache_save(path.encode()))
    L.qb200_tune_cache_clear()
    assert L.qb200_tune_cache_load(path.encode()) >= 1
    # graph replay
    for p in probs:
        p.out.zero_()
    g = op.capture(steps=3)
    for p in probs:
        p.out.zero_()
    g.replay()
    torch.cuda.synchronize()
    for p, r in zip(probs, refs):
        assert torch.equal(p.out, r)


def test_batch_rejects_mixed_layouts(cuda):
    probs, _ = _problems(F32, 4, "wilson", "dslash", False, cuda)
    g2 = probs[1].g.with_(soalen=2, veclen=2)
    probs[1].g = g2
    with pytest.raises(_lib.QB200Error):
        batch.BatchedDslash("wilson", "dslash", 1, probs)()


@pytest.mark.parametrize("ft,S,dims", [
    (F32, 4, [(24, 6, 4, 4), (8, 6, 4, 4), (16, 8, 4, 4)]),
    (F16, 8, [(48, 6, 4, 4), (16, 6, 4, 4), (48, 2, 4, 4)])])
def test_batched_ragged_planes(cuda, ft, S, dims):
    """planes whose site count is not a multiple of 32 (the batched kernels
    pad each plane to whole warps) and, at 16 bits, rows of three blocks that
    do not line up with a warp's blocks (the x region)"""
    global DIMS
    saved = DIMS
    try:
        DIMS = dims
        for family in ("clover", "tm", "tm_clover"):
            for kernel in H.KERNELS:
                probs, refs = _problems(ft, S, family, kernel, True, cuda, seed=320)
                op = batch.BatchedDslash(family, kernel, 1, probs)
                for grid, block in ((0, 128), (2, 128), (5, 64)):
                    for p in probs:
                        p.out.zero_()
                    op(grid=grid, block=block)
                    torch.cuda.synchronize()
                    for p, r in zip(probs, refs):
                        assert torch.equal(p.out, r), (family, kernel, grid, block)
    finally:
        DIMS = saved
