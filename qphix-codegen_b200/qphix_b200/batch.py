"""One operator over several lattices in one launch (qb200_dslash_batched),
launch tuning (qb200_tune_batched) and CUDA-graph replay.

    probs = [batch.Problem(g, cb, psi, out, gauge, chi=chi, clover=A, coeff_s=0.125, ...), ...]
    op = batch.BatchedDslash("clover", "achimbdpsi", +1, probs)
    op.tune()                 # times launch shapes once, remembers the best
    op()                      # one launch over every lattice
    graph = op.capture(10)    # ten applications as one CUDA graph
    graph.replay()

Problems share storage type, SOALEN, VECLEN (== SOALEN for SOALEN >= 4) and
link compression; their sizes, fields, checkerboards and coefficients may
differ.  Every hop wraps around its own lattice (no halo).
"""
import ctypes

import torch

from . import _lib, ops
from .lattice import Geometry
from .solver import FAMILY


class Problem:
    """One lattice of a batch: geometry, output checkerboard, fields (device
    tensors in the layouts of g) and scalar coefficients (coeff_s, coeff_t_f,
    coeff_t_b, alpha, mu, muinv, rho, tbc_mask, tbc_phases)."""

    def __init__(self, g: Geometry, cb, psi, out, gauge, chi=None, clover=None, **coeffs):
        self.g, self.cb, self.psi, self.out, self.gauge = g, cb, psi, out, gauge
        self.chi, self.clover, self.coeffs = chi, clover, coeffs


def _coeffs(kw):
    c = _lib.Coeffs()
    c.coeff_s = kw.get("coeff_s", 1.0)
    c.coeff_t_f = kw.get("coeff_t_f", 1.0)
    c.coeff_t_b = kw.get("coeff_t_b", 1.0)
    c.alpha = kw.get("alpha", 1.0)
    c.mu = kw.get("mu", 0.0)
    c.muinv = kw.get("muinv", 1.0)
    c.rho = kw.get("rho", 0.0)
    c.tbc_mask = int(kw.get("tbc_mask", 0))
    ph = kw.get("tbc_phases") or [[1.0, 0.0]] * 4
    for m in range(4):
        c.tbc_phases[m][0], c.tbc_phases[m][1] = float(ph[m][0]), float(ph[m][1])
    return c


class BatchedDslash:
    def __init__(self, family, kernel, isign, problems):
        if family not in FAMILY:
            raise ValueError("unknown family %r" % family)
        if kernel not in ("dslash", "achimbdpsi"):
            raise ValueError("unknown kernel %r" % kernel)
        if not 1 <= len(problems) <= _lib.MAX_BATCH:
            raise ValueError("a batch holds 1..%d problems" % _lib.MAX_BATCH)
        self.family, self.kernel, self.isign = family, kernel, isign
        self.problems = list(problems)
        items = (_lib.BatchItem * len(problems))()
        for it, p in zip(items, problems):
            g = p.g
            ops._check_field("psi", p.psi, g, g.spinor_elems)
            ops._check_field("out", p.out, g, g.spinor_elems)
            ops._check_field("gauge", p.gauge, g, g.gauge_elems)
            if kernel == "achimbdpsi":
                ops._check_field("chi", p.chi, g, g.spinor_elems)
            if family in ("clover", "tm_clover"):
                ops._check_field("clover", p.clover, g,
                                 g.clover_elems if family == "clover" else g.full_clover_elems)
            it.lat = g.c_struct()
            it.cb = p.cb
            it.psi, it.out, it.gauge = p.psi.data_ptr(), p.out.data_ptr(), p.gauge.data_ptr()
            it.chi = p.chi.data_ptr() if p.chi is not None else None
            it.clov = p.clover.data_ptr() if p.clover is not None else None
            it.coeffs = _coeffs(p.coeffs)
        self.items = items
        self.cfg = None
        self.sites = sum(p.g.vol_cb for p in problems)

    def _args(self):
        return (FAMILY[self.family], 1 if self.kernel == "achimbdpsi" else 0, 1 if self.isign > 0 else -1,
                len(self.items), self.items)

    def tune(self, stream=None):
        """Time the launch shapes (writes the result to every out); returns
        (grid, block, ms per launch) and uses the winner from then on."""
        cfg = _lib.LaunchCfg()
        ms = ctypes.c_double(0.0)
        _lib.check(_lib.lib().qb200_tune_batched(*self._args(), ctypes.byref(cfg), ctypes.byref(ms),
                                                 ops._stream(stream)))
        self.cfg = cfg
        return cfg.grid, cfg.block, ms.value

    def __call__(self, grid=None, block=None, stream=None):
        """One launch over every problem; grid/block override the tuned shape
        (grid 0: one thread per site)."""
        cfg = self.cfg
        if grid is not None or block is not None:
            cfg = _lib.LaunchCfg(grid if grid is not None else 0, block if block is not None else 128)
        _lib.check(_lib.lib().qb200_dslash_batched(*self._args(), ctypes.byref(cfg) if cfg is not None else None,
                                                   ops._stream(stream)))

    def capture(self, steps=1):
        """A CUDA graph of `steps` launches (tune first: tuning synchronises
        and cannot run inside a capture)."""
        graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self()                       # warm-up launch outside the capture
        torch.cuda.current_stream().wait_stream(side)
        with torch.cuda.graph(graph):
            for _ in range(steps):
                self()
        return graph
