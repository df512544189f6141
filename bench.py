#!/usr/bin/env python3
"""Benchmark of the headline configuration: Wilson-clover A.chi - b.D.psi
(clov_dslash_achimbdpsi_plus) on a 32^3 x 64 lattice per GPU, FP32 storage
and arithmetic, 12-real links, b = kappa = 0.125 (coeff_s = coeff_t = 0.125),
rho = 0, clover blocks I + 0.1 H (H random Hermitian), random SU(3) links and
Gaussian spinors (seeded, synthetic: the reference publishes no dataset).

One step = one application of the operator to one checkerboard
(V/2 = 1,048,576 sites on 32^3 x 64): 1824 flop/site (1320 Wilson + 504
clover) and 960 algorithmic bytes/site (psi 96 + chi 96 + out 96 + 8 links
x 48 + clover 288).  The fields (~1 GB) are larger than the 126 MB L2, so
no flush is needed between steps.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

N > 1 (torchrun, one rank per GPU): weak scaling over t slabs, each rank
holds a 32^3 x 64 slab of a 32^3 x 64N lattice; faces are exchanged with
NCCL send/recv while the interior runs (qphix_b200.halo).
--impl reference: the reference's own generated kernels (built from its
sources into oracle/_ref) on all host cores, rank 0 only.
"""
import argparse
import json
import os
import statistics
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [REPO, os.path.join(REPO, "qphix-codegen_b200")]

import numpy as np  # noqa: E402
import torch  # noqa: E402

FLOP_SITE = 1824
METRIC = "Dslash GFLOP/s (clover A.chi - b.D.psi, 32^3x64 per GPU, FP32, 12-real links)"
WORKLOAD = "clov_dslash_achimbdpsi_plus 32^3x64 FP32 compress12"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--soalen", type=int, default=16)
    ap.add_argument("--veclen", type=int, default=0)
    ap.add_argument("--dims", default="32,32,32,64")
    ap.add_argument("--e2e-steps", type=int, default=40,
                    help="steps of the end-to-end pipeline; its drain (one kernel and one device-to-host "
                         "copy) is amortised over them")
    ap.add_argument("--nrhs", type=int, default=8,
                    help="right-hand sides of --only solve_tm_mrhs / solve_tm_clover_mrhs")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="bound of the CPU baseline sample")
    ap.add_argument("--no-extras", action="store_true", help="skip the multi-RHS and solver measurements")
    ap.add_argument("--only", choices=["mrhs", "force", "batch", "solve", "tm", "solve_tm", "solve_tm_clover",
                                       "solve_tm_mrhs", "solve_tm_clover_mrhs"],
                    help="run one secondary measurement alone (on --dims) and print its JSON line")
    return ap.parse_args()


def bytes_per_site(ft_bytes=4, rows=2):
    return ft_bytes * (24 * 3 + 8 * rows * 6 + 72)


# ---------------------------------------------------------------------------
# clocks during the timed region (NVML, sampled every 2 ms)

class ClockSampler:
    REASONS = {
        "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
        "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80,
    }

    def __init__(self, index):
        self.samples = []
        self.reasons = 0
        self.max_mhz = None
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                self.reasons |= self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            except Exception:
                pass
            time.sleep(0.002)

    def __enter__(self):
        if self.nv is not None:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.nv is not None:
            self._stop.set()
            self.t.join()

    def summary(self, other=None):
        """median SM clock, max clock, sample count and active throttle
        reasons; other: a second sampler whose samples are merged in"""
        if self.nv is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"]}
        smp = list(self.samples) + (list(other.samples) if other is not None else [])
        rs = self.reasons | (other.reasons if other is not None else 0)
        return {"sm_mhz": statistics.median(smp) if smp else None,
                "sm_max_mhz": self.max_mhz, "samples": len(smp),
                "reasons": [k for k, v in self.REASONS.items() if rs & v]}


def measured_peak():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_from_profile(workload_key):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/*.json), or None."""
    p = os.path.join(REPO, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f).get(workload_key)
    except Exception:
        return None


# ---------------------------------------------------------------------------
# fields

def make_fields(g, device, cb=0, seed=1234):
    from qphix_b200 import fields, layout
    U = fields.random_gauge(g, seed=seed, device=device)
    gauge = layout.pack_gauge(g, U, cb)
    del U
    psi = layout.pack_spinor(g, fields.random_spinor(g, seed=seed + 1, device=device))
    chi = layout.pack_spinor(g, fields.random_spinor(g, seed=seed + 2, device=device))
    clov = layout.pack_clover(g, fields.random_clover(g, seed=seed + 3, device=device))
    return {"psi": psi, "chi": chi, "gauge": gauge, "clover": clov}


PARAMS = dict(coeff_s=0.125, coeff_t_f=0.125, coeff_t_b=0.125, rho=0.0)


# ---------------------------------------------------------------------------
# CPU: the reference's generated kernels

def pick_reference_lib():
    import oracle as O
    flags = open("/proc/cpuinfo").read()
    for name, flag in (("avx512_f32_s16", "avx512f"), ("avx2_f32_s8", "avx2"), ("scalar_f32", "")):
        if O.ref_available(name) and (not flag or flag in flags):
            return name
    return None


def run_reference_cpu(dims, steps, warmup, seconds, fields_gpu=None, g_gpu=None, name=None, kernel="achimbdpsi",
                      flop_site=None):
    """Time the reference kernels (library `name`, default the best the host
    runs) on the host for the clover `kernel` ("achimbdpsi", or "dslash":
    the plain clov_dslash with the clover field as given, A^-1 for the
    inverse-clover variant); returns a dict."""
    import oracle as O
    from qphix_b200 import layout
    from qphix_b200.lattice import Geometry
    name = name or pick_reference_lib()
    if name is None or not O.ref_available(name):
        return {"unavailable": "reference kernels not built (python oracle/ref_build.py)"}
    flop_site = flop_site or FLOP_SITE
    info = O.ref_info(name)
    g = Geometry(*dims, soalen=info["soalen"], veclen=info["veclen"], compress12=True, t_boundary=-1.0)
    if fields_gpu is not None:
        # same canonical fields, repacked into the reference's layout
        f = {}
        for k, v in fields_gpu.items():
            if k in ("psi", "chi"):
                f[k] = layout.pack_spinor(g, layout.unpack_spinor(g_gpu, v)).cpu().numpy()
            elif k == "gauge":
                gg = layout.unpack_gauge(g_gpu, v)
                r = torch.view_as_real(gg).reshape(g.nt, g.nz, g.ny, g.nxh, -1).to(torch.float32)
                f[k] = layout._to_tiles(g, r).cpu().numpy()
            else:
                f[k] = layout.pack_clover(g, layout.unpack_clover(g_gpu, v)).cpu().numpy()
    else:
        f = {k: v.numpy() for k, v in make_fields(g, "cpu").items()}
    A = {k: O.aligned(v) for k, v in f.items()}
    out = O.aligned(np.zeros(g.spinor_elems, dtype=np.float32))
    prm = O.make_params(**PARAMS)
    nthreads = os.cpu_count() or 1
    call = lambda: O.ref_dslash(name, g, "clover", kernel, 1, 0, A["psi"], A["gauge"], chi=A["chi"],
                                clover=A["clover"], params=prm, out=out, nthreads=nthreads)
    for _ in range(max(1, warmup)):
        call()
    times = []
    t_start = time.perf_counter()
    for _ in range(max(1, steps)):
        t0 = time.perf_counter()
        call()
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > seconds:
            break
    per = sum(times) / len(times)
    gflops = flop_site * g.vol_cb / per / 1e9
    wl = WORKLOAD if kernel == "achimbdpsi" else "clov_dslash_plus (A^-1) 32^3x64 FP32 compress12"
    return {"value": gflops, "unit": "GFLOP/s", "cores": nthreads, "kind": "reference",
            "sample": "%d full-lattice calls of %s on %s (%s)" % (len(times), wl, "x".join(map(str, dims)), name),
            "ms_per_step": per * 1e3, "lib": name, "out": out}


# ---------------------------------------------------------------------------

def _time(fn, reps, stream):
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def bench_mrhs(g, f, dev):
    """Multi-RHS clover A.chi - b.D.psi: nrhs right-hand sides share one link
    and clover field; per right-hand-side site 3 spinors + (links + clover) /
    nrhs bytes: FP32 288 + 672/nrhs, FP16 144 + 336/nrhs."""
    from qphix_b200 import mrhs
    from qphix_b200.lattice import F16
    res = {}
    stream = torch.cuda.current_stream()
    g16 = g.with_(ftype=F16)
    fields16 = {"gauge": f["gauge"].half(), "clover": f["clover"].half()}
    for tag, gg, ff, sp_b, lc_b in (("f32", g, f, 96, 672), ("f16", g16, fields16, 48, 336)):
        for n in (4, 8, 16):
            psi = torch.randn(gg.spinor_elems * n, device=dev).to(gg.dtype)
            chi = torch.randn(gg.spinor_elems * n, device=dev).to(gg.dtype)
            out = torch.zeros_like(psi)
            ms = _time(lambda: mrhs.dslash(gg, n, "clover", "achimbdpsi", 1, 0, psi, out, ff["gauge"], chi=chi,
                                           clover=ff["clover"], **PARAMS), 20, stream)
            bps = 3 * sp_b + lc_b / n
            res["%s_nrhs_%d" % (tag, n)] = {"ms_per_call": ms,
                                            "gflops": FLOP_SITE * g.vol_cb * n / (ms * 1e-3) / 1e9,
                                            "gbs": bps * g.vol_cb * n / (ms * 1e-3) / 1e9, "bytes_per_rhs_site": bps}
            del psi, chi, out
    res["note"] = ("two right-hand sides per thread in packed FP32x2 arithmetic; GB/s against the algorithmic "
                   "bytes per right-hand-side site")
    return res


def fp64_cg(op, b, tol=1e-10):
    """FP64 CG to |b - Mhat x| / |b| <= tol.  CG on the normal equations stops
    on |Mhat^dag r| / |Mhat^dag b|, so it is continued from its solution with a
    tighter bound until the residual of Mhat itself meets tol."""
    x, info = op.cg(b, tol=tol, max_iter=5000)
    iters, t = info["iters"], tol
    while info["rel_res"] > tol and t > tol * 1e-3:
        t *= 0.5
        x, info = op.cg(b, x=x, tol=t, max_iter=5000)
        iters += info["iters"]
    return x, dict(info, iters=iters)


def bench_solve(dims, dev, nrhs=8, kappa=0.16):
    """Even-odd clover system (b = kappa = 0.16, the kappa of the twisted-mass
    configuration) on the bench lattice solved to |b - Mhat x|/|b| <= 1e-10
    for nrhs Gaussian sources: (a) one FP64 CG per source (continued until
    its FP64 residual is <= 1e-10), (b) FP32-corrected-by-FP64 CG per source,
    (c) all sources at once with FP16-storage multi-RHS corrections of FP64
    solutions, (d) all sources in one FP16 multi-RHS CG with FP64 reliable
    updates (the speed-ups are those of (d)).  Each path runs once untimed
    first (module loading, workspaces), then three times; the median is
    reported."""
    from qphix_b200 import fields, layout, mrhs
    from qphix_b200.lattice import F16, F32, F64, Geometry
    from qphix_b200.solver import EvenOddOperator, mixed_solve
    G = Geometry(*dims, soalen=16, compress12=True, t_boundary=-1.0, ftype=F64)
    U = fields.random_gauge(G, seed=77, device=dev)
    gauge = [layout.pack_gauge(G, U, cb, torch.float64) for cb in (0, 1)]
    del U
    A1 = fields.random_clover(G, seed=78, device=dev)
    A0 = fields.invert_blocks(fields.random_clover(G, seed=79, device=dev))
    clov = [layout.pack_clover(G, A0, torch.float64), layout.pack_clover(G, A1, torch.float64)]
    del A0, A1
    p = dict(coeff_s=kappa, coeff_t_f=kappa, coeff_t_b=kappa, rho=0.0)
    ops_ = {}
    for ft, dt in ((F64, torch.float64), (F32, torch.float32), (F16, torch.float16)):
        gg = G.with_(ftype=ft)
        ops_[ft] = EvenOddOperator(gg, "clover", gauge=[x.to(dt) for x in gauge], clov=[x.to(dt) for x in clov],
                                   target_cb=1, **p)
    gen = torch.Generator(device=dev)
    gen.manual_seed(80)
    bs = [layout.pack_spinor(G, fields.random_spinor(G, seed=81 + i, device=dev), torch.float64)
          for i in range(nrhs)]
    out = {"lattice": list(dims), "nrhs": nrhs, "tol": 1e-10, "kappa": kappa, "family": "clover"}
    # warm-up of each path on one source
    ops_[F64].cg(bs[0], tol=1e-4, max_iter=50)
    mixed_solve(ops_[F64], ops_[F32], bs[0], tol=1e-4, inner_tol=1e-2)
    mrhs.mixed_solve(ops_[F64], ops_[F16], bs, tol=1e-3, inner_tol=1e-2)
    mrhs.mixed_solve(ops_[F64], ops_[F16], bs, tol=1e-3, inner_tol=1e-2, solver="cg_reliable")

    def timed(fn, reps=3):
        """median wall time of reps runs (each synchronised) and the last result"""
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return statistics.median(ts), r, ts

    t64, r64, a64 = timed(lambda: [fp64_cg(ops_[F64], b) for b in bs])
    out["fp64_cg"] = {"seconds": t64, "runs": a64, "iters": [r[1]["iters"] for r in r64],
                      "max_rel_res": max(r[1]["rel_res"] for r in r64)}
    t32, r32, a32 = timed(lambda: [mixed_solve(ops_[F64], ops_[F32], b, tol=1e-10, inner_tol=1e-5) for b in bs])
    out["fp32_fp64_single_rhs"] = {"seconds": t32, "runs": a32, "inner_iters": [r[1]["inner_iters"] for r in r32],
                                   "max_rel_res": max(r[1]["rel_res"] for r in r32)}
    t16, r16, a16 = timed(lambda: mrhs.mixed_solve(ops_[F64], ops_[F16], bs, tol=1e-10, inner_tol=1e-2))
    out["fp16_multi_rhs_mixed"] = {"seconds": t16, "runs": a16, "inner_iters": r16[1]["inner_iters"],
                                   "outer_iters": r16[1]["outer_iters"], "max_rel_res": max(r16[1]["rel_res"])}
    # one multi-RHS FP16 CG with FP64 reliable updates whenever the residuals fell 100x
    tr, rr_, ar = timed(lambda: mrhs.mixed_solve(ops_[F64], ops_[F16], bs, tol=1e-10, inner_tol=1e-2,
                                                 solver="cg_reliable"))
    out["fp16_multi_rhs_reliable"] = {"seconds": tr, "runs": ar, "iters": rr_[1]["inner_iters"],
                                      "updates": rr_[1]["outer_iters"], "max_rel_res": max(rr_[1]["rel_res"])}
    out["speedup_vs_fp32_fp64_single_rhs"] = t32 / tr
    out["speedup_vs_fp64_cg"] = t64 / tr
    return out


def tm_operators(G, dev, family, kappa, mu, types):
    """Even-odd operators of the twisted-mass ("tm") or twisted-mass clover
    ("tm_clover") system of bench_solve_tm on the FP64 geometry G, one per
    (storage type, torch dtype) in types, from the same seeded fields."""
    from qphix_b200 import fields, layout
    from qphix_b200.solver import EvenOddOperator
    U = fields.random_gauge(G, seed=177, device=dev)
    gauge = [layout.pack_gauge(G, U, cb, torch.float64) for cb in (0, 1)]
    del U
    ops_ = {}
    if family == "tm":
        alpha = 1.0 / (2 * kappa)
        p = dict(coeff_s=0.5, coeff_t_f=0.5, coeff_t_b=0.5, alpha=alpha, mu=mu / alpha,
                 muinv=alpha / (alpha ** 2 + mu ** 2))
        for ft, dt in types:
            ops_[ft] = EvenOddOperator(G.with_(ftype=ft), "tm", gauge=[x.to(dt) for x in gauge], target_cb=1, **p)
        return ops_
    mut = 2 * kappa * mu
    g5 = torch.tensor([1.0, -1.0], dtype=torch.float64, device=dev).reshape(2, 1, 1)
    eye = torch.eye(6, dtype=torch.complex128, device=dev)
    clov, clov_dag = [None, None], [None, None]
    for cb, seed in ((1, 178), (0, 179)):
        F = fields.random_full_clover(G, seed=seed, device=dev) + 1j * mut * g5 * eye
        if cb == 0:
            F = fields.invert_blocks(F)
        clov[cb] = layout.pack_full_clover(G, F, torch.float64)
        clov_dag[cb] = layout.pack_full_clover(G, F.conj().transpose(-1, -2), torch.float64)
        del F
    p = dict(coeff_s=kappa, coeff_t_f=kappa, coeff_t_b=kappa, rho=0.0)
    for ft, dt in types:
        ops_[ft] = EvenOddOperator(G.with_(ftype=ft), "tm_clover", gauge=[x.to(dt) for x in gauge],
                                   clov=[x.to(dt) for x in clov], clov_dag=[x.to(dt) for x in clov_dag],
                                   target_cb=1, **p)
    return ops_


def bench_solve_tm(dev, dims=(48, 48, 48, 96), kappa=0.16, mu=0.01, family="tm"):
    """Even-odd twisted-mass (family "tm") or twisted-mass clover ("tm_clover")
    system at 48^3x96, solved for one Gaussian source to |b - Mhat x|/|b| <=
    1e-10 by (a) FP64 CG on Mhat^dag Mhat, (b) FP32 CG corrected in FP64,
    (c) FP16 + per-site norm CG corrected in FP64 (the configuration's
    storage), (d) one FP16 + per-site norm CG with FP64 reliable updates (the
    speed-ups are those of (d)).  Twisted mass: M = 1/(2 kappa) (1 + i mu~
    gamma5) - D/2 with mu~ = 2 kappa mu (operator convention alpha = 1/(2
    kappa), mu = mu~ and muinv = alpha / (alpha^2 + mu^2) with the untwisted
    mu; hopping coefficient 1/2).  Twisted-mass clover: the dense
    FullCloverBlock F = I + 0.1 M + i mu~ gamma5 per block (M a seeded
    complex Gaussian 6x6 of unit Frobenius norm; gamma5 = +1 on the upper,
    -1 on the lower block), F_oo on the target checkerboard and F_ee^-1 on
    the other, hopping coefficient kappa.  The residual of every solution is
    recomputed with the FP64 operator.  Each path runs once untimed on a
    loose tolerance, then three times; the median is reported."""
    from qphix_b200 import fields, layout
    from qphix_b200.lattice import F16N, F32, F64, Geometry
    from qphix_b200.solver import mixed_solve
    G = Geometry(*dims, soalen=8, veclen=8, compress12=True, t_boundary=-1.0, ftype=F64)
    ops_ = tm_operators(G, dev, family, kappa, mu, ((F64, torch.float64), (F32, torch.float32),
                                                    (F16N, torch.float16)))
    b = layout.pack_spinor(G, fields.random_spinor(G, seed=181, device=dev), torch.float64)
    out = {"lattice": list(dims), "family": family, "kappa": kappa, "mu": mu, "tol": 1e-10,
           "inner_storage": "fp16 + per-site norm (links%s fp16, 12-real)" % (" and clover" if family != "tm" else ""),
           "soalen": 8}
    ops_[F64].cg(b, tol=1e-4, max_iter=50)
    mixed_solve(ops_[F64], ops_[F32], b, tol=1e-4, inner_tol=1e-2)
    mixed_solve(ops_[F64], ops_[F16N], b, tol=1e-4, inner_tol=1e-2)
    mixed_solve(ops_[F64], ops_[F16N], b, solver="cg_reliable", tol=1e-4, inner_tol=1e-2)

    def timed(fn, reps=3):
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return statistics.median(ts), r, ts

    def true_res(x):
        r = ops_[F64].apply(x)
        return float((b - r).norm() / b.norm())

    t64, r64, a64 = timed(lambda: fp64_cg(ops_[F64], b))
    out["fp64_cg"] = {"seconds": t64, "runs": a64, "iters": r64[1]["iters"], "rel_res": true_res(r64[0])}
    t32, r32, a32 = timed(lambda: mixed_solve(ops_[F64], ops_[F32], b, tol=1e-10, inner_tol=1e-5))
    out["fp32_fp64_mixed"] = {"seconds": t32, "runs": a32, "inner_iters": r32[1]["inner_iters"],
                              "outer_iters": r32[1]["outer_iters"], "rel_res": true_res(r32[0])}
    t16, r16, a16 = timed(lambda: mixed_solve(ops_[F64], ops_[F16N], b, tol=1e-10, inner_tol=1e-2))
    out["fp16n_fp64_mixed"] = {"seconds": t16, "runs": a16, "inner_iters": r16[1]["inner_iters"],
                               "outer_iters": r16[1]["outer_iters"], "rel_res": true_res(r16[0])}
    # one FP16+norm CG with FP64 reliable updates whenever the residual fell 100x
    tr, rr_, ar = timed(lambda: mixed_solve(ops_[F64], ops_[F16N], b, solver="cg_reliable", tol=1e-10,
                                            inner_tol=1e-2))
    out["fp16n_fp64_reliable"] = {"seconds": tr, "runs": ar, "iters": rr_[1]["inner_iters"],
                                  "updates": rr_[1]["outer_iters"], "rel_res": true_res(rr_[0])}
    out["speedup_vs_fp64_cg"] = t64 / tr
    out["speedup_vs_fp32_fp64_mixed"] = t32 / tr
    return out


def bench_solve_tm_mrhs(dev, dims=(48, 48, 48, 96), kappa=0.16, mu=0.01, nrhs=8, family="tm"):
    """The even-odd twisted-mass (family "tm") or twisted-mass clover
    ("tm_clover") system of bench_solve_tm (48^3x96, kappa = 0.16, mu = 0.01,
    12-real links, SOALEN 8) for nrhs Gaussian sources to |b - Mhat x|/|b| <=
    1e-10: (a) the single-RHS FP32 CG corrected in FP64, source by source,
    against (b) all sources in one FP16-storage multi-RHS CG with FP64
    reliable updates (links and clover FP16, each right-hand side scaled to
    unit norm in its FP16 slot).  Every solution's residual is recomputed
    with the FP64 operator.  One untimed run of each path on a loose
    tolerance, then three timed runs; the median is reported."""
    from qphix_b200 import fields, layout, mrhs
    from qphix_b200.lattice import F16, F32, F64, Geometry
    from qphix_b200.solver import mixed_solve
    G = Geometry(*dims, soalen=8, veclen=8, compress12=True, t_boundary=-1.0, ftype=F64)
    ops_ = tm_operators(G, dev, family, kappa, mu, ((F64, torch.float64), (F32, torch.float32),
                                                    (F16, torch.float16)))
    bs = [layout.pack_spinor(G, fields.random_spinor(G, seed=281 + i, device=dev), torch.float64)
          for i in range(nrhs)]
    out = {"lattice": list(dims), "family": family, "kappa": kappa, "mu": mu, "tol": 1e-10, "nrhs": nrhs,
           "soalen": 8, "inner_storage": "fp16 multi-RHS (links%s fp16, 12-real)" % (
               " and clover" if family != "tm" else "")}
    # the FP16 multi-RHS operator's two kernels on this lattice: the plain
    # dslash (other checkerboard) and the A.chi - b.D.psi form; bytes per
    # right-hand-side site: psi + out (+ chi) 48 each + 12-real FP16 links
    # 192 / nrhs (+ the FullCloverBlock's 288 / nrhs)
    g16 = G.with_(ftype=F16)
    stream = torch.cuda.current_stream()
    peak = measured_peak()[0]
    op16 = ops_[F16]
    mp = torch.randn(g16.spinor_elems * nrhs, device=dev).half()
    mc = torch.randn(g16.spinor_elems * nrhs, device=dev).half()
    mo = torch.zeros_like(mp)
    if family == "tm":
        alpha = 1.0 / (2 * kappa)
        kw = dict(coeff_s=0.5, coeff_t_f=0.5, coeff_t_b=0.5, mu=mu / alpha, muinv=alpha / (alpha ** 2 + mu ** 2))
        fixed, cl_b = {}, 0
    else:
        alpha = 1.0
        kw = dict(coeff_s=kappa, coeff_t_f=kappa, coeff_t_b=kappa)
        fixed, cl_b = {"clover": op16.keep[1][1]}, 288
    n_rs = g16.vol_cb * nrhs
    for kern, extra, bps in (("dslash", {}, 96 + (192 + cl_b) / nrhs),
                             ("achimbdpsi", {"chi": mc, "alpha": alpha}, 144 + (192 + cl_b) / nrhs)):
        ms = _time(lambda: mrhs.dslash(g16, nrhs, family, kern, 1, 0, mp, mo, op16.keep[0][0], **fixed, **extra, **kw),
                   20, stream)
        out["mrhs_%s_%s" % (family, kern)] = {"ms": ms, "gbs": bps * n_rs / (ms * 1e-3) / 1e9,
                                              "frac_of_peak": bps * n_rs / (ms * 1e-3) / 1e9 / peak,
                                              "bytes_per_rhs_site": bps}
    del mp, mc, mo
    mixed_solve(ops_[F64], ops_[F32], bs[0], tol=1e-4, inner_tol=1e-2)
    mrhs.mixed_solve(ops_[F64], ops_[F16], bs, tol=1e-3, inner_tol=1e-2, solver="cg_reliable")

    def timed(fn, reps=3):
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return statistics.median(ts), r, ts

    def true_res(b, x):
        return float((b - ops_[F64].apply(x)).norm() / b.norm())

    t32, r32, a32 = timed(lambda: [mixed_solve(ops_[F64], ops_[F32], b, tol=1e-10, inner_tol=1e-5) for b in bs])
    out["fp32_fp64_single_rhs"] = {"seconds": t32, "runs": a32, "inner_iters": [r[1]["inner_iters"] for r in r32],
                                   "max_rel_res": max(true_res(b, r[0]) for b, r in zip(bs, r32))}
    del r32
    tr, rr_, ar = timed(lambda: mrhs.mixed_solve(ops_[F64], ops_[F16], bs, tol=1e-10, inner_tol=1e-2,
                                                 solver="cg_reliable"))
    out["fp16_multi_rhs_reliable"] = {"seconds": tr, "runs": ar, "iters": rr_[1]["inner_iters"],
                                      "updates": rr_[1]["outer_iters"],
                                      "max_rel_res": max(true_res(b, x) for b, x in zip(bs, rr_[0]))}
    out["speedup_vs_fp32_fp64_single_rhs"] = t32 / tr
    return out


def bench_force(dev, dims=(24, 24, 24, 48)):
    """Backward of the hopping term at 24^3x48, FP32, 18-real links: the
    link-force kernel (plain and su(3)-projected) against its algorithmic
    bytes (chi + psi read once, 8 x 72 B written per site; + 8 x 72 B of links
    when projecting), the forward dslash it differentiates, and one full
    torch.autograd step (forward, dagger for the spinor cotangent, force,
    fold onto the full-lattice links)."""
    from qphix_b200 import autograd as AG
    from qphix_b200 import fields, layout, ops
    from qphix_b200.lattice import F32, Geometry
    g = Geometry(*dims, soalen=4, ftype=F32, t_boundary=-1.0)     # nx/2 = 12 sites: SOALEN 4
    n = g.vol_cb
    stream = torch.cuda.current_stream()
    U = fields.random_gauge(g, seed=90, device=dev).to(torch.complex64)
    gauge0 = layout.pack_gauge(g, U, 0)
    psi = layout.pack_spinor(g, fields.random_spinor(g, seed=91, device=dev))
    chi = layout.pack_spinor(g, fields.random_spinor(g, seed=92, device=dev))
    F = torch.empty(144 * n, dtype=torch.float32, device=dev)
    out = torch.zeros_like(psi)
    t_force = _time(lambda: AG.hop_force(g, 0, 1, chi, psi, out=F), 20, stream)
    t_proj = _time(lambda: AG.hop_force(g, 0, 1, chi, psi, gauge0, out=F), 20, stream)
    t_fwd = _time(lambda: ops.dslash(g, "wilson", "dslash", 1, 0, psi, out, gauge0), 20, stream)
    Ur = U.clone().requires_grad_(True)
    pr = psi.clone().requires_grad_(True)

    def step():
        Ur.grad = None
        pr.grad = None
        (chi * AG.WilsonHop.apply(pr, Ur, g, 0, 1, None)).sum().backward()

    t_step = _time(step, 5, stream)
    b_force, b_proj = 96 + 96 + 576, 96 + 96 + 576 + 576
    return {"lattice": list(dims), "dtype": "f32", "sites_per_cb": n,
            "force_ms": t_force, "force_gbs": b_force * n / (t_force * 1e-3) / 1e9, "force_bytes_per_site": b_force,
            "projected_force_ms": t_proj, "projected_force_gbs": b_proj * n / (t_proj * 1e-3) / 1e9,
            "projected_force_bytes_per_site": b_proj, "wilson_dslash_ms": t_fwd,
            "autograd_step_ms": t_step,
            "note": "autograd step = forward dslash + dagger dslash + force + torch packing/folding of links"}


def bench_batch(dev, peak):
    """Clover A.chi - b.D.psi (FP32, 12-real links, SOALEN = VECLEN = 4) over
    the uneven batch 3 x 16^3x32 + 2 x 24^3x48 + 1 x 32^3x64 (seeded random
    fields; 960 algorithmic bytes and 1824 flop per site): one launch per
    lattice, one batched launch (one thread per site), the tuned batched
    launch, and ten tuned launches replayed from a CUDA graph."""
    from qphix_b200 import batch, ops
    from qphix_b200.lattice import F32, Geometry
    dims = [(16, 16, 16, 32)] * 3 + [(24, 24, 24, 48)] * 2 + [(32, 32, 32, 64)]
    gen = torch.Generator(device=dev)
    gen.manual_seed(95)
    probs = []
    for d in dims:
        g = Geometry(*d, soalen=4, veclen=4, ftype=F32, compress12=True, t_boundary=-1.0)
        r = lambda n: torch.randn(n, generator=gen, device=dev)  # noqa: E731
        probs.append(batch.Problem(g, 0, r(g.spinor_elems), torch.zeros(g.spinor_elems, device=dev),
                                   r(g.gauge_elems), chi=r(g.spinor_elems), clover=r(g.clover_elems), **PARAMS))
    sites = sum(p.g.vol_cb for p in probs)
    stream = torch.cuda.current_stream()
    op = batch.BatchedDslash("clover", "achimbdpsi", 1, probs)

    def seq():
        for p in probs:
            ops.dslash(p.g, "clover", "achimbdpsi", 1, 0, p.psi, p.out, p.gauge, chi=p.chi, clover=p.clover,
                       **PARAMS)

    res = {"lattices": ["x".join(map(str, d)) for d in dims], "sites": sites, "bytes_per_site": 960}
    t_seq = _time(seq, 20, stream)
    t_one = _time(lambda: op(grid=0, block=128), 20, stream)
    grid, block, _ = op.tune()
    t_tuned = _time(op, 20, stream)
    graph = op.capture(steps=10)
    t_graph = _time(graph.replay, 5, stream) / 10
    for name, t in (("per_lattice_launches", t_seq), ("batched_one_thread_per_site", t_one),
                    ("batched_tuned", t_tuned), ("batched_tuned_graph", t_graph)):
        gbs = 960 * sites / (t * 1e-3) / 1e9
        res[name] = {"ms": t, "gflops": FLOP_SITE * sites / (t * 1e-3) / 1e9, "gbs": gbs, "frac_of_peak": gbs / peak}
    res["tuned_launch"] = {"grid": grid, "block": block}
    del graph
    return res


def bench_tm(dev, dims=(48, 48, 48, 96)):
    """Twisted-mass dslash, and twisted-mass clover, at 48^3x96 with FP16
    spinors scaled by a per-site norm (QB200_F16N; links and clover FP16,
    12-real links), SOALEN = VECLEN = 8 (nx/2 = 24).  mu = 0.01, kappa = 0.16:
    alpha = 1/(2 kappa), mu~ = mu/alpha and muinv = alpha/(alpha^2 + mu^2)
    as the caller passes them.  Algorithmic bytes per site: psi + out
    (24 halves + 4-byte norm each) + 8 x 12 halves of links = 296 (+ 2 x 144
    halves of clover for TM clover = 584); flop per site: 1320 + 72 (TM) or
    1320 + 504 (TM clover, counted as clover)."""
    from qphix_b200 import fields, layout, ops
    from qphix_b200.lattice import F16N, Geometry
    g = Geometry(*dims, soalen=8, veclen=8, ftype=F16N, compress12=True, t_boundary=-1.0)
    U = fields.random_gauge(g, seed=96, device=dev)
    gauge = layout.pack_gauge(g, U, 0)
    del U
    psi = layout.pack_spinor(g, fields.random_spinor(g, seed=97, device=dev))
    fcl = layout.pack_full_clover(g, fields.random_full_clover(g, seed=98, device=dev))
    out = torch.zeros_like(psi)
    kappa, mu = 0.16, 0.01
    alpha = 1.0 / (2 * kappa)
    kw = dict(coeff_s=1.0, coeff_t_f=1.0, coeff_t_b=1.0, mu=mu / alpha, muinv=alpha / (alpha ** 2 + mu ** 2))
    stream = torch.cuda.current_stream()
    peak = measured_peak()[0]
    n = g.vol_cb
    res = {"lattice": list(dims), "storage": "fp16 + per-site norm", "soalen": 8, "sites_per_cb": n}
    t = _time(lambda: ops.dslash(g, "tm", "dslash", 1, 0, psi, out, gauge, **kw), 20, stream)
    res["tm_dslash"] = {"ms": t, "gbs": 296 * n / (t * 1e-3) / 1e9, "frac_of_peak": 296 * n / (t * 1e-3) / 1e9 / peak,
                        "gflops": 1392 * n / (t * 1e-3) / 1e9, "bytes_per_site": 296}
    t = _time(lambda: ops.dslash(g, "tm_clover", "dslash", 1, 0, psi, out, gauge, clover=fcl), 20, stream)
    res["tm_clover_dslash"] = {"ms": t, "gbs": 584 * n / (t * 1e-3) / 1e9,
                               "frac_of_peak": 584 * n / (t * 1e-3) / 1e9 / peak,
                               "gflops": FLOP_SITE * n / (t * 1e-3) / 1e9, "bytes_per_site": 584}
    return res


def site_rel_err(ga, a, gb, b):
    """max over spinor components of |a - b| / max(|b_i|, rms of b's site):
    the per-component relative error (a, b: spinor arrays of lattices ga, gb)"""
    from qphix_b200 import layout
    ta = layout.unpack_spinor(ga, a.detach().cpu()).reshape(-1, 12)
    tb = layout.unpack_spinor(gb, b.detach().cpu()).reshape(-1, 12)
    ra = torch.cat([ta.real, ta.imag], 1).double()
    rb = torch.cat([tb.real, tb.imag], 1).double()
    site = (rb.pow(2).sum(1, keepdim=True) / 24).sqrt()
    den = torch.maximum(rb.abs(), site).clamp_min(1e-300)
    return float(((ra - rb).abs() / den).max())


def cpu_baselines(g, f, dims, seconds, kernel, flop_site=FLOP_SITE):
    """The reference's AVX512 (or the best the host runs) and scalar builds
    on all host threads, each on a bounded sample of the same workload and
    the same inputs as the GPU; the first is the baseline, both are listed
    with their per-component difference from the GPU result."""
    from qphix_b200 import ops
    builds = []
    names = [n for n in (pick_reference_lib(), "scalar_f32") if n]
    names = list(dict.fromkeys(names))
    out = torch.zeros_like(f["psi"])
    ops.dslash(g, "clover", kernel, 1, 0, f["psi"], out, f["gauge"], chi=f["chi"], clover=f["clover"], **PARAMS)
    torch.cuda.synchronize()
    import oracle as O
    for i, name in enumerate(names):
        r = run_reference_cpu(dims, 1000, 1, seconds if i == 0 else seconds / 2, fields_gpu=f, g_gpu=g, name=name,
                              kernel=kernel, flop_site=flop_site)
        if "unavailable" in r:
            builds.append({"lib": name, "unavailable": r["unavailable"]})
            continue
        info = O.ref_info(r["lib"])
        gr = g.with_(soalen=info["soalen"], veclen=info["veclen"])
        b = torch.from_numpy(r["out"][: gr.spinor_elems].copy())
        e = {k: r[k] for k in ("value", "unit", "cores", "kind", "sample", "lib", "ms_per_step")}
        e["rel_err_vs_gpu"] = site_rel_err(gr, b, g, out)
        builds.append(e)
    ok = [b for b in builds if "value" in b]
    if not ok:
        return {"unavailable": "reference kernels not built (python oracle/ref_build.py)"}
    cpu = {k: ok[0][k] for k in ("value", "unit", "cores", "kind", "sample")}
    cpu["builds"] = builds
    return cpu


def bench_inverse_clover(g, f, dims, dev, peak, cpu_seconds):
    """The inverse-clover variant: the plain clov_dslash_plus with A^-1
    (FP64 block inverses of the clover blocks I + 0.1 H, packed to FP32) on
    the headline lattice and layout.  1824 flop/site; 864 algorithmic
    bytes/site (psi 96 + out 96 + 8 links x 48 + clover 288).  The
    reference's builds run the same call on the same inputs (bounded CPU
    samples)."""
    from qphix_b200 import fields, layout, ops
    A = fields.random_clover(g, seed=1234 + 3, device=dev)
    Ainv = layout.pack_clover(g, fields.invert_blocks(A))
    del A
    fi = dict(f, clover=Ainv)
    out = torch.zeros_like(f["psi"])
    stream = torch.cuda.current_stream()
    ms = _time(lambda: ops.dslash(g, "clover", "dslash", 1, 0, fi["psi"], out, fi["gauge"], clover=fi["clover"],
                                  **PARAMS), 50, stream)
    bps = 864
    res = {"workload": "clov_dslash_plus with A^-1, %s FP32 compress12 SOALEN %d" % ("x".join(map(str, dims)),
                                                                                  g.soalen),
           "ms": ms, "gflops": FLOP_SITE * g.vol_cb / (ms * 1e-3) / 1e9,
           "gbs": bps * g.vol_cb / (ms * 1e-3) / 1e9, "bytes_per_site": bps}
    res["frac_of_peak"] = res["gbs"] / peak
    if cpu_seconds:
        res["cpu_baseline"] = cpu_baselines(g, fi, dims, cpu_seconds, "dslash")
    return res


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl == "b200" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def reference_arm(args, world, rank):
    dims = tuple(int(x) for x in args.dims.split(","))
    if rank != 0:
        return
    r = run_reference_cpu(dims, args.steps, args.warmup, 1e9)
    if "unavailable" in r:
        print(json.dumps({"impl": "reference", "unavailable": r["unavailable"]}))
        return
    line = {
        "metric": METRIC, "value": r["value"], "unit": "GFLOP/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
        "config": {"workload": WORKLOAD, "dims": list(dims), "layout": r["lib"], "host_threads": r["cores"]},
        "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": r["value"], "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def b200_arm(args, world, rank, local):
    import torch.distributed as dist
    from qphix_b200 import ops
    from qphix_b200.halo import GPUKernels, TComm, TSlabDslash
    from qphix_b200.lattice import F32, Geometry

    dev = torch.device("cuda", local)
    dims = tuple(int(x) for x in args.dims.split(","))
    G = Geometry(dims[0], dims[1], dims[2], dims[3] * world, soalen=args.soalen, veclen=args.veclen,
                 ftype=F32, compress12=True, t_boundary=-1.0)
    from qphix_b200.halo import local_geometry
    g = local_geometry(G, rank, world)
    f = make_fields(g, dev, seed=1234 + 17 * rank)
    out = torch.zeros_like(f["psi"])
    op = TSlabDslash(g, TComm(), GPUKernels(torch.float32, dev))
    stream = torch.cuda.current_stream()

    def step():
        op.apply("clover", "achimbdpsi", 1, 0, f["psi"], out, f["gauge"], chi=f["chi"], clover=f["clover"],
                 **PARAMS)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(max(3, args.warmup)):
        step()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index if dev.index is not None else 0) as clk:
        barrier()
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        barrier()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    sites_all = g.vol_cb * world
    gflops = FLOP_SITE * sites_all / (ms_step * 1e-3) / 1e9
    launches_per_step = 1 if world == 1 else 5

    # a window of the same step after the timed region, long enough (about
    # 0.3 s) for dozens of clock samples even when the timed region is a few
    # milliseconds; its time x median SM clock ties the two together
    nwin = max(50, min(20000, int(300.0 / max(ms_step, 1e-3))))
    w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index if dev.index is not None else 0) as clkw:
        barrier()
        w0.record(stream)
        for _ in range(nwin):
            step()
        w1.record(stream)
        barrier()
    win_ms = w0.elapsed_time(w1) / nwin
    cw = clkw.summary()
    clock_window = {"steps": nwin, "ms_per_step": win_ms, "sm_mhz": cw.get("sm_mhz"), "samples": cw.get("samples"),
                    "reasons": cw.get("reasons"),
                    "ms_x_mhz": win_ms * cw["sm_mhz"] if cw.get("sm_mhz") else None,
                    "timed_region_ms_x_mhz": (ms_step * clk.summary()["sm_mhz"]
                                              if clk.summary().get("sm_mhz") else None)}

    # roofline of the body kernel: its own events over the same timed region
    bps = bytes_per_site()
    if world == 1:
        launch_ms = ms_step
    else:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            ops.dslash(g, "clover", "achimbdpsi", 1, 0, f["psi"], out, f["gauge"], chi=f["chi"],
                       clover=f["clover"], **PARAMS)
        e1.record(stream)
        barrier()
        launch_ms = e0.elapsed_time(e1) / args.steps
    achieved = bps * g.vol_cb / (launch_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    key = "clov_dslash_achimbdpsi_f32_c12_s%d_v%d_%s" % (g.soalen, g.veclen, "x".join(map(str, dims)))
    traffic = traffic_from_profile(key)

    # e2e through the public API with host buffers: H2D psi, chi -> dslash -> D2H out
    e2e = None
    if world == 1 and args.e2e_steps > 0:
        hpsi = f["psi"].cpu().pin_memory()
        hchi = f["chi"].cpu().pin_memory()
        nb = f["psi"].numel() * 4
        # serial: each step copies in, computes and copies out on one stream
        hout = torch.empty_like(hpsi).pin_memory()
        dpsi, dchi = torch.empty_like(f["psi"]), torch.empty_like(f["chi"])

        def e2e_step():
            dpsi.copy_(hpsi, non_blocking=True)
            dchi.copy_(hchi, non_blocking=True)
            ops.dslash(g, "clover", "achimbdpsi", 1, 0, dpsi, out, f["gauge"], chi=dchi, clover=f["clover"],
                       **PARAMS)
            hout.copy_(out, non_blocking=True)

        for _ in range(2):
            e2e_step()
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(args.e2e_steps):
            e2e_step()
        a1.record(stream)
        torch.cuda.synchronize()
        serial_ms = a0.elapsed_time(a1) / args.e2e_steps
        # pipelined: double buffers on three streams, so that the host-to-device
        # copies of step i+1 overlap the device-to-host copy of step i (the PCIe
        # link carries both directions at once)
        s_in, s_run, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
        bufs = [(torch.empty_like(f["psi"]), torch.empty_like(f["chi"]), torch.empty_like(out),
                 torch.empty_like(hpsi).pin_memory()) for _ in range(2)]
        ev_in = [torch.cuda.Event() for _ in range(2)]
        ev_run = [torch.cuda.Event() for _ in range(2)]
        ev_out = [torch.cuda.Event() for _ in range(2)]

        def pipelined(nsteps):
            for i in range(nsteps):
                b = i % 2
                bp, bc, bo, bh = bufs[b]
                if i >= 2:
                    s_in.wait_event(ev_run[b])          # step i-2 has read this input buffer
                with torch.cuda.stream(s_in):
                    bp.copy_(hpsi, non_blocking=True)
                    bc.copy_(hchi, non_blocking=True)
                    ev_in[b].record(s_in)
                s_run.wait_event(ev_in[b])
                if i >= 2:
                    s_run.wait_event(ev_out[b])         # step i-2's result has left this buffer
                ops.dslash(g, "clover", "achimbdpsi", 1, 0, bp, bo, f["gauge"], chi=bc, clover=f["clover"],
                           stream=s_run, **PARAMS)
                ev_run[b].record(s_run)
                s_out.wait_event(ev_run[b])
                with torch.cuda.stream(s_out):
                    bh.copy_(bo, non_blocking=True)
                    ev_out[b].record(s_out)

        pipelined(2)
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(s_in)
        pipelined(args.e2e_steps)
        p1.record(s_out)
        torch.cuda.synchronize()
        e_ms = p0.elapsed_time(p1) / args.e2e_steps
        assert torch.equal(bufs[(args.e2e_steps - 1) % 2][3], hout), "pipelined result differs from the serial one"
        e2e = {"value": FLOP_SITE * g.vol_cb / (e_ms * 1e-3) / 1e9, "unit": "GFLOP/s",
               "h2d_bytes_per_step": 2 * nb, "d2h_bytes_per_step": nb, "ms_per_step": e_ms,
               "serial_ms_per_step": serial_ms,
               "path": ("qb200_clov_dslash_achimbdpsi_plus_vec via ctypes, pinned host buffers; psi and chi "
                        "copied in and out copied back every step, double-buffered over steps")}

    cpu = None
    inv = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baselines(g, f, dims, args.cpu_seconds, "achimbdpsi")
    if rank == 0 and world == 1 and not args.no_extras:
        inv = bench_inverse_clover(g, f, dims, dev, peak, None if args.no_cpu_baseline else args.cpu_seconds / 2)

    extras = {}
    if inv is not None:
        extras["inverse_clover"] = inv
    if world == 1 and not args.no_extras:
        extras["mrhs"] = bench_mrhs(g, f, dev)
        extras["solve"] = bench_solve(dims, dev)
        extras["force"] = bench_force(dev)
        extras["batch"] = bench_batch(dev, peak)
        extras["tm_fp16n"] = bench_tm(dev)
        extras["solve_tm"] = bench_solve_tm(dev)
        extras["solve_tm_clover"] = bench_solve_tm(dev, family="tm_clover")
        extras["solve_tm_mrhs"] = bench_solve_tm_mrhs(dev)
        extras["solve_tm_clover_mrhs"] = bench_solve_tm_mrhs(dev, family="tm_clover")

    if rank == 0:
        line = {
            "metric": METRIC, "value": gflops, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "dims_per_gpu": list(dims), "global_dims": list(G.dims),
                       "soalen": g.soalen, "veclen": g.veclen, "cb_sites_per_gpu": g.vol_cb,
                       "parallelism": "t-slab halo over %d GPUs" % world if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (%.2f GB per step)" % (bps * g.vol_cb / 1e9),
                       "flop_per_site": FLOP_SITE, "bytes_per_site": bps},
            "gbs": achieved,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel_ms": launch_ms},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clk.summary(clkw),
            "clocks_timed_region": clk.summary(),
            "clock_window": clock_window,
        }
        line.update(extras)
        print(json.dumps(line))
    if world > 1:
        dist.barrier()


def run_only(args):
    """One secondary measurement alone, for profiling it on a chosen size."""
    dev = torch.device("cuda", 0)
    dims = tuple(int(x) for x in args.dims.split(","))
    if args.only == "mrhs":
        from qphix_b200.lattice import F32, Geometry
        g = Geometry(*dims, soalen=args.soalen, veclen=args.veclen, ftype=F32, compress12=True, t_boundary=-1.0)
        r = bench_mrhs(g, make_fields(g, dev), dev)
    elif args.only == "force":
        r = bench_force(dev, dims)
    elif args.only == "batch":
        r = bench_batch(dev, measured_peak()[0])
    elif args.only == "tm":
        r = bench_tm(dev, dims)
    elif args.only == "solve_tm":
        r = bench_solve_tm(dev, dims)
    elif args.only == "solve_tm_clover":
        r = bench_solve_tm(dev, dims, family="tm_clover")
    elif args.only == "solve_tm_mrhs":
        r = bench_solve_tm_mrhs(dev, dims, nrhs=args.nrhs)
    elif args.only == "solve_tm_clover_mrhs":
        r = bench_solve_tm_mrhs(dev, dims, nrhs=args.nrhs, family="tm_clover")
    else:
        r = bench_solve(dims, dev)
    print(json.dumps({"only": args.only, "dims": list(dims), "result": r}))


def main():
    args = parse()
    if args.only:
        run_only(args)
        return
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            reference_arm(args, world, rank)
        else:
            b200_arm(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
