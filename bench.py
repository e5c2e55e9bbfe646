"""Benchmark: full decomposition (first pass + matte refinement) throughput.

Workload (one step): the 1024x1024, 5-layer synthetic image (normal,
multiply, screen, overlay, color-dodge; alpha blobs 20-200 px; seed 2 + rank),
colour unmixing then matte refinement with an opaque, smoothed background
(the reference CLI's configuration, unblending-cli/main.cpp:58-66) and the
reference's refinement radius 60*min(w,h)/1000 = 61.

  value      : pixels/s of the library's default solve (the v1 ABI's: the
               reference's FP64 method and arithmetic, which meets the parity
               bar), image resident in HBM, per-step device time from CUDA
               events on the launching stream; a 256 MiB buffer is written
               between steps (L2 flush, untimed).
  e2e        : the same through the v1 C ABI calls unblending_unmix +
               unblending_refine with pinned host buffers (uploads, the first
               pass's host round trip and downloads inside the timed region).
  e2e_pageable : the same calls with plain pageable host buffers, which the
               library copies through its page-locked staging chunks.
  fp32       : the FP32 solve with its FP64 check and FP64 re-solve of misses
               (faster, below the parity bar: ~1 % of pixels stop more than
               1e-3 from the reference's result).
  warm_start : the default solve started from the learned start (network
               trained beforehand on 64 seeded 256x256 images of the same layer
               set, 2^22 pixels, batch 8192, Adam lr 1e-3), misses re-solved
               from the reference's start.
  parity     : every output above against the reference's own FP64 solver
               (oracle/_ref, compiled from its sources; else the oracle) over
               the whole image, both passes.
  cpu_baseline : that same whole-image reference decomposition, timed on all
               host cores (nothing extrapolated).
  rgb256_l3 / rgb4096_l6 : the BASELINE's 256x256 three-layer (r = 4) and
               4096x4096 six-layer (r = 8, colour noise) configurations, timed
               with the default solve, with their parity (whole image / a
               16384-pixel sample).

`--workload batch64`: the batched first pass over 64 images (sides 256-2048,
3-6 layers, one shared layer set per layer count).

Multi-GPU: one process per GPU, each decomposing its own image (weak
scaling, no collective on the data path); time = max over ranks.

`--impl reference` times the reference's own CPU implementation
(oracle/_ref: the reference's FP64 solver and CPU guided filter compiled from
its sources; else the oracle restatement) on all host cores: each step is the
full decomposition of one 128-row band of the image (both solves of its
pixels, the guided filter over the band and the two radii of rows each side
that its windows reach), so each step's time is what ran.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "pixels/sec, full decomposition, warm-start vs plain on B200 at ≤1e-3 RGBA err"
UNIT = "pixels/s"
WORKLOAD = "rgb1024_l5"
# Nominal CUDA-core peaks (MEASURED_PEAKS.json has neither): SMs x lanes x FMA x max clock.
PEAK_FP64_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12
PEAK_FP32_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12
PARITY_SAMPLE = 16384      # pixels of the sampled parity checks
BAND_ROWS = 128            # rows per step of the reference arm
PROFILES = os.path.join(ROOT, "profiles")


def load_workload(name, width=None, rank=0):
    """A named single-image workload (its own seed + rank)."""
    from unblending_b200 import synthetic as syn
    seed = syn.WORKLOADS[name]["seed"] + rank
    return syn.workload(name, width, width, seed=seed)


def refinement_radius(wl):
    from unblending_b200 import synthetic as syn
    return wl.radius if wl.radius is not None else syn.reference_radius(wl.width, wl.height)


def workload_label(wl):
    return (f"{wl.name} {wl.width}x{wl.height} L={len(wl.layers)} unmix+refine(opaque, smooth bg, "
            f"r={refinement_radius(wl)})")


def config(wl, world):
    """The `config` of both arms' lines (same keys and workload)."""
    return {"workload": workload_label(wl), "precision": "fp64 (the reference's FP64 method and arithmetic)",
            "warm_start": False, "starts": 1, "l2": "256 MiB buffer written between steps, outside the timed region",
            "parallelism": f"{world} independent images (one per GPU)"}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default=WORKLOAD, choices=["rgb1024_l5", "rgb4096_l6", "batch64"])
    p.add_argument("--width", type=int, default=None, help="square side (default: the workload's own)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-warm", action="store_true")
    p.add_argument("--no-fp32", action="store_true")
    p.add_argument("--no-configs", action="store_true", help="skip the rgb256_l3 / rgb4096_l6 keys")
    p.add_argument("--fp64-variant", type=int, default=-1, help="FP64 kernel variant of the default solve (-1: tuned)")
    p.add_argument("--pixel-order", type=int, default=1, choices=[0, 1],
                   help="work-queue order of the default solve: 1 grouped by colour (default), 0 image order")
    return p.parse_args()


# ---------------------------------------------------------------- clocks --
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        num = lambda v: v.replace('.', '', 1).isdigit()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and num(r[1])]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and num(r[2])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows if len(r) >= 9 for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------ flop count --
def evaluation_flops(L: int, modes: list[int]) -> tuple[float, float]:
    """Algorithmic flops of one value evaluation and of one value+gradient
    evaluation of the per-pixel objective: composite 3 channels x (L-1)
    layers, 3x3 Gaussian prior per layer, AL rows; the gradient adds the
    (P+P^T) rows and the reverse sweep. add/mul = 1, fma = 2, division/sqrt = 1.
    The same count serves both precisions (the same arithmetic)."""
    blend_v = {0: 0, 1: 1, 2: 3, 3: 4, 4: 1, 5: 1, 6: 3, 7: 4, 8: 4, 9: 8, 10: 1, 11: 4, 12: 1}
    blend_g = {0: 0, 1: 1, 2: 5, 3: 6, 4: 1, 5: 1, 6: 7, 7: 8, 8: 6, 9: 14, 10: 1, 11: 8, 12: 1}
    val = 0.0
    for l in range(1, L):
        val += 7                                   # composite alpha A_l
        val += 3 * (blend_v[modes[l]] + 11 + 1)    # per channel: pre (11) + divide
    val += L * (3 + 3 * 5 + 5 + 2)                 # deltas, P delta, quadratic form, alpha*D
    val += L + 4 * 5                               # minimum term, AL rows
    grad = val
    grad += L * 3 * (6 + 1)                        # (P + P^T) rows, scale by alpha
    for l in range(1, L):
        grad += 8                                  # da, db
        grad += 3 * (blend_g[modes[l]] + 30)       # ds, dc, pa, pd, ga, gp, gradient, adjoint
    return val, grad


ITERATION_EDGES = [0, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096]


def iteration_histogram(c):
    """Per-pixel work of one pass from its (n, 5) counters: a histogram of the
    L-BFGS iterations a pixel took over all its outer steps (bins
    [edge_k, edge_k+1), the last open), the outer-step counts, and quantiles.
    A pixel that an FP32 solve missed carries the counts of its FP64 re-solve,
    the solve that produced its output."""
    it, outer = c[:, 2], c[:, 4]
    bins = ITERATION_EDGES + [int(max(it.max(), ITERATION_EDGES[-1])) + 1]
    counts, _ = np.histogram(it, bins=bins)
    q = np.quantile(it, [0.5, 0.9, 0.99, 0.999])
    return {"iterations": {"edges": ITERATION_EDGES, "counts": counts.tolist(),
                           "p50": float(q[0]), "p90": float(q[1]), "p99": float(q[2]), "p99.9": float(q[3]),
                           "max": int(it.max()), "mean": float(it.mean())},
            "outer_steps": {str(k): int(v) for k, v in enumerate(np.bincount(outer)) if v}}


def profile_traffic(name):
    """DRAM bytes per pixel of one solve launch from the committed ncu summary
    `profiles/<name>` (its line `dram_bytes_per_pixel: <value>`), or None."""
    path = os.path.join(PROFILES, name)
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_pixel:"):
            return float(line.split(":", 1)[1])
    return None


# ------------------------------------------------------------ reference --
def reference_impl():
    """The reference's CPU implementation: its own FP64 solver and CPU
    guided filter compiled from its sources (oracle/_ref), else the oracle
    restatement."""
    import oracle
    impl = oracle.ref_lib()
    return (impl, "reference") if impl is not None else (oracle.lib(), "port")


def reference_targets(impl, kind, wl, first_x, rows, threads):
    """Refinement targets (L+3, pixels of `rows`) of the reference's CPU
    guided filter, run over rows [rows) plus the rows its two box passes
    reach on either side (2r), from the pixel-major first pass first_x."""
    import oracle
    from unblending_b200 import synthetic as syn
    L, w, h = len(wl.layers), wl.width, wl.height
    r = refinement_radius(wl)
    y0, y1 = rows
    s0, s1 = max(0, y0 - 2 * r), min(h, y1 + 2 * r)
    sub = slice(s0 * w, s1 * w)
    rgb_planar = wl.image.reshape(-1, 3)[sub].T.copy()
    first_planar = first_x[sub].T.copy()
    layers = syn.layer_array(wl.layers)
    sh = s1 - s0
    if kind == "reference":
        targets = np.zeros((L + 3, sh * w))
        status = np.zeros(sh * w, np.int32)
        impl.dll.ref_refine_targets(rgb_planar.ctypes.data_as(oracle._dp), first_planar.ctypes.data_as(oracle._dp),
                                    layers, L, w, sh, 1, 1, r, threads, targets.ctypes.data_as(oracle._dp),
                                    status.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    else:
        targets, status = oracle.refine_targets(rgb_planar, first_planar, layers, L, w, sh, True, True, r)
    k0 = (y0 - s0) * w
    return targets[:, k0:k0 + (y1 - y0) * w]


def reference_refine(impl, wl, first_x, targets, idx, threads):
    """The reference's refinement solve of pixels idx from the first pass
    first_x (pixel-major) with filter targets (L+3, len(idx))."""
    import oracle
    from unblending_b200 import synthetic as syn
    L = len(wl.layers)
    alpha = targets[:L].T.copy()
    bg = targets[L:L + 3].T.copy()
    init = first_x[idx].copy()
    init[:, :L] = alpha
    init[:, 0] = 1.0
    init[:, L:L + 3] = bg
    x, _ = impl.solve(syn.layer_array(wl.layers), oracle.problem(L, True, True, True), oracle.options(),
                      wl.image.reshape(-1, 3)[idx], init, alpha=alpha, bg=bg, threads=threads)
    x[:, :L] = alpha
    x[:, L:L + 3] = bg
    return x


def reference_unmix(impl, wl, idx, threads):
    import oracle
    from unblending_b200 import synthetic as syn
    L = len(wl.layers)
    x, _ = impl.solve(syn.layer_array(wl.layers), oracle.problem(L, False, True), oracle.options(),
                      wl.image.reshape(-1, 3)[idx], np.tile(oracle.initial_first(wl.layers, True), (len(idx), 1)),
                      threads=threads)
    return x


def reference_decomposition(wl, threads):
    """The reference's full decomposition of the whole image on `threads`
    host cores, timed per stage. Returns (first_x, final_x, seconds, kind)."""
    impl, kind = reference_impl()
    n, h = wl.pixels, wl.height
    idx = np.arange(n)
    t0 = time.perf_counter()
    first = reference_unmix(impl, wl, idx, threads)
    t1 = time.perf_counter()
    targets = reference_targets(impl, kind, wl, first, (0, h), threads)
    t2 = time.perf_counter()
    final = reference_refine(impl, wl, first, targets, idx, threads)
    t3 = time.perf_counter()
    times = {"unmix_s": t1 - t0, "filter_s": t2 - t1, "refine_s": t3 - t2, "total_s": t3 - t0}
    # One core: both solves of a seeded sample of the image's pixels (the
    # filter's share of the all-core time is small and is left out here).
    sample = np.sort(np.random.default_rng(17).choice(n, size=min(n, 4096), replace=False))
    s0 = time.perf_counter()
    reference_unmix(impl, wl, sample, 1)
    s1 = time.perf_counter()
    reference_refine(impl, wl, first, targets[:, sample], sample, 1)
    s2 = time.perf_counter()
    times["single_core"] = {"value": len(sample) / (s2 - s0), "unit": UNIT, "cores": 1,
                            "sample": f"both solves of {len(sample)} seeded pixels of the image, one thread",
                            "unmix_s": s1 - s0, "refine_s": s2 - s1}
    return first, final, times, kind


def parity_whole(wl, first_gpu, final_gpu, ref_first, ref_final, threads, sample_seed=0):
    """Parity of one GPU decomposition against the reference's: the first
    pass over the whole image; the refinement over the whole image against
    the reference's own pipeline; and the refinement against the reference's
    refinement from the GPU's first pass (same targets) on a pixel sample."""
    import oracle
    from tests.parity import report
    L, n, w, h = len(wl.layers), wl.pixels, wl.width, wl.height
    out = {"first_pass": report(first_gpu, oracle.pack(ref_first, L, w, h), wl.layers, False)}
    if final_gpu is None:
        return out
    out["pipeline"] = report(final_gpu, oracle.pack(ref_final, L, w, h), wl.layers, True)
    impl, kind = reference_impl()
    gfirst = oracle.unpack(first_gpu, L)
    targets = reference_targets(impl, kind, wl, gfirst, (0, h), threads)
    rng = np.random.default_rng(sample_seed)
    idx = np.sort(rng.choice(n, size=min(PARITY_SAMPLE, n), replace=False))
    x2 = reference_refine(impl, wl, gfirst, targets[:, idx], idx, threads)
    m = len(idx)
    g2 = oracle.pack(oracle.unpack(final_gpu, L)[idx], L, m, 1)
    out["refinement_same_first_pass"] = report(g2, oracle.pack(x2, L, m, 1), wl.layers, True)
    out["refinement_same_first_pass"]["sample"] = f"{m} seeded pixels, filter targets over the whole image"
    return out


def parity_sampled(wl, first_gpu, final_gpu, threads):
    """Parity on a pixel sample (images too large for a whole-image CPU
    run): the reference's first pass of the sample pixels, and its refinement
    of them from the GPU's first pass (filter targets over the whole image)."""
    import oracle
    from tests.parity import report
    L, n, h = len(wl.layers), wl.pixels, wl.height
    impl, kind = reference_impl()
    rng = np.random.default_rng(0)
    idx = np.sort(rng.choice(n, size=min(PARITY_SAMPLE, n), replace=False))
    m = len(idx)
    x1 = reference_unmix(impl, wl, idx, threads)
    gfirst = oracle.unpack(first_gpu, L)
    targets = reference_targets(impl, kind, wl, gfirst, (0, h), threads)
    x2 = reference_refine(impl, wl, gfirst, targets[:, idx], idx, threads)
    g1 = oracle.pack(gfirst[idx], L, m, 1)
    g2 = oracle.pack(oracle.unpack(final_gpu, L)[idx], L, m, 1)
    return {"sample": f"{m} seeded pixels", "first_pass": report(g1, oracle.pack(x1, L, m, 1), wl.layers, False),
            "refinement_same_first_pass": report(g2, oracle.pack(x2, L, m, 1), wl.layers, True)}


def reference_arm(args):
    from unblending_b200 import dist
    rank, world, _ = dist.env()
    if rank != 0:
        return
    if args.workload == "batch64":
        return reference_batch_arm(args)
    wl = load_workload(args.workload, args.width)
    n, w, h = wl.pixels, wl.width, wl.height
    threads = os.cpu_count() or 1
    impl, kind = reference_impl()
    # The first pass that the bands' filters read (untimed; each step's own
    # first-pass solve of its band recomputes the same values).
    first = reference_unmix(impl, wl, np.arange(n), threads)
    bands = [(y, min(h, y + BAND_ROWS)) for y in range(0, h, BAND_ROWS)]
    times, pixels = [], []
    for step in range(args.warmup + args.steps):
        y0, y1 = bands[step % len(bands)]
        idx = np.arange(y0 * w, y1 * w)
        t0 = time.perf_counter()
        reference_unmix(impl, wl, idx, threads)
        targets = reference_targets(impl, kind, wl, first, (y0, y1), threads)
        reference_refine(impl, wl, first, targets, idx, threads)
        dt = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(dt)
            pixels.append(len(idx))
    sec = float(np.mean(times))
    value = float(np.sum(pixels) / np.sum(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, unblending_b200/synthetic.py)",
        "config": config(wl, args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"per step: the full decomposition of one {BAND_ROWS}-row band of the "
                                   f"{w}x{h} image (both solves of its {BAND_ROWS * w} pixels, the CPU guided "
                                   f"filter over the band and 2r rows each side); steps cycle over the bands"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ b200 --
class Decomposition:
    """Device buffers and the two device calls of one decomposition step."""

    def __init__(self, U, torch, wl, stream):
        self.U, self.torch, self.wl, self.stream = U, torch, wl, stream
        L, n = len(wl.layers), wl.pixels
        self.d_img = torch.from_numpy(wl.image.reshape(-1)).cuda()
        self.d_first = torch.empty(4 * L * n, dtype=torch.float64, device="cuda")
        self.d_out = torch.empty_like(self.d_first)
        self.d_status = torch.empty(n, dtype=torch.int32, device="cuda")
        self.c1 = torch.zeros((n, 5), dtype=torch.int32, device="cuda")
        self.c2 = torch.zeros((n, 5), dtype=torch.int32, device="cuda")

    def step(self, solver, counters=False, stats=False):
        U, wl = self.U, self.wl
        s1 = U.unmix_device(wl.width, wl.height, self.d_img.data_ptr(), wl.layers, self.d_first.data_ptr(),
                            solver=solver, d_status=self.d_status.data_ptr(),
                            d_counters=self.c1.data_ptr() if counters else None, stream=self.stream, stats=stats)
        k = U.last_launch_count()
        s2 = U.refine_device(wl.width, wl.height, self.d_img.data_ptr(), wl.layers, self.d_first.data_ptr(),
                             self.d_out.data_ptr(), smooth=True, solver=solver, d_status=self.d_status.data_ptr(),
                             d_counters=self.c2.data_ptr() if counters else None, stream=self.stream, stats=stats)
        return s1, s2, k + U.last_launch_count()

    def timed(self, solver, steps, warmup, flush):
        torch = self.torch
        for _ in range(warmup):
            self.step(solver)
        torch.cuda.synchronize()
        times, launches = [], 0
        stream = torch.cuda.ExternalStream(self.stream)
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _, _, k = self.step(solver)
            e1.record(stream)
            launches += k
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
        return float(np.mean(times)), launches

    def stages(self, solver, reps=3):
        """Device stage times (library CUDA events on the launching stream)
        and evaluation totals, averaged over `reps` steps."""
        rows = []
        for _ in range(reps):
            rows.append(self.step(solver, stats=True)[:2])
        self.torch.cuda.synchronize()
        avg = lambda k, p: float(np.mean([r[p][k] for r in rows]))
        s1, s2 = rows[-1]
        return {"unmix_solve": avg("ms_solve", 0), "unmix_resolve_fp64": avg("ms_resolve", 0),
                "filter": avg("ms_filter", 1), "refine_solve": avg("ms_solve", 1),
                "refine_resolve_fp64": avg("ms_resolve", 1)}, s1, s2

    def host(self, kind):
        t = self.d_first if kind == "first" else self.d_out
        L = len(self.wl.layers)
        return t.cpu().numpy().reshape(L, self.wl.height, self.wl.width, 4)


def train_warm_start(U, torch, wl):
    """The warm-start network for this layer set: 64 seeded 256x256 images of
    the workload's distributions (2^22 pixels), batch 8192, 2048 Adam steps
    (four passes over the pixels) at lr 1e-3. Targets: the default solve's
    first passes of those images."""
    from unblending_b200 import synthetic as syn
    modes = [s.mode for s in wl.layers]
    t0 = time.perf_counter()
    sigma, noise = wl.meta.get("sigma", (20.0, 200.0)), wl.meta.get("noise", 0.0)
    imgs = [syn.generate(256, 256, modes, sigma, seed=10_000 + k, noise=noise, layers=wl.layers) for k in range(64)]
    d = [torch.from_numpy(w.image.reshape(-1)).cuda() for w in imgs]
    t_gen = time.perf_counter() - t0
    t0 = time.perf_counter()
    model = U.mlp_train_device([(x.data_ptr(), 256, 256) for x in d], wl.layers, batch=8192, steps=2048,
                               learning_rate=1e-3, seed=1)
    torch.cuda.synchronize()
    return model, {"images": 64, "pixels": 64 * 256 * 256, "batch": 8192, "steps": 2048, "lr": 1e-3,
                   "final_batch_mse": model.loss, "train_s": time.perf_counter() - t0, "generate_s": t_gen}


def solve_roofline(wl, s1, s2, stages, precision):
    """Roofline of the dominant kernels, the solves: algorithmic flops of the
    evaluations that ran (the library's evaluation totals x the per-evaluation
    count of evaluation_flops) over the solve stages' device time, against the
    nominal CUDA-core peak of that precision."""
    L = len(wl.layers)
    f_val, f_grad = evaluation_flops(L, [s.mode for s in wl.layers])
    if precision == "fp64":
        vals = s1["fp64_values"] + s2["fp64_values"]
        grads = s1["fp64_gradients"] + s2["fp64_gradients"]
        ms = stages["unmix_solve"] + stages["refine_solve"]
        peak, kernel = PEAK_FP64_TFLOPS, f"solve_pixels<double,{L},...>"
        traffic = profile_traffic("solve_pixels_fp64_rgb1024_l5.md")
    else:
        vals = s1["fp32_values"] + s2["fp32_values"]
        grads = s1["fp32_gradients"] + s2["fp32_gradients"]
        ms = stages["unmix_solve"] + stages["refine_solve"]
        peak, kernel = PEAK_FP32_TFLOPS, f"solve_pixels<float,{L},...>"
        traffic = profile_traffic("solve_pixels_fp32_rgb1024_l5.md")
    flops = float((vals - grads) * f_val + grads * f_grad)
    achieved = flops / (ms / 1e3) / 1e12
    return {"bound": precision, "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": traffic * wl.pixels * 2 if traffic is not None else None,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per pixel of the solve launches "
                              "(profiles/), times the two passes' pixels",
            "peak_source": f"nominal {precision.upper()} (148 SMs x lanes x 2 x 1.965 GHz); MEASURED_PEAKS.json has "
                           f"no {precision.upper()} figure",
            "flops_per_step": flops, "evaluations": {"values": int(vals), "gradients": int(grads)},
            "solve_ms": ms, "kernel": kernel}


def config_leg(U, torch, name, stream, flush, steps, warmup, threads, whole_parity):
    """One of the BASELINE's other single-image configurations, timed with
    the default solve, with its parity."""
    wl = load_workload(name)
    D = Decomposition(U, torch, wl, stream)
    so = U.solver_options(radius=refinement_radius(wl))
    ms, _ = D.timed(so, steps, warmup, flush)
    stages, s1, s2 = D.stages(so, reps=1)
    first, final = D.host("first"), D.host("final")
    out = {"workload": workload_label(wl), "value": wl.pixels / (ms / 1e3), "unit": UNIT, "ms_per_step": ms,
           "steps": steps, "warmup": warmup, "stages_ms": stages,
           "misses": {"unmix_failed": s1["failed"], "refine_failed": s2["failed"]},
           "roofline": solve_roofline(wl, s1, s2, stages, "fp64")}
    if threads:
        if whole_parity:
            rf, rr, t, kind = reference_decomposition(wl, threads)
            out["parity"] = parity_whole(wl, first, final, rf, rr, threads)
            out["cpu_baseline"] = {"value": wl.pixels / t["total_s"], "unit": UNIT, "cores": threads, "kind": kind,
                                   "sample": "the whole image, both passes", **t}
        else:
            out["parity"] = parity_sampled(wl, first, final, threads)
    del D
    torch.cuda.empty_cache()
    return out


def batch_leg(U, torch, stream, flush, threads):
    """The BASELINE's uneven batch (64 images, sides 256-2048, 3-6 layers)
    through the batched first pass with the default solve: one warm-up call
    (which also builds and captures the plan), one timed replay, and the
    parity of 8,192 seeded pixels spread over the images against the
    reference's FP64 solver."""
    import oracle
    from tests.parity import report
    wls = batch_workload()
    n = sum(w.pixels for w in wls)
    imgs = [torch.from_numpy(w.image.reshape(-1)).cuda() for w in wls]
    outs = [torch.empty(4 * len(w.layers) * w.pixels, dtype=torch.float64, device="cuda") for w in wls]
    jobs = [dict(width=w.width, height=w.height, d_image=i.data_ptr(), layers=w.layers, d_output=o.data_ptr())
            for w, i, o in zip(wls, imgs, outs)]
    so = U.solver_options()
    st = U.unmix_batch_device(jobs, solver=so, stream=stream, stats=True)
    torch.cuda.synchronize()
    flush.fill_(1.0)
    ext = torch.cuda.ExternalStream(stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    U.unmix_batch_device(jobs, solver=so, stream=stream)
    e1.record(ext)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    out = {"workload": batch_label(wls), "value": n / (ms / 1e3), "unit": UNIT, "ms_per_step": ms, "steps": 1,
           "warmup": 1, "gpu_launches": U.last_launch_count(), "failed": st["failed"]}
    if threads:
        impl, kind = reference_impl()
        rng = np.random.default_rng(23)
        totals, rows = {}, []
        for w, o in zip(wls, outs):
            L = len(w.layers)
            k = max(1, int(round(8192 * w.pixels / n)))
            idx = np.sort(rng.choice(w.pixels, size=min(k, w.pixels), replace=False))
            rx = reference_unmix(impl, w, idx, threads)
            gx = oracle.unpack(o.cpu().numpy().reshape(L, w.height, w.width, 4), L)[idx]
            r = report(oracle.pack(gx, L, len(idx), 1), oracle.pack(rx, L, len(idx), 1), w.layers, False)
            rows.append((len(idx), r))
        m = sum(c for c, _ in rows)
        for key in ("frac_rgba_1e-3", "frac_objective"):
            totals[key] = sum(c * r[key] for c, r in rows) / m
        totals["max_rgba"] = max(r["max_rgba"] for _, r in rows)
        out["parity"] = {"sample": f"{m} seeded pixels over the {len(wls)} images", "kind": kind, **totals}
    del imgs, outs
    torch.cuda.empty_cache()
    return out


def b200_arm(args):
    import torch
    from unblending_b200 import dist
    rank, world, local = dist.env()
    if world > 1:
        import datetime
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    import unblending_b200 as U
    from unblending_b200 import synthetic as syn

    wl = load_workload(args.workload, args.width, rank)
    L, n, w, h = len(wl.layers), wl.pixels, wl.width, wl.height
    radius = refinement_radius(wl)
    stream = torch.cuda.Stream()
    D = Decomposition(U, torch, wl, stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    # UNBLENDING_SOLVER_OPTIONS_INIT with the workload's radius.
    default = U.solver_options(radius=radius, fp64_variant=args.fp64_variant, pixel_order=args.pixel_order)

    sampler = ClockSampler(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    sampler.start()
    wall0 = time.perf_counter()
    ms, launches = D.timed(default, args.steps, args.warmup, flush)
    wall = time.perf_counter() - wall0
    clocks = sampler.stop()
    value = dist.throughput(n, ms, "cuda")
    ms_max = dist.reduce_max(ms, "cuda")

    stages, s1, s2 = D.stages(default)
    D.step(default, counters=True)
    torch.cuda.synchronize()
    c1 = D.c1.cpu().numpy().astype(np.int64)
    c2 = D.c2.cpu().numpy().astype(np.int64)
    first_default, final_default = D.host("first"), D.host("final")

    # ---- FP32 solve (below the parity bar)
    fp32 = None
    if not args.no_fp32:
        so32 = U.solver_options(precision=U.PRECISION_FP32, radius=radius)
        fms, _ = D.timed(so32, args.steps, args.warmup, flush)
        fstages, fs1, fs2 = D.stages(so32)
        fp32 = {"value": dist.throughput(n, fms, "cuda"), "ms_per_step": dist.reduce_max(fms, "cuda"),
                "note": "below the parity bar: the method stops at its own loose tolerance, so FP32 arithmetic "
                        "moves ~1 % of pixels more than 1e-3 from the reference's FP64 result",
                "stages_ms": fstages, "misses": {"unmix": fs1["misses"], "refine": fs2["misses"]},
                "roofline": solve_roofline(wl, fs1, fs2, fstages, "fp32")}
        first_fp32, final_fp32 = D.host("first"), D.host("final")

    # ---- learned warm start on the first pass
    warm = None
    if not args.no_warm:
        model, training = train_warm_start(U, torch, wl)
        wsolver = U.solver_options(warm_start=model, radius=radius)
        wms, _ = D.timed(wsolver, args.steps, args.warmup, flush)
        wstages, ws1, ws2 = D.stages(wsolver)
        D.step(wsolver, counters=True)
        torch.cuda.synchronize()
        wc1 = D.c1.cpu().numpy().astype(np.int64)
        warm = {"value": dist.throughput(n, wms, "cuda"), "ms_per_step": dist.reduce_max(wms, "cuda"),
                "speedup_vs_plain": ms / wms, "training": training,
                "unmix_counters_mean": wc1.mean(0).tolist(),
                "unmix_iteration_histogram": iteration_histogram(wc1), "stages_ms": wstages,
                "misses": {"unmix": ws1["misses"], "unmix_failed": ws1["failed"]}}
        first_warm, final_warm = D.host("first"), D.host("final")

    # ---- e2e through the v1 C ABI: page-locked host buffers (the headline),
    # then plain pageable ones (as the reference CLI's), which the library
    # copies through its own page-locked staging chunks.
    arr = syn.layer_array(wl.layers)
    opts_unmix, opts_refine = U.options(True, False), U.options(True, True)
    dp = ctypes.POINTER(ctypes.c_double)

    def e2e_leg(host_img, host_first, host_out):
        view = U.RgbView(host_img.ctypes.data_as(dp), host_img.size, w, h, 0)

        def e2e_step():
            if wl.radius is None:
                # The v1 entry points (default solver options, the reference's radius).
                rc = U.lib.unblending_unmix(ctypes.byref(view), arr, L, ctypes.byref(opts_unmix),
                                            host_first.ctypes.data_as(dp), host_first.size)
                assert rc == 0, rc
                rc = U.lib.unblending_refine(ctypes.byref(view), arr, L, host_first.ctypes.data_as(dp),
                                             host_first.size, ctypes.byref(opts_refine), host_out.ctypes.data_as(dp),
                                             host_out.size)
            else:
                # The workload names its own radius: the _ex entry points carry it.
                rc = U.lib.unblending_unmix_ex(ctypes.byref(view), arr, L, ctypes.byref(opts_unmix),
                                               ctypes.byref(default), host_first.ctypes.data_as(dp), host_first.size,
                                               None, None, None)
                assert rc == 0, rc
                rc = U.lib.unblending_refine_ex(ctypes.byref(view), arr, L, host_first.ctypes.data_as(dp),
                                                host_first.size, ctypes.byref(opts_refine), ctypes.byref(default),
                                                host_out.ctypes.data_as(dp), host_out.size, None, None, None)
            assert rc == 0, rc

        for _ in range(max(1, args.warmup - 1)):
            e2e_step()
        torch.cuda.synchronize()
        times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            e2e_step()
            times.append(time.perf_counter() - t0)
        return float(np.mean(times)) * 1e3, np.array_equal(host_out, final_default)

    host_img = torch.from_numpy(wl.image.copy()).pin_memory().numpy()
    host_first = torch.empty((L, h, w, 4), dtype=torch.float64).pin_memory().numpy()
    host_out = torch.empty((L, h, w, 4), dtype=torch.float64).pin_memory().numpy()
    e2e_ms, e2e_check = e2e_leg(host_img, host_first, host_out)
    h2d = 2 * host_img.nbytes + host_first.nbytes
    d2h = host_first.nbytes + host_out.nbytes
    del host_img, host_first, host_out
    pageable_ms, pageable_check = e2e_leg(wl.image.copy(), np.empty((L, h, w, 4)), np.empty((L, h, w, 4)))

    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(peaks_path)) if os.path.exists(peaks_path) else {}
    filter_bytes = 4 * (3 + 2 * (L + 3)) * n
    filter_gbs = filter_bytes / (stages["filter"] / 1e3) / 1e9
    hbm_peak = peaks.get("hbm_gbs", 6650.0)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded generator, unblending_b200/synthetic.py)",
        "config": config(wl, world),
        "clocks": clocks,
        "gpu_launches": launches,
        "wall_s_timed_region": wall,
        "stages_ms": stages,
        "misses": {"unmix_failed": s1["failed"], "refine_failed": s2["failed"]},
        "counters_mean": {"unmix": c1.mean(0).tolist(), "refine": c2.mean(0).tolist(),
                          "fields": ["values", "gradients", "iterations", "line_search_trials", "outer"]},
        "iteration_histogram": {"unmix": iteration_histogram(c1), "refine": iteration_histogram(c2)},
        "roofline": solve_roofline(wl, s1, s2, stages, "fp64"),
        "roofline_filter": {"bound": "hbm", "achieved": filter_gbs, "peak": hbm_peak, "unit": "GB/s",
                            "frac": filter_gbs / hbm_peak, "algorithmic_bytes": filter_bytes,
                            "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback",
                            "kernels": "guided filter (7 launches), refinement targets"},
        "fp32": fp32,
        "warm_start": warm,
        "e2e": {"value": dist.throughput(n, e2e_ms, "cuda"), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms,
                "output_equals_device_path": bool(e2e_check)},
        "e2e_pageable": {"value": dist.throughput(n, pageable_ms, "cuda"), "unit": UNIT, "ms_per_step": pageable_ms,
                         "output_equals_device_path": bool(pageable_check),
                         "note": "the same v1 calls with plain (pageable) host buffers, copied through the "
                                 "library's page-locked staging chunks"},
    }
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rf, rr, t, kind = reference_decomposition(wl, threads)
        line["cpu_baseline"] = {"value": n / t["total_s"], "unit": UNIT, "cores": threads, "kind": kind,
                                "sample": "the whole image, both passes (nothing extrapolated)", **t}
        parity = {"default": parity_whole(wl, first_default, final_default, rf, rr, threads)}
        if fp32 is not None:
            parity["fp32"] = parity_whole(wl, first_fp32, final_fp32, rf, rr, threads)
        if warm is not None:
            parity["warm_start"] = parity_whole(wl, first_warm, final_warm, rf, rr, threads)
        line["parity"] = parity
    if rank == 0 and not args.no_configs and world == 1:
        threads = 0 if args.no_cpu_baseline else (os.cpu_count() or 1)
        line["configs"] = {
            "rgb256_l3": config_leg(U, torch, "rgb256_l3", stream.cuda_stream, flush, args.steps, args.warmup,
                                    threads, True),
            "rgb4096_l6": config_leg(U, torch, "rgb4096_l6", stream.cuda_stream, flush, 1, 1, threads, False),
            "batch64": batch_leg(U, torch, stream.cuda_stream, flush, threads),
        }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


# ------------------------------------------------------------- batch64 --
BATCH_COUNT = 64


def batch_workload(rank=0):
    from unblending_b200 import synthetic as syn
    return syn.batch(count=BATCH_COUNT, seed=4 + rank, sides=(256, 2048), shared_layers=True)


def batch_label(wls):
    Ls = sorted({len(w.layers) for w in wls})
    return (f"batch64: {len(wls)} images, sides 256-2048, layers {Ls[0]}-{Ls[-1]} (one layer set per count), "
            f"{sum(w.pixels for w in wls)} pixels, first pass")


def batch_arm(args):
    """The batched first pass (one persistent launch per layer count, one
    captured graph), plain and with a learned start per layer count."""
    import torch
    from unblending_b200 import dist
    rank, world, local = dist.env()
    if world > 1:
        import datetime
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    import unblending_b200 as U
    wls = batch_workload(rank)
    n = sum(w.pixels for w in wls)
    imgs = [torch.from_numpy(w.image.reshape(-1)).cuda() for w in wls]
    outs = [torch.empty(4 * len(w.layers) * w.pixels, dtype=torch.float64, device="cuda") for w in wls]
    sts = [torch.empty(w.pixels, dtype=torch.int32, device="cuda") for w in wls]
    stream = torch.cuda.Stream()
    ext = torch.cuda.ExternalStream(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def jobs(nets):
        return [dict(width=w.width, height=w.height, d_image=i.data_ptr(), layers=w.layers, d_output=o.data_ptr(),
                     d_status=s.data_ptr(), warm_start=nets.get(len(w.layers)) if nets else None)
                for w, i, o, s in zip(wls, imgs, outs, sts)]

    def timed(job_list, solver):
        st = U.unmix_batch_device(job_list, solver=solver, stream=stream.cuda_stream, stats=True)
        for _ in range(max(0, args.warmup - 1)):
            U.unmix_batch_device(job_list, solver=solver, stream=stream.cuda_stream)
        torch.cuda.synchronize()
        times = []
        for _ in range(args.steps):
            with torch.cuda.stream(ext):
                flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            U.unmix_batch_device(job_list, solver=solver, stream=stream.cuda_stream)
            e1.record(ext)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        return float(np.mean(times)), st, U.last_launch_count()

    sampler = ClockSampler(local)
    torch.cuda.synchronize()
    sampler.start()
    default = U.solver_options()
    ms, st, launches = timed(jobs(None), default)
    clocks = sampler.stop()
    fms, fst, _ = timed(jobs(None), U.solver_options(precision=U.PRECISION_FP32))
    nets, training = {}, {}
    for L in sorted({len(w.layers) for w in wls}):
        ref = next(w for w in wls if len(w.layers) == L)
        nets[L], training[L] = train_warm_start(U, torch, ref)
    wms, wst, _ = timed(jobs(nets), default)
    line = {
        "metric": "pixels/sec, batched first pass, warm-start vs plain", "value": dist.throughput(n, ms, "cuda"),
        "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dist.reduce_max(ms, "cuda"), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, unblending_b200/synthetic.py)",
        "config": {"workload": batch_label(wls), "precision": "fp64 (the reference's FP64 method and arithmetic)",
                   "l2": "256 MiB buffer written between steps, outside the timed region"},
        "clocks": clocks, "gpu_launches": launches * args.steps,
        "plain": {"misses": st["misses"], "failed": st["failed"]},
        "fp32": {"value": dist.throughput(n, fms, "cuda"), "ms_per_step": dist.reduce_max(fms, "cuda"),
                 "note": "below the parity bar", "failed": fst["failed"]},
        "warm_start": {"value": dist.throughput(n, wms, "cuda"), "ms_per_step": dist.reduce_max(wms, "cuda"),
                       "speedup_vs_plain": ms / wms, "misses": wst["misses"], "failed": wst["failed"],
                       "training_final_batch_mse": {L: t["final_batch_mse"] for L, t in training.items()}},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def reference_batch_arm(args):
    """The reference's FP64 solver on first-pass solves of pixel samples
    spread over the batch's images; each step solves one sample (its own
    seed) and is timed as it ran."""
    import oracle
    from unblending_b200 import synthetic as syn
    wls = batch_workload()
    n = sum(w.pixels for w in wls)
    threads = os.cpu_count() or 1
    impl, kind = reference_impl()
    per_step = 32768
    times, pixels = [], []
    for step in range(args.warmup + args.steps):
        rng = np.random.default_rng(step)
        per = [max(1, int(round(per_step * w.pixels / n))) for w in wls]
        samples = [np.sort(rng.choice(w.pixels, size=min(k, w.pixels), replace=False)) for w, k in zip(wls, per)]
        t0 = time.perf_counter()
        for w, idx in zip(wls, samples):
            L = len(w.layers)
            impl.solve(syn.layer_array(w.layers), oracle.problem(L, False, True), oracle.options(),
                       w.image.reshape(-1, 3)[idx], np.tile(oracle.initial_first(w.layers, True), (len(idx), 1)),
                       threads=threads)
        dt = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(dt)
            pixels.append(sum(len(x) for x in samples))
    value = float(np.sum(pixels) / np.sum(times))
    line = {
        "impl": "reference", "metric": "pixels/sec, batched first pass, warm-start vs plain", "value": value,
        "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": float(np.mean(times)) * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, unblending_b200/synthetic.py)",
        "config": {"workload": batch_label(wls), "precision": "fp64 (the reference's FP64 method and arithmetic)",
                   "l2": "256 MiB buffer written between steps, outside the timed region"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"per step: first-pass solves of ~{per_step} seeded pixels spread over the "
                                   f"images in proportion to their size"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    elif args.workload == "batch64":
        batch_arm(args)
    else:
        b200_arm(args)


if __name__ == "__main__":
    main()
