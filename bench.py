"""Benchmark: full decomposition (first pass + matte refinement) throughput.

Workload (one step): the 1024x1024, 5-layer synthetic image (normal,
multiply, screen, overlay, color-dodge; alpha blobs 20-200 px; seed 2 + rank),
colour unmixing then matte refinement with an opaque, smoothed background
(the reference CLI's configuration, unblending-cli/main.cpp:58-66) and the
reference's refinement radius 60*min(w,h)/1000 = 61.

  value      : pixels/s of the plain (reference-start) FP32 solve with its
               FP64 check and FP64 re-solve of misses, image resident in HBM,
               per-step device time from CUDA events; a 256 MiB buffer is
               written between steps (L2 flush, untimed).
  warm_start : the same with the learned start on the first pass (network
               trained beforehand on 64 seeded 256x256 images of the same layer
               set, 2^22 pixels, batch 8192, Adam lr 1e-3).
  fp64       : the same with the FP64 solve (replays the reference's FP64
               solver; pixels whose outer steps stop moving them end early,
               with results equal to the full schedule).
  e2e        : the plain configuration through the C ABI calls
               unblending_unmix + unblending_refine with pinned host buffers.

Other workloads (`--workload`, extra measurements beside the default line):
  rgb4096_l6 : the same step on the 4096x4096 six-layer image (soft-light on
               top, blobs 50-800 px, N(0, 0.01) colour noise, filter r = 8).
  batch64    : the batched first pass over 64 images (sides 256-2048, 3-6
               layers, one shared layer set per layer count), plain and with
               a learned start per layer count.

Multi-GPU: one process per GPU, each decomposing its own image (weak
scaling, no collective on the data path); time = max over ranks.

`--impl reference` times the reference's own CPU implementation
(oracle/_ref: the reference's FP64 solver and CPU guided filter compiled from
its sources; else the CPU oracle restatement) on all host cores.
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
PEAK_FP32_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12   # nominal: SMs x FP32 lanes x FMA x max clock
SAMPLE = 4096                                        # pixels in the CPU baseline / parity sample
# DRAM bytes (read + write) per pixel of one FP32 first-pass solve launch on this
# workload, from an ncu capture of that kernel (dram__bytes x duration): the
# image read and the packed-RGBA output write, no re-reads.
SOLVE_TRAFFIC_BYTES_PER_PIXEL = 145.0


def load_workload(args, rank=0):
    """The single-image workload of this run (its own seed + rank)."""
    from unblending_b200 import synthetic as syn
    seed = syn.WORKLOADS[args.workload]["seed"] + rank
    return syn.workload(args.workload, args.width, args.width, seed=seed)


def refinement_radius(wl):
    from unblending_b200 import synthetic as syn
    return wl.radius if wl.radius is not None else syn.reference_radius(wl.width, wl.height)


def workload_label(wl):
    return (f"{wl.name} {wl.width}x{wl.height} L={len(wl.layers)} unmix+refine(opaque, smooth bg, "
            f"r={refinement_radius(wl)})")


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
    p.add_argument("--no-fp64", action="store_true")
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
    """FP32 flops of one value evaluation and of one value+gradient
    evaluation of the per-pixel objective (all four lanes of a quad):
    composite 3 channels x (L-1) layers, 3x3 Gaussian prior per layer, AL
    rows; the gradient adds the (P+P^T) rows and the reverse sweep.
    add/mul = 1, fma = 2, reciprocal/sqrt = 1."""
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
    A pixel that the FP32 solve missed carries the counts of its FP64
    re-solve, the solve that produced its output."""
    it, outer = c[:, 2], c[:, 4]
    bins = ITERATION_EDGES + [int(max(it.max(), ITERATION_EDGES[-1])) + 1]
    counts, _ = np.histogram(it, bins=bins)
    q = np.quantile(it, [0.5, 0.9, 0.99, 0.999])
    return {"iterations": {"edges": ITERATION_EDGES, "counts": counts.tolist(),
                           "p50": float(q[0]), "p90": float(q[1]), "p99": float(q[2]), "p99.9": float(q[3]),
                           "max": int(it.max()), "mean": float(it.mean())},
            "outer_steps": {str(k): int(v) for k, v in enumerate(np.bincount(outer)) if v}}


# ------------------------------------------------------------ reference --
def cpu_reference(wl, first_gpu, finals, threads, sample_idx):
    """The reference's CPU implementation on this host: its FP64 solver
    (general::Optimizer<double>) for both passes over a pixel sample, and its
    CPU guided filter (general::StreamingFilterCPU) over the whole image.
    Returns (seconds per full image, kind, details, parity of each GPU output
    in `finals` (name -> (first, final)) on the sample)."""
    import oracle
    from unblending_b200 import synthetic as syn
    from tests.parity import report
    impl = oracle.ref_lib()
    kind = "reference" if impl is not None else "port"
    impl = impl or oracle.lib()
    L, n, w, h = len(wl.layers), wl.pixels, wl.width, wl.height
    layers = syn.layer_array(wl.layers)
    target = wl.image.reshape(n, 3)[sample_idx]
    init = np.tile(oracle.initial_first(wl.layers, True), (len(sample_idx), 1))
    t0 = time.perf_counter()
    x1, _ = impl.solve(layers, oracle.problem(L, False, True), oracle.options(), target, init, threads=threads)
    t_unmix = time.perf_counter() - t0
    rgb_planar = wl.image.reshape(n, 3).T.copy()
    first_x = oracle.unpack(first_gpu, L)
    first_planar = first_x.T.copy()
    radius = refinement_radius(wl)
    t0 = time.perf_counter()
    if kind == "reference":
        targets = np.zeros((L + 3, n))
        status = np.zeros(n, np.int32)
        impl.dll.ref_refine_targets(rgb_planar.ctypes.data_as(oracle._dp), first_planar.ctypes.data_as(oracle._dp),
                                    layers, L, w, h, 1, 1, radius, threads, targets.ctypes.data_as(oracle._dp),
                                    status.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    else:
        targets, status = oracle.refine_targets(rgb_planar, first_planar, layers, L, w, h, True, True, radius)
    t_filter = time.perf_counter() - t0
    alpha = targets[:L].T[sample_idx].copy()
    bg = targets[L:L + 3].T[sample_idx].copy()
    init2 = first_x[sample_idx].copy()
    init2[:, :L] = alpha
    init2[:, 0] = 1.0
    init2[:, L:L + 3] = bg
    t0 = time.perf_counter()
    x2, _ = impl.solve(layers, oracle.problem(L, True, True, True), oracle.options(), target, init2, alpha=alpha,
                       bg=bg, threads=threads)
    t_refine = time.perf_counter() - t0
    x2[:, :L] = alpha
    x2[:, L:L + 3] = bg
    seconds = t_filter + (t_unmix + t_refine) / len(sample_idx) * n
    m = len(sample_idx)
    ref1 = oracle.pack(x1, L, m, 1)
    ref2 = oracle.pack(x2, L, m, 1)
    parity = {}
    for name, (first, final) in finals.items():
        g1 = oracle.pack(oracle.unpack(first, L)[sample_idx], L, m, 1)
        g2 = oracle.pack(oracle.unpack(final, L)[sample_idx], L, m, 1)
        parity[name] = {"first_pass": report(g1, ref1, wl.layers, False),
                        "refinement_same_first_pass": report(g2, ref2, wl.layers, True) if name == "plain" else None}
    details = {"t_unmix_sample_s": t_unmix, "t_refine_sample_s": t_refine, "t_filter_full_s": t_filter}
    # The same on one host core: both solves over the first 512 sample pixels,
    # the filter over the whole image.
    k = min(512, m)
    t0 = time.perf_counter()
    impl.solve(layers, oracle.problem(L, False, True), oracle.options(), target[:k], init[:k], threads=1)
    t1_unmix = time.perf_counter() - t0
    t0 = time.perf_counter()
    if kind == "reference":
        impl.dll.ref_refine_targets(rgb_planar.ctypes.data_as(oracle._dp), first_planar.ctypes.data_as(oracle._dp),
                                    layers, L, w, h, 1, 1, radius, 1, targets.ctypes.data_as(oracle._dp),
                                    status.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        t1_filter = time.perf_counter() - t0
    else:
        t1_filter = t_filter
    t0 = time.perf_counter()
    impl.solve(layers, oracle.problem(L, True, True, True), oracle.options(), target[:k], init2[:k], alpha=alpha[:k],
               bg=bg[:k], threads=1)
    t1_refine = time.perf_counter() - t0
    details["single_core"] = {"value": n / (t1_filter + (t1_unmix + t1_refine) / k * n), "cores": 1,
                              "sample": f"both solves on {k} sample pixels, the filter over the full image"}
    return seconds, kind, details, parity


def reference_arm(args):
    from unblending_b200 import dist, synthetic as syn
    import oracle
    rank, world, _ = dist.env()
    if rank != 0:
        return
    if args.workload == "batch64":
        return reference_batch_arm(args)
    wl = load_workload(args)
    L, n = len(wl.layers), wl.pixels
    threads = os.cpu_count() or 1
    impl = oracle.ref_lib()
    kind = "reference" if impl is not None else "port"
    impl = impl or oracle.lib()
    rng = np.random.default_rng(0)
    sample = np.sort(rng.choice(n, size=SAMPLE, replace=False))
    layers = syn.layer_array(wl.layers)
    x_first_sample, _ = impl.solve(layers, oracle.problem(L, False, True), oracle.options(),
                                   wl.image.reshape(n, 3)[sample],
                                   np.tile(oracle.initial_first(wl.layers, True), (SAMPLE, 1)), threads=threads)
    first_full = np.tile(oracle.initial_first(wl.layers, True), (n, 1))
    first_full[sample] = x_first_sample
    first_packed = oracle.pack(first_full, L, wl.width, wl.height)
    times = []
    for step in range(args.warmup + args.steps):
        seconds, kind, details, _ = cpu_reference(wl, first_packed, {}, threads, sample)
        if step >= args.warmup:
            times.append(seconds)
    sec = float(np.mean(times))
    value = n / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, unblending_b200/synthetic.py)",
        "config": {"workload": workload_label(wl), "warm_start": False},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"per step: CPU guided filter over the full image + both solves on {SAMPLE} "
                                   f"seeded pixels, extrapolated to {n} pixels"},
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

    def host(self, kind):
        t = self.d_first if kind == "first" else self.d_out
        L = len(self.wl.layers)
        return t.cpu().numpy().reshape(L, self.wl.height, self.wl.width, 4)


def train_warm_start(U, torch, wl):
    """The warm-start network for this layer set: 64 seeded 256x256 images of
    the workload's distributions (2^22 pixels), batch 8192, 2048 Adam steps
    (four passes over the pixels) at lr 1e-3."""
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

    wl = load_workload(args, rank)
    L, n, w, h = len(wl.layers), wl.pixels, wl.width, wl.height
    radius = refinement_radius(wl)
    stream = torch.cuda.Stream()
    D = Decomposition(U, torch, wl, stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    plain = U.solver_options(precision=U.PRECISION_FP32, radius=radius)

    sampler = ClockSampler(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    sampler.start()
    wall0 = time.perf_counter()
    ms, launches = D.timed(plain, args.steps, args.warmup, flush)
    wall = time.perf_counter() - wall0
    clocks = sampler.stop()
    value = dist.throughput(n, ms, "cuda")
    ms_max = dist.reduce_max(ms, "cuda")

    # Stage breakdown and work counters of one step.
    s1, s2, _ = D.step(plain, counters=True, stats=True)
    torch.cuda.synchronize()
    c1 = D.c1.cpu().numpy().astype(np.int64)
    c2 = D.c2.cpu().numpy().astype(np.int64)
    first_plain, final_plain = D.host("first"), D.host("final")

    # ---- learned warm start on the first pass
    warm = None
    if not args.no_warm:
        model, training = train_warm_start(U, torch, wl)
        wsolver = U.solver_options(precision=U.PRECISION_FP32, warm_start=model, radius=radius)
        wms, _ = D.timed(wsolver, args.steps, args.warmup, flush)
        ws1, ws2, _ = D.step(wsolver, counters=True, stats=True)
        torch.cuda.synchronize()
        wc1 = D.c1.cpu().numpy().astype(np.int64)
        warm = {"value": dist.throughput(n, wms, "cuda"), "ms_per_step": dist.reduce_max(wms, "cuda"),
                "speedup_vs_plain": ms / wms, "training": training,
                "unmix_counters_mean": wc1.mean(0).tolist(),
                "unmix_iteration_histogram": iteration_histogram(wc1),
                "stages_ms": {"unmix_solve": ws1["ms_solve"], "unmix_resolve_fp64": ws1["ms_resolve"],
                              "filter": ws2["ms_filter"], "refine_solve": ws2["ms_solve"],
                              "refine_resolve_fp64": ws2["ms_resolve"]},
                "misses": {"unmix": ws1["misses"], "unmix_failed": ws1["failed"]}}
        first_warm, final_warm = D.host("first"), D.host("final")

    # ---- FP64 solve (replays the reference's FP64 solver)
    fp64 = None
    if not args.no_fp64:
        fsolver = U.solver_options(precision=U.PRECISION_FP64, radius=radius)
        fms, _ = D.timed(fsolver, max(2, args.steps // 2), 1, flush)
        fp64 = {"value": dist.throughput(n, fms, "cuda"), "ms_per_step": dist.reduce_max(fms, "cuda")}
        first_fp64, final_fp64 = D.host("first"), D.host("final")

    # ---- e2e through the C ABI with pinned host buffers
    host_img = torch.from_numpy(wl.image.copy()).pin_memory().numpy()
    host_first = torch.empty((L, h, w, 4), dtype=torch.float64).pin_memory().numpy()
    host_out = torch.empty((L, h, w, 4), dtype=torch.float64).pin_memory().numpy()
    arr = syn.layer_array(wl.layers)
    view = U.RgbView(host_img.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), host_img.size, w, h, 0)
    opts_unmix, opts_refine = U.options(True, False), U.options(True, True)
    dp = ctypes.POINTER(ctypes.c_double)

    def e2e_step():
        if wl.radius is None:
            # The v1 entry points (their radius is the reference's formula).
            rc = U.lib.unblending_unmix(ctypes.byref(view), arr, L, ctypes.byref(opts_unmix),
                                        host_first.ctypes.data_as(dp), host_first.size)
            assert rc == 0, rc
            rc = U.lib.unblending_refine(ctypes.byref(view), arr, L, host_first.ctypes.data_as(dp), host_first.size,
                                         ctypes.byref(opts_refine), host_out.ctypes.data_as(dp), host_out.size)
        else:
            # The workload names its own radius: the _ex entry points carry it.
            rc = U.lib.unblending_unmix_ex(ctypes.byref(view), arr, L, ctypes.byref(opts_unmix), ctypes.byref(plain),
                                           host_first.ctypes.data_as(dp), host_first.size, None, None, None)
            assert rc == 0, rc
            rc = U.lib.unblending_refine_ex(ctypes.byref(view), arr, L, host_first.ctypes.data_as(dp),
                                            host_first.size, ctypes.byref(opts_refine), ctypes.byref(plain),
                                            host_out.ctypes.data_as(dp), host_out.size, None, None, None)
        assert rc == 0, rc

    for _ in range(max(1, args.warmup - 1)):
        e2e_step()
    torch.cuda.synchronize()
    e2e_times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        e2e_step()
        e2e_times.append(time.perf_counter() - t0)
    e2e_ms = float(np.mean(e2e_times)) * 1e3
    h2d = 2 * host_img.nbytes + host_first.nbytes
    d2h = host_first.nbytes + host_out.nbytes

    # ---- roofline of the dominant kernel (the FP32 solve)
    modes = [s.mode for s in wl.layers]
    f_val, f_grad = evaluation_flops(L, modes)
    flops1 = float((c1[:, 0] - c1[:, 1]).sum() * f_val + c1[:, 1].sum() * f_grad)
    flops2 = float((c2[:, 0] - c2[:, 1]).sum() * f_val + c2[:, 1].sum() * f_grad)
    solve_ms = s1["ms_solve"] + s2["ms_solve"]
    achieved = (flops1 + flops2) / (solve_ms / 1e3) / 1e12
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(peaks_path)) if os.path.exists(peaks_path) else {}
    filter_bytes = 4 * (3 + 2 * (L + 3)) * n
    filter_gbs = filter_bytes / (s2["ms_filter"] / 1e3) / 1e9
    hbm_peak = peaks.get("hbm_gbs", 6650.0)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded generator, unblending_b200/synthetic.py)",
        "config": {"workload": workload_label(wl),
                   "precision": "fp32 solve + fp64 check/re-solve of misses", "warm_start": False, "starts": 1,
                   "l2": "256 MiB buffer written between steps, outside the timed region",
                   "parallelism": f"{world} independent images (one per GPU)"},
        "clocks": clocks,
        "gpu_launches": launches,
        "wall_s_timed_region": wall,
        "stages_ms": {"unmix_solve": s1["ms_solve"], "unmix_resolve_fp64": s1["ms_resolve"],
                      "filter": s2["ms_filter"], "refine_solve": s2["ms_solve"], "refine_resolve_fp64": s2["ms_resolve"]},
        "misses": {"unmix": s1["misses"], "unmix_failed": s1["failed"], "refine": s2["misses"],
                   "refine_failed": s2["failed"]},
        "counters_mean": {"unmix": c1.mean(0).tolist(), "refine": c2.mean(0).tolist(),
                          "fields": ["values", "gradients", "iterations", "line_search_trials", "outer"]},
        "iteration_histogram": {"unmix": iteration_histogram(c1), "refine": iteration_histogram(c2)},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": PEAK_FP32_TFLOPS, "unit": "TFLOP/s",
                     "frac": achieved / PEAK_FP32_TFLOPS, "traffic": SOLVE_TRAFFIC_BYTES_PER_PIXEL * n,
                     "peak_source": "nominal FP32 (148 SMs x 128 lanes x 2 x 1.965 GHz); MEASURED_PEAKS.json has no FP32 figure",
                     "flops_per_step": flops1 + flops2, "kernel": "solve_pixels<float,5,...>"},
        "roofline_filter": {"bound": "hbm", "achieved": filter_gbs, "peak": hbm_peak, "unit": "GB/s",
                            "frac": filter_gbs / hbm_peak, "algorithmic_bytes": filter_bytes,
                            "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback"},
        "warm_start": warm,
        "fp64": fp64,
        "e2e": {"value": dist.throughput(n, e2e_ms, "cuda"), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms},
    }
    if rank == 0 and not args.no_cpu_baseline:
        rng = np.random.default_rng(0)
        sample = np.sort(rng.choice(n, size=SAMPLE, replace=False))
        finals = {"plain": (first_plain, final_plain)}
        if warm is not None:
            finals["warm_start"] = (first_warm, final_warm)
        if fp64 is not None:
            finals["fp64"] = (first_fp64, final_fp64)
        threads = os.cpu_count() or 1
        sec, kind, details, parity = cpu_reference(wl, first_plain, finals, threads, sample)
        line["cpu_baseline"] = {"value": n / sec, "unit": UNIT, "cores": threads, "kind": kind,
                                "sample": f"CPU guided filter over the full image + both solves on {SAMPLE} seeded "
                                          f"pixels, extrapolated to {n} pixels", **details}
        line["parity_sample"] = parity
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

    def timed(job_list):
        st = U.unmix_batch_device(job_list, stream=stream.cuda_stream, stats=True)   # plan, autotune, graph
        for _ in range(max(0, args.warmup - 1)):
            U.unmix_batch_device(job_list, stream=stream.cuda_stream)
        torch.cuda.synchronize()
        times = []
        for _ in range(args.steps):
            with torch.cuda.stream(ext):
                flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            U.unmix_batch_device(job_list, stream=stream.cuda_stream)
            e1.record(ext)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        return float(np.mean(times)), st, U.last_launch_count()

    sampler = ClockSampler(local)
    torch.cuda.synchronize()
    sampler.start()
    ms, st, launches = timed(jobs(None))
    clocks = sampler.stop()
    nets, training = {}, {}
    for L in sorted({len(w.layers) for w in wls}):
        ref = next(w for w in wls if len(w.layers) == L)
        nets[L], training[L] = train_warm_start(U, torch, ref)
    wms, wst, _ = timed(jobs(nets))
    line = {
        "metric": "pixels/sec, batched first pass, warm-start vs plain", "value": dist.throughput(n, ms, "cuda"),
        "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dist.reduce_max(ms, "cuda"), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, unblending_b200/synthetic.py)",
        "config": {"workload": batch_label(wls), "precision": "fp32 solve + fp64 check/re-solve of misses",
                   "l2": "256 MiB buffer written between steps, outside the timed region"},
        "clocks": clocks, "gpu_launches": launches * args.steps,
        "plain": {"misses": st["misses"], "failed": st["failed"]},
        "warm_start": {"value": dist.throughput(n, wms, "cuda"), "ms_per_step": dist.reduce_max(wms, "cuda"),
                       "speedup_vs_plain": ms / wms, "misses": wst["misses"], "failed": wst["failed"],
                       "training_final_batch_mse": {L: t["final_batch_mse"] for L, t in training.items()}},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def reference_batch_arm(args):
    """The reference's FP64 solver on a 4096-pixel sample spread over the
    batch's images (first pass), extrapolated to all of its pixels."""
    import oracle
    from unblending_b200 import synthetic as syn
    wls = batch_workload()
    n = sum(w.pixels for w in wls)
    threads = os.cpu_count() or 1
    impl = oracle.ref_lib()
    kind = "reference" if impl is not None else "port"
    impl = impl or oracle.lib()
    rng = np.random.default_rng(0)
    per = [max(1, int(round(SAMPLE * w.pixels / n))) for w in wls]
    samples = [np.sort(rng.choice(w.pixels, size=min(k, w.pixels), replace=False)) for w, k in zip(wls, per)]
    times = []
    for step in range(args.warmup + args.steps):
        t, m = 0.0, 0
        for w, idx in zip(wls, samples):
            L = len(w.layers)
            t0 = time.perf_counter()
            impl.solve(syn.layer_array(w.layers), oracle.problem(L, False, True), oracle.options(),
                       w.image.reshape(-1, 3)[idx], np.tile(oracle.initial_first(w.layers, True), (len(idx), 1)),
                       threads=threads)
            t += (time.perf_counter() - t0) * w.pixels / len(idx)
        if step >= args.warmup:
            times.append(t)
    sec = float(np.mean(times))
    value = n / sec
    line = {
        "impl": "reference", "metric": "pixels/sec, batched first pass, warm-start vs plain", "value": value,
        "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, unblending_b200/synthetic.py)", "config": {"workload": batch_label(wls)},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"per step: first-pass solves of {sum(len(x) for x in samples)} seeded pixels "
                                   f"spread over the images, extrapolated to {n} pixels"},
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
