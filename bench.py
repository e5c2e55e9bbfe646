"""Benchmark: full decomposition (first pass + matte refinement) throughput.

Workload (one step): the 1024x1024, 5-layer synthetic image (normal,
multiply, screen, overlay, color-dodge; alpha blobs 20-200 px; seed 2),
colour unmixing then matte refinement with an opaque, smoothed background
(the reference CLI's configuration, unblending-cli/main.cpp:58-66) and the
reference's refinement radius 60*min(w,h)/1000 = 61.

  value : pixels/s with the image resident in HBM (device entry points),
          per-step device time from CUDA events on the library's stream;
          a 256 MiB buffer is written between steps (L2 flush, untimed).
  e2e   : the same through the C ABI calls unblending_unmix +
          unblending_refine with pinned host buffers (uploads, the first
          pass's round trip through the host, and downloads are timed).

Multi-GPU: one process per GPU, each decomposing its own image (weak
scaling, no collective on the data path); time = max over ranks.

`--impl reference` times the reference's own CPU implementation
(oracle/_ref, the reference's FP64 solver and CPU guided filter compiled
from its sources; else the CPU oracle restatement) on all host cores.
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


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    p.add_argument("--width", type=int, default=1024)
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


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
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
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
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace('.', '', 1).isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace('.', '', 1).isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows if len(r) >= 9 for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------ flop count --
def evaluation_flops(L: int, modes: list[int]) -> tuple[float, float]:
    """FP32 flops of one value evaluation and of one value+gradient evaluation
    of the per-pixel objective, counted from the solver's arithmetic per
    pixel (all four lanes of a quad): composite 3 channels x (L-1) layers,
    Gaussian prior 3x3 per layer, AL terms; the gradient adds the (P+P^T)
    rows and the reverse sweep. add/mul = 1, fma = 2, div/sqrt = 1."""
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


# ------------------------------------------------------------ reference --
def cpu_reference(wl, first_gpu, final_gpu, threads, sample_idx):
    """The reference's CPU implementation on this host: its FP64 solver
    (general::Optimizer<double>) for both passes over a pixel sample, and its
    CPU guided filter (general::StreamingFilterCPU) over the whole image.
    Returns (seconds per full image extrapolated, details, parity dict)."""
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
    # Filter over the whole image from the GPU first pass (same input for both).
    rgb_planar = wl.image.reshape(n, 3).T.copy()
    first_x = oracle.unpack(first_gpu, L)
    first_planar = first_x.T.copy()
    t0 = time.perf_counter()
    radius = syn.reference_radius(w, h)
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
    per_px = (t_unmix + t_refine) / len(sample_idx)
    seconds = t_filter + per_px * n
    # Parity of the GPU outputs on the sample pixels.
    gpu1 = oracle.unpack(first_gpu, L)[sample_idx]
    gpu2 = oracle.unpack(final_gpu, L)[sample_idx]
    par1 = report(oracle.pack(gpu1, L, len(sample_idx), 1), oracle.pack(x1, L, len(sample_idx), 1), wl.layers, False)
    par2 = report(oracle.pack(gpu2, L, len(sample_idx), 1), oracle.pack(x2, L, len(sample_idx), 1), wl.layers, True)
    details = {"t_unmix_sample_s": t_unmix, "t_refine_sample_s": t_refine, "t_filter_full_s": t_filter}
    return seconds, kind, details, {"first_pass": par1, "refinement": par2}


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from unblending_b200 import synthetic as syn
    import oracle
    wl = syn.workload(WORKLOAD, args.width, args.width)
    L, n = len(wl.layers), wl.pixels
    threads = os.cpu_count() or 1
    impl = oracle.ref_lib()
    kind = "reference" if impl is not None else "port"
    impl = impl or oracle.lib()
    rng = np.random.default_rng(0)
    sample = np.sort(rng.choice(n, size=SAMPLE, replace=False))
    layers = syn.layer_array(wl.layers)
    # The reference's first pass over the whole image (needed for its filter) is
    # too slow for every step; steps time: full filter + solves on the sample.
    x_first_sample, _ = impl.solve(layers, oracle.problem(L, False, True), oracle.options(),
                                   wl.image.reshape(n, 3)[sample],
                                   np.tile(oracle.initial_first(wl.layers, True), (SAMPLE, 1)), threads=threads)
    first_full = np.tile(oracle.initial_first(wl.layers, True), (n, 1))
    first_full[sample] = x_first_sample
    first_packed = oracle.pack(first_full, L, wl.width, wl.height)
    times = []
    for step in range(args.warmup + args.steps):
        seconds, kind, details, _ = cpu_reference(wl, first_packed, first_packed, threads, sample)
        if step >= args.warmup:
            times.append(seconds)
    sec = float(np.mean(times))
    value = n / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, unblending_b200/synthetic.py)",
        "config": {"workload": f"{WORKLOAD} {args.width}x{args.width} L=5 unmix+refine(smooth, r=ref formula)",
                   "warm_start": False},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"per step: CPU guided filter over the full image + both solves on {SAMPLE} "
                                   f"seeded pixels, extrapolated to {n} pixels"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ b200 --
def b200_arm(args):
    import torch
    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    import unblending_b200 as U
    from unblending_b200 import synthetic as syn

    wl = syn.workload(WORKLOAD, args.width, args.width, seed=2 + rank)
    L, n, w, h = len(wl.layers), wl.pixels, wl.width, wl.height
    precision = U.PRECISION_FP64 if args.precision == "fp64" else U.PRECISION_FP32
    so = U.solver_options(precision=precision)
    stream = torch.cuda.Stream()
    d_img = torch.from_numpy(wl.image.reshape(-1)).cuda()
    d_first = torch.empty(4 * L * n, dtype=torch.float64, device="cuda")
    d_out = torch.empty_like(d_first)
    d_status = torch.empty(n, dtype=torch.int32, device="cuda")
    d_counters1 = torch.zeros((n, 5), dtype=torch.int32, device="cuda")
    d_counters2 = torch.zeros((n, 5), dtype=torch.int32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    sp = stream.cuda_stream

    def step(counters=False, st=False):
        s1 = U.unmix_device(w, h, d_img.data_ptr(), wl.layers, d_first.data_ptr(), solver=so,
                            d_status=d_status.data_ptr(),
                            d_counters=d_counters1.data_ptr() if counters else None, stream=sp, stats=st)
        launches = U.last_launch_count()
        s2 = U.refine_device(w, h, d_img.data_ptr(), wl.layers, d_first.data_ptr(), d_out.data_ptr(), smooth=True,
                             solver=so, d_status=d_status.data_ptr(),
                             d_counters=d_counters2.data_ptr() if counters else None, stream=sp, stats=st)
        return s1, s2, launches + U.last_launch_count()

    # Warm-up (also records stage timings and counters once).
    s1 = s2 = None
    for i in range(args.warmup):
        s1, s2, _ = step(counters=(i == 0), st=True)
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    sampler.start()
    times, launches = [], 0
    wall0 = time.perf_counter()
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, _, k = step()
        e1.record(stream)
        launches += k
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    clocks = sampler.stop()
    ms = float(np.mean(times))
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    value = n * world / (ms / 1e3)

    # Per-kernel breakdown of one step (device events inside the library).
    s1, s2, _ = step(counters=True, st=True)
    torch.cuda.synchronize()
    c1 = d_counters1.cpu().numpy().astype(np.int64)
    c2 = d_counters2.cpu().numpy().astype(np.int64)

    # ---- e2e through the C ABI with pinned host buffers
    host_img = torch.from_numpy(wl.image.copy()).pin_memory().numpy()
    host_first = torch.empty((L, h, w, 4), dtype=torch.float64).pin_memory().numpy()
    host_out = torch.empty((L, h, w, 4), dtype=torch.float64).pin_memory().numpy()
    arr = syn.layer_array(wl.layers)
    view = U.RgbView(host_img.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), host_img.size, w, h, 0)
    opts_unmix = U.options(True, False)
    opts_refine = U.options(True, True)
    dp = ctypes.POINTER(ctypes.c_double)

    def e2e_step():
        rc = U.lib.unblending_unmix(ctypes.byref(view), arr, L, ctypes.byref(opts_unmix),
                                    host_first.ctypes.data_as(dp), host_first.size)
        assert rc == 0, rc
        rc = U.lib.unblending_refine(ctypes.byref(view), arr, L, host_first.ctypes.data_as(dp), host_first.size,
                                     ctypes.byref(opts_refine), host_out.ctypes.data_as(dp), host_out.size)
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
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())
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
    filter_bytes = 4 * (3 + 2 * (L + 3)) * n     # algorithmic bytes of the filter (f32 equivalent, by definition)
    filter_gbs = filter_bytes / (s2["ms_filter"] / 1e3) / 1e9
    hbm_peak = peaks.get("hbm_gbs", 6650.0)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if precision == U.PRECISION_FP32 else "f64",
        "data": "synthetic (seeded generator, unblending_b200/synthetic.py)",
        "config": {"workload": f"{WORKLOAD} {w}x{h} L=5 unmix+refine(opaque, smooth bg, r={s2['radius']})",
                   "precision": args.precision, "warm_start": False, "starts": 1,
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
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": PEAK_FP32_TFLOPS, "unit": "TFLOP/s",
                     "frac": achieved / PEAK_FP32_TFLOPS, "traffic": None,
                     "peak_source": "nominal FP32 (148 SMs x 128 lanes x 2 x 1.965 GHz); MEASURED_PEAKS.json has no FP32 figure",
                     "flops_per_step": flops1 + flops2},
        "roofline_filter": {"bound": "hbm", "achieved": filter_gbs, "peak": hbm_peak, "unit": "GB/s",
                            "frac": filter_gbs / hbm_peak, "algorithmic_bytes": filter_bytes,
                            "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback"},
        "e2e": {"value": n * world / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms},
    }
    if rank == 0 and not args.no_cpu_baseline:
        rng = np.random.default_rng(0)
        sample = np.sort(rng.choice(n, size=SAMPLE, replace=False))
        first = d_first.cpu().numpy().reshape(L, h, w, 4)
        final = d_out.cpu().numpy().reshape(L, h, w, 4)
        threads = os.cpu_count() or 1
        sec, kind, details, parity = cpu_reference(wl, first, final, threads, sample)
        line["cpu_baseline"] = {"value": n / sec, "unit": UNIT, "cores": threads, "kind": kind,
                                "sample": f"CPU guided filter over the full image + both solves on {SAMPLE} seeded "
                                          f"pixels, extrapolated to {n} pixels", **details}
        line["parity_sample"] = parity
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    else:
        b200_arm(args)


if __name__ == "__main__":
    main()
