#!/usr/bin/env python
"""Benchmark of the neighbourhood-filter hot path on B200.

Workload (the headline configuration): ipf::gaussianBlur, sigma = 2.0 (13 taps
by the reference's size rule), BorderMode::Reflect101, on 3840x2160x3 uint8
images with i.i.d. uniform 0-255 pixels from a seed.  A step filters
`images_per_step` images held resident in HBM, rotating over enough
source/destination buffer pairs that the working set exceeds the 126 MB L2.
Each step is one CUDA-graph replay of that many launches; the timed region is
bracketed by a barrier and cudaDeviceSynchronize and timed with CUDA events on
the launching stream; N > 1 GPUs run independent replicas (weak scaling) and
the job time is the maximum over ranks.

Keys beyond the driver contract:
  e2e          -- the same metric through the C ABI (ipfc_gaussian_blur) with
                  pinned HOST buffers: H2D copy, kernel and D2H copy every step.
                  The call is synchronous; the steps are spread over
                  --e2e-threads host threads, each on its own stream, so that
                  uploads and downloads overlap as a threaded caller's would;
  roofline     -- algorithmic bytes (one read of the source + one write of the
                  destination) per launch / average launch time, against the
                  measured HBM copy bandwidth;
  cpu_baseline -- the reference's own threaded CPU path (its headers compiled
                  into oracle/_ref, ipf::setNumThreads(0)) on a bounded sample.

`--impl reference` runs only the reference's CPU implementation of the same
workload on the host cores (rank 0), each step a band of rows of one image.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import re
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W_IMG, H_IMG, C_IMG = 3840, 2160, 3
SIGMA = 2.0
BORDER_REFLECT101 = 3
METRIC = "Mpix/s plain vs batched/served at <=1 LSB; p50/p99 latency; % HBM roofline"
UNIT = "Mpix/s"
WORKLOAD = "gaussianBlur sigma=2 (13 taps) Reflect101, 3840x2160x3 uint8 -> uint8"
FALLBACK_HBM_GBS = 6650.0
PROFILE_SUMMARY = os.path.join(ROOT, "profiles", "sep_tcol_4k_rgb_u8.md")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--images-per-step", type=int, default=100)
    ap.add_argument("--buffers", type=int, default=6)
    ap.add_argument("--e2e-steps", type=int, default=30,
                    help="images through the e2e leg (at least one per host thread), independent of --steps")
    ap.add_argument("--e2e-threads", type=int, default=3,
                    help="host threads (each with its own stream) calling the synchronous C ABI in the e2e leg")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="leave the shortened filter2D / batch / serve measurements out of the default line")
    ap.add_argument("--extras-serve-requests", type=int, default=6000)
    ap.add_argument("--launches-only", type=int, default=0,
                    help="run this many launches of the workload on one resident image and exit (for ncu captures)")
    ap.add_argument("--workload", default="headline",
                    choices=["headline", "batch", "serve", "filter2d", "sep_sweep", "erode", "median3", "median5"],
                    help="headline: 4K RGB gaussianBlur (the driver's line); batch: 512-image uneven mix, "
                         "batched vs plain per-image launches; serve: Poisson request stream through the "
                         "continuous-batching server vs one request at a time; filter2d: FP32 vs split forms; "
                         "sep_sweep: f32 separable and Sobel sweep; erode, median3, median5: per-image calls "
                         "on 4K RGB (with --launches-only N: the profiling programs)")
    ap.add_argument("--serve-requests", type=int, default=20000)
    ap.add_argument("--serve-rate", type=float, default=3000.0, help="arrivals per second")
    ap.add_argument("--serve-seed", type=int, default=77)
    ap.add_argument("--serve-out-arena-mib", type=int, default=2048)
    ap.add_argument("--batch-images", type=int, default=512)
    ap.add_argument("--batch-seed", type=int, default=2024)
    ap.add_argument("--batch-max-side", type=int, default=2048)
    return ap.parse_args()


# ---------------------------------------------------------------------------
# CPU side: reference (oracle/_ref) or, where it was not built, the restatement
# ---------------------------------------------------------------------------

def cpu_impl():
    import oracle

    ref = oracle.reference()
    if ref is not None:
        ref.lib.ref_set_threads(0)
        return ref, "reference", int(ref.lib.ref_get_threads())
    return oracle.restatement(), "port", 1


def seeded_image(w, h, c):
    import oracle

    return oracle.random_image(w, h, c, "uint8", 1)


def time_cpu_baseline(img, seconds):
    impl, kind, cores = cpu_impl()
    impl.gaussian_blur(img[:64], SIGMA, 0.0, 0, BORDER_REFLECT101)  # warm-up
    t0 = time.perf_counter()
    n = 0
    while True:
        impl.gaussian_blur(img, SIGMA, 0.0, 0, BORDER_REFLECT101)
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or (n >= 3 and el >= seconds * 0.5):
            break
    mpix = n * W_IMG * H_IMG / el / 1e6
    return {"value": round(mpix, 3), "unit": UNIT, "cores": cores, "kind": kind,
            "sample": f"{n} full {W_IMG}x{H_IMG}x{C_IMG} uint8 images, gaussianBlur sigma=2 Reflect101, "
                      f"wall clock, {el:.1f} s"}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    impl, kind, cores = cpu_impl()
    img = seeded_image(W_IMG, H_IMG, C_IMG)
    # calibrate a band of rows to ~50 ms of work per step
    t0 = time.perf_counter()
    impl.gaussian_blur(img, SIGMA, 0.0, 0, BORDER_REFLECT101)
    t_full = time.perf_counter() - t0
    rows = int(max(16, min(H_IMG, H_IMG * 0.05 / max(t_full, 1e-6))))
    band = img[:rows].copy()
    for _ in range(args.warmup):
        impl.gaussian_blur(band, SIGMA, 0.0, 0, BORDER_REFLECT101)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        impl.gaussian_blur(band, SIGMA, 0.0, 0, BORDER_REFLECT101)
    el = time.perf_counter() - t0
    value = args.steps * W_IMG * rows / el / 1e6
    sample = f"each step: a {W_IMG}x{rows}x{C_IMG} uint8 band of the seeded image, whole-band gaussianBlur"
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(el / args.steps * 1e3, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded uniform 0-255)",
            "config": {"workload": WORKLOAD, "images_per_step": f"band of {rows} rows", "cpu_threads": cores},
            "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU side
# ---------------------------------------------------------------------------

def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic():
    """dram bytes per launch recorded from an ncu capture (profiles/)."""
    try:
        with open(PROFILE_SUMMARY) as f:
            m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", f.read())
        return float(m.group(1)) if m else None
    except OSError:
        return None


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.proc = None
        self.gpu = gpu_index

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        if not getattr(self, "lines", None):
            return None
        sm, mx, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def run_ours(args):
    import torch
    import torch.distributed as dist

    import imageprocessingflex_b200 as ipf
    from imageprocessingflex_b200 import _lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local if world > 1 else torch.cuda.current_device())
    lib = _lib.load()

    host = seeded_image(W_IMG, H_IMG, C_IMG)
    nbuf = max(2, args.buffers)
    srcs = [torch.from_numpy(host).to(dev) for _ in range(nbuf)]
    for i in range(1, nbuf):  # distinct contents per buffer
        srcs[i] = torch.roll(srcs[0], shifts=i * 7, dims=1).contiguous()
    dsts = [torch.empty_like(srcs[0]) for _ in range(nbuf)]

    stream = torch.cuda.Stream(dev)
    views = []
    for s, d in zip(srcs, dsts):
        sv = _lib.IpfcImage(s.data_ptr(), W_IMG, H_IMG, C_IMG, 0, W_IMG * C_IMG, 1)
        dv = _lib.IpfcImage(d.data_ptr(), W_IMG, H_IMG, C_IMG, 0, W_IMG * C_IMG, 1)
        views.append((sv, dv))
    sptr = ctypes.c_void_p(stream.cuda_stream)

    def one_step():
        for i in range(args.images_per_step):
            sv, dv = views[i % nbuf]
            rc = lib.ipfc_gaussian_blur(ctypes.byref(sv), ctypes.byref(dv), SIGMA, 0.0, 0, BORDER_REFLECT101, sptr)
            if rc:
                raise RuntimeError(lib.ipfc_last_error().decode())

    # one untimed pass before capture: loads the kernels, sizes the pool
    with torch.cuda.stream(stream):
        one_step()
    stream.synchronize()

    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream, capture_error_mode="thread_local"):
        one_step()
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize(dev)

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk:
        with torch.cuda.stream(stream):
            start.record(stream)
            for _ in range(args.steps):
                graph.replay()
            end.record(stream)
        end.synchronize()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    ms = start.elapsed_time(end)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    images = args.steps * args.images_per_step
    value = world * images * W_IMG * H_IMG / (ms_max / 1e3) / 1e6
    ms_per_launch = ms / images
    alg_bytes = 2.0 * W_IMG * H_IMG * C_IMG
    peak, peak_kind = measured_peak()
    achieved = alg_bytes / (ms_per_launch / 1e3) / 1e9
    traffic = profiled_traffic()

    # End to end through the C ABI with pinned host buffers.  The call is
    # synchronous (the result is in host memory when it returns), so a caller
    # overlaps uploads, kernels and downloads by calling from a few host
    # threads, each with its own stream and destination buffer.
    from concurrent.futures import ThreadPoolExecutor

    hsrc = torch.from_numpy(host).pin_memory()
    hsv = _lib.IpfcImage(hsrc.data_ptr(), W_IMG, H_IMG, C_IMG, 0, W_IMG * C_IMG, 0)
    n_thr = max(1, args.e2e_threads)
    lanes = []
    for _ in range(n_thr):
        hd = torch.empty_like(hsrc).pin_memory()
        st = torch.cuda.Stream(dev)
        lanes.append((hd, _lib.IpfcImage(hd.data_ptr(), W_IMG, H_IMG, C_IMG, 0, W_IMG * C_IMG, 0),
                      ctypes.c_void_p(st.cuda_stream), st))

    def e2e_lane(k, count):
        _, hdv, sp, _ = lanes[k]
        for _ in range(count):
            rc = lib.ipfc_gaussian_blur(ctypes.byref(hsv), ctypes.byref(hdv), SIGMA, 0.0, 0, BORDER_REFLECT101, sp)
            if rc:
                raise RuntimeError(lib.ipfc_last_error().decode())

    for k in range(n_thr):
        e2e_lane(k, 2)
    ref_out = dsts[0].cpu()
    ok_e2e = all(torch.equal(hd, ref_out) for hd, _, _, _ in lanes)
    e2e_steps = max(n_thr, args.e2e_steps)
    shares = [e2e_steps // n_thr + (1 if k < e2e_steps % n_thr else 0) for k in range(n_thr)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    w0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=n_thr) as pool:
        for f in [pool.submit(e2e_lane, k, shares[k]) for k in range(n_thr)]:
            f.result()
    e1.record(stream)
    e1.synchronize()
    wall = time.perf_counter() - w0
    ok_e2e = ok_e2e and all(torch.equal(hd, ref_out) for hd, _, _, _ in lanes)
    e_ms = max(e0.elapsed_time(e1), wall * 1e3)
    te = torch.tensor([e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
        dist.barrier()
    e2e_value = world * e2e_steps * W_IMG * H_IMG / (float(te.item()) / 1e3) / 1e6

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded uniform 0-255)",
            "config": {"workload": WORKLOAD, "images_per_step": args.images_per_step,
                       "resident_buffers": nbuf, "working_set_bytes": int(nbuf * alg_bytes),
                       "l2_policy": "inputs larger than L2: rotating buffer pairs, working set > 126 MB",
                       "accumulate": "f32", "parallelism": f"replicas x{world}", "timing": "CUDA graph replay, "
                       "CUDA events on the launching stream, max over ranks"},
            "gpu_launches": images,
            "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": int(W_IMG * H_IMG * C_IMG),
                    "d2h_bytes_per_step": int(W_IMG * H_IMG * C_IMG), "steps": e2e_steps,
                    "path": "ipfc_gaussian_blur, pinned host src/dst (IPFC_MEM_HOST)", "host_threads": n_thr,
                    "streams": n_thr, "matches_resident": ok_e2e},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else "fallback 6.65 TB/s", "kernel": "sep_tcol_kernel<13, 3, false> (tcgen05 column pass, saturation compiled out)",
                         "alg_bytes_per_launch": int(alg_bytes), "ms_per_launch": round(ms_per_launch, 5)},
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = time_cpu_baseline(host, args.cpu_seconds)
        if world == 1 and not args.no_extras:
            line.update(measure_extras(args))
        print(json.dumps(line), flush=True)
    del graph
    if world > 1:
        dist.destroy_process_group()
    return 0


def measure_extras(args):
    """The other measured configurations, shortened, for the default line:
    split vs FP32 filter2D 31x31 on 4096x4096 uint8 (with FP64 error), the
    512-image batched uneven mix against per-image launches, and a served
    stream of `extras_serve_requests` requests (continuous vs one at a time).
    Each is the same code as its --workload line, with fewer steps."""
    out = {}
    t0 = time.perf_counter()
    try:
        rows, tf, _, _ = filter2d_cases(args, (("u8", 31),), 5)
        r = tf[("u8", 31)]
        out["d3_filter2d_31x31_u8_4096"] = {
            "split_ms": r["split"]["ms"], "fp32_ms": r["fp32"]["ms"], "speedup_split_vs_fp32": r["speedup_split_vs_fp32"],
            "split_tflops": r["split"]["tflops"], "split_frac_of_bf16_peak": r["split"]["frac_of_bf16_peak"],
            "fp32_frac_of_fp32_fma_peak": r["fp32"]["frac_of_fp32_fma_peak"],
            "err_vs_fp64_max": {"split": r["split"]["err_vs_fp64_max"], "fp32": r["fp32"]["err_vs_fp64_max"]},
            "err_vs_fp64_mean": {"split": r["split"]["err_vs_fp64_mean"], "fp32": r["fp32"]["err_vs_fp64_mean"]},
            "u8_max_lsb": r["split"].get("u8_max_lsb"), "u8_mismatch_rate": r["split"].get("u8_mismatch_rate"),
            "error_sample": "1024x512 crop, same taps"}
    except Exception as exc:  # reported, never silently dropped
        out["d3_filter2d_31x31_u8_4096"] = {"error": str(exc)[:300]}
    try:
        ba = argparse.Namespace(**vars(args))
        ba.steps, ba.warmup = 5, 2
        bl = run_batch(ba, quiet=True)
        out["d4_batch_512"] = {"batched_ms": bl["batched"]["ms"], "plain_ms": bl["plain"]["ms"],
                               "speedup_vs_plain": bl["speedup_vs_plain"], "mpix_s": bl["value"],
                               "results_equal_per_image": bl["results_equal_per_image"],
                               "roofline_frac": bl["roofline"]["frac"], "kernels_per_step": bl["gpu_launches"] // 5,
                               "plan_seconds": bl["batched"]["plan_seconds"]}
    except Exception as exc:
        out["d4_batch_512"] = {"error": str(exc)[:300]}
    try:
        sa = argparse.Namespace(**vars(args))
        sa.serve_requests = args.extras_serve_requests
        sl = run_serve(sa, quiet=True)
        c, p = sl["continuous"], sl["plain"]
        out["d5_serve"] = {"requests": sa.serve_requests, "rate_per_s": sa.serve_rate,
                           "continuous": {k: c[k] for k in ("p50_ms", "p99_ms", "mpix_s", "failed", "capacity_mpix_s")},
                           "plain": {k: p[k] for k in ("p50_ms", "p99_ms", "mpix_s", "failed", "capacity_mpix_s")},
                           "speedup_vs_plain_mpix": sl["speedup_vs_plain_mpix"],
                           "capacity_speedup_vs_plain": sl["capacity_speedup_vs_plain"]}
    except Exception as exc:
        out["d5_serve"] = {"error": str(exc)[:300]}
    out["extras_seconds"] = round(time.perf_counter() - t0, 1)
    return out


def run_batch(args, quiet=False):
    """The batched uneven mix (512 uint8 images, w and h uniform in [64, 2048],
    channels from {1, 3, 4}; gaussianBlur sigma ~ U[0.5, 4] 50 %, medianBlur 3
    or 5 25 %, erode / dilate 3x3 rect 25 %), resident in HBM.  Three forms of
    the same work, each timed with CUDA events over `steps` repetitions:
      batched      -- one ipfc_batch_run per step (graph of the persistent
                      kernels: one launch per register class);
      plain        -- one C-ABI call per image, issued from the host each step
                      (the per-image-launch form a caller writes);
      plain_graph  -- the same per-image calls captured once in a CUDA graph
                      (what per-image launches cost without host overhead).
    Every batched image is checked equal to its per-image result first."""
    import torch

    import imageprocessingflex_b200 as ipf
    from imageprocessingflex_b200 import _lib, mix
    from imageprocessingflex_b200 import batch as B

    dev = torch.device("cuda", torch.cuda.current_device())
    lib = _lib.load()
    items = mix.uneven_mix(args.batch_images, seed=args.batch_seed, lo=64, hi=args.batch_max_side)
    srcs, dst_b, dst_p = [], [], []
    for it in items:
        shape = (it.height, it.width, it.channels) if it.channels > 1 else (it.height, it.width)
        s_ = torch.empty(shape, dtype=torch.uint8, device=dev)
        mix.fill_uniform_u8(s_, it.seed)
        srcs.append(s_)
        dst_b.append(torch.empty_like(s_))
        dst_p.append(torch.empty_like(s_))
    se = ipf.getStructuringElement(ipf.MorphShape.Rect, 3)
    stream = torch.cuda.Stream(dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    views = [(_lib.IpfcImage(s_.data_ptr(), it.width, it.height, it.channels, 0, it.width * it.channels, 1),
              _lib.IpfcImage(d_.data_ptr(), it.width, it.height, it.channels, 0, it.width * it.channels, 1))
             for it, s_, d_ in zip(items, srcs, dst_p)]
    se_p = se.ctypes.data

    def plain_step():
        for it, (sv, dv) in zip(items, views):
            if it.op == "gaussian":
                rc = lib.ipfc_gaussian_blur(ctypes.byref(sv), ctypes.byref(dv), it.sigma, 0.0, 0, BORDER_REFLECT101,
                                            sptr)
            elif it.op == "median":
                rc = lib.ipfc_median_blur(ctypes.byref(sv), ctypes.byref(dv), it.ksize, 1, sptr)
            elif it.op == "erode":
                rc = lib.ipfc_erode(ctypes.byref(sv), ctypes.byref(dv), se_p, 3, 3, 1, sptr)
            else:
                rc = lib.ipfc_dilate(ctypes.byref(sv), ctypes.byref(dv), se_p, 3, 3, 1, sptr)
            if rc:
                raise RuntimeError(lib.ipfc_last_error().decode())

    b = B.Batch()
    for it, s_, d_ in zip(items, srcs, dst_b):
        if it.op == "gaussian":
            b.add_gaussianBlur(s_, d_, it.sigma)
        elif it.op == "median":
            b.add_medianBlur(s_, d_, it.ksize)
        elif it.op == "erode":
            b.add_erode(s_, d_, se)
        else:
            b.add_dilate(s_, d_, se)

    t_plan = time.perf_counter()
    b.run(stream)  # plans: autotunes unseen keys, captures the graph
    stream.synchronize()
    t_plan = time.perf_counter() - t_plan
    with torch.cuda.stream(stream):
        plain_step()
    stream.synchronize()
    # Batched separable items run the CUDA-core tile code; per-image calls on
    # large uint8 images run the tensor-core kernel.  Both are within 1 LSB of
    # the reference, so they agree within 1 LSB (bit for bit elsewhere).
    same = all(torch.equal(x, y) for x, y in zip(dst_b, dst_p))
    within1 = all(int((x.int() - y.int()).abs().max()) <= 1 for x, y in zip(dst_b, dst_p) if x.numel())
    if not within1:
        raise RuntimeError("batched results differ from the per-image calls by more than 1 LSB")

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        stream.synchronize()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(steps):
                fn()
            e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / steps

    with ClockSampler(dev.index) as clk:
        ms_batched = timed(lambda: b.run(stream), args.steps)
    ms_plain = timed(plain_step, max(1, min(args.steps, 5)))
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream, capture_error_mode="thread_local"):
        plain_step()
    ms_plain_graph = timed(g.replay, max(1, min(args.steps, 5)))
    del g
    # where the per-image form's time goes: each op's images alone
    by_op = {}
    all_items, all_views = items, views
    for op in (() if quiet else ("gaussian", "median", "erode", "dilate")):
        sel = [i for i, it in enumerate(all_items) if it.op == op]
        items = [all_items[i] for i in sel]
        views = [all_views[i] for i in sel]
        by_op[op] = round(timed(plain_step, max(1, min(args.steps, 3))), 3)
    items, views = all_items, all_views

    mpix = sum(it.pixels for it in items) / 1e6
    alg_bytes = 2.0 * sum(it.pixels * it.channels for it in items)
    peak, peak_kind = measured_peak()
    achieved = alg_bytes / (ms_batched / 1e3) / 1e9
    kernels = b.info("kernels")
    ops = {o: sum(1 for it in items if it.op == o) for o in ("gaussian", "median", "erode", "dilate")}
    line = {
        "metric": METRIC, "value": round(mpix / (ms_batched / 1e3), 3), "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_batched, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded uniform 0-255)",
        "config": {"workload": f"batched uneven mix: {len(items)} uint8 images, w,h ~ U[64,{args.batch_max_side}], "
                               "C in {1,3,4}; gaussianBlur sigma~U[0.5,4] 50%, medianBlur 3|5 25%, "
                               "erode|dilate 3x3 rect 25%", "seed": args.batch_seed, "ops": ops,
                   "megapixels_per_step": round(mpix, 3), "bytes_per_step": int(alg_bytes),
                   "l2_policy": "inputs larger than L2 (working set of several GB)",
                   "timing": "CUDA events on the launching stream"},
        "gpu_launches": kernels * args.steps,
        "batched": {"ms": round(ms_batched, 4), "mpix_s": round(mpix / (ms_batched / 1e3), 1),
                    "kernels_per_step": kernels, "tiles": b.info("tiles_light") + b.info("tiles_heavy") + b.info("tiles_mem"),
                    "plan_seconds": round(t_plan, 3)},
        "plain": {"ms": round(ms_plain, 4), "mpix_s": round(mpix / (ms_plain / 1e3), 1),
                  "launches_per_step": len(items), "form": "one C-ABI call per image from the host"},
        "plain_graph": {"ms": round(ms_plain_graph, 4), "mpix_s": round(mpix / (ms_plain_graph / 1e3), 1)},
        "plain_ms_by_op": by_op,
        "speedup_vs_plain": round(ms_plain / ms_batched, 3),
        "speedup_vs_plain_graph": round(ms_plain_graph / ms_batched, 3),
        "results_equal_per_image": same, "results_within_1lsb_of_per_image": within1,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None,
                     "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                     else "fallback 6.65 TB/s",
                     "alg_bytes_per_step": int(alg_bytes)},
        "clocks": clk.summary(),
    }
    b.close()
    if quiet:
        return line
    print(json.dumps(line), flush=True)
    return 0


def run_serve(args, quiet=False):
    """The served stream: `serve_requests` requests with Poisson arrivals at
    `serve_rate`/s (area lognormal, median 1 MP, log-sd 1, clipped to
    0.01-33 MP; aspect U[0.5, 2]; C in {1, 3}; uint8; gaussianBlur 45 %,
    sobel 20 %, medianBlur 5x5 15 %, filter2D 15x15 20 %) from pinned host
    memory and back, replayed open-loop through two servers on the same trace:
      continuous -- ipfc_server defaults: 40 GiB budget, 64 slots, 4 streams,
                    batchable requests merged into persistent launches;
      plain      -- one request at a time (1 slot, 1 stream, no batching).
    Latency = completion - scheduled arrival (the host's submit jitter counts
    against the server).  Mpix/s = pixels served / (last completion - first
    arrival).  Capacity: the same requests again with every arrival already
    due, pixels / (last completion - first submit): the highest rate each
    form sustains."""
    from collections import deque

    import numpy as np
    import torch

    from imageprocessingflex_b200 import mix
    from imageprocessingflex_b200 import serve as S

    reqs = mix.served_stream(args.serve_requests, rate=args.serve_rate, seed=args.serve_seed)
    taps = mix.filter2d_taps()
    in_bytes = 512 << 20
    g = torch.Generator()
    g.manual_seed(args.serve_seed)
    arena_in = torch.randint(0, 256, (in_bytes,), dtype=torch.uint8, generator=g).pin_memory()
    out_bytes = args.serve_out_arena_mib << 20
    arena_out = torch.empty(out_bytes, dtype=torch.uint8).pin_memory()
    rng = np.random.default_rng(args.serve_seed + 1)
    offs = []
    for r in reqs:
        nb = r.pixels * r.channels
        offs.append(int(rng.integers(0, (in_bytes - nb) // 256 + 1)) * 256)

    def shape(r):
        return (r.height, r.width, r.channels) if r.channels > 1 else (r.height, r.width)

    def run_arm(server, trace, t0):
        ring = deque()
        done = {}
        pos = 0

        def collect(wait_ms=0):
            for c in server.poll(4096, wait_ms):
                done[c.ticket] = c

        for i, r in trace:
            nb = r.pixels * r.channels
            src = arena_in[offs[i]:offs[i] + nb].view(shape(r))
            ob = nb * (4 if r.op == "sobel" else 1)
            need = (ob + 255) // 256 * 256
            if need > out_bytes:
                raise RuntimeError("output arena smaller than one request")
            if pos + need > out_bytes:
                pos = 0
            while ring and ring[0][1] < pos + need and ring[0][2] > pos:
                if ring[0][0] in done:
                    ring.popleft()
                else:
                    collect(1)
            raw = arena_out[pos:pos + ob]
            dst = raw.view(torch.float32).view(shape(r)) if r.op == "sobel" else raw.view(shape(r))
            target = t0 + r.arrival
            while server.now() < target:
                pass
            if r.op == "gaussian":
                t = server.submit("gaussian", src, dst, target, sigma_x=r.sigma, keep=False)
            elif r.op == "sobel":
                t = server.submit("sobel", src, dst, target, dx=r.dx, dy=r.dy, ksize=3, keep=False)
            elif r.op == "median":
                t = server.submit("median", src, dst, target, ksize=5, keep=False)
            else:
                t = server.submit("filter2d", src, dst, target, kernel=taps, keep=False)
            ring.append((t, pos, pos + need))
            pos += need
            if (i & 63) == 0:
                collect()
        server.drain()
        collect()
        return done

    arms = {}
    for name, kw in (("continuous", {}), ("plain", {"max_inflight": 1, "streams": 1, "batch": False})):
        server = S.Server(**kw)
        # warm-up, all due at once: the first 200 requests plus the first request
        # of every (op, taps, channels) kind in the trace, so that every kernel
        # variant is loaded before the timed replay
        warm_idx, kinds = list(range(min(200, len(reqs)))), set()
        for i, r in enumerate(reqs):
            kind = (r.op, 2 * int(3.0 * r.sigma + 0.5) + 1 if r.op == "gaussian" else 0, r.channels)
            if kind not in kinds:
                kinds.add(kind)
                if i >= 200:
                    warm_idx.append(i)
        warm = [(i, reqs[i]) for i in warm_idx]
        run_arm(server, warm, server.now() - reqs[0].arrival)
        torch.cuda.synchronize()
        t0 = server.now() + 0.1
        with ClockSampler(torch.cuda.current_device()) as clk:
            done = run_arm(server, list(enumerate(reqs)), t0)
        st = server.stats()
        # capacity: the same requests replayed with every arrival already due,
        # so the rate is the server's, not the stream's
        t_cap = server.now()
        done_cap = run_arm(server, list(enumerate(reqs)), t_cap - max(r.arrival for r in reqs) - 1.0)
        cap_span = max(c.done for c in done_cap.values()) - t_cap
        cap_bad = sum(1 for c in done_cap.values() if c.status != 0)
        server.close()
        timed = [done[t] for t in sorted(done)]
        if len(timed) != len(reqs):
            raise RuntimeError(f"{name}: {len(timed)} completions for {len(reqs)} requests")
        bad = sum(1 for c in timed if c.status != 0)
        lat = np.array([c.latency for c in timed]) * 1e3
        span = max(c.done for c in timed) - min(c.arrival for c in timed)
        mpix = sum(r.pixels for r in reqs) / 1e6
        arms[name] = {"mpix_s": round(mpix / span, 1), "requests_per_s": round(len(reqs) / span, 1),
                      "p50_ms": round(float(np.percentile(lat, 50)), 3),
                      "p99_ms": round(float(np.percentile(lat, 99)), 3), "mean_ms": round(float(lat.mean()), 3),
                      "max_ms": round(float(lat.max()), 3), "failed": bad, "span_s": round(span, 3),
                      "max_inflight": int(st["max_inflight"]), "max_device_bytes": int(st["max_bytes"]),
                      "batched_requests": int(st["batched"]), "batch_launches": int(st["batch_launches"]),
                      "capacity_mpix_s": round(sum(r.pixels for r in reqs) / 1e6 / cap_span, 1),
                      "capacity_requests_per_s": round(len(reqs) / cap_span, 1), "capacity_failed": cap_bad,
                      "clocks": clk.summary()}
    c, p = arms["continuous"], arms["plain"]
    ops = {o: sum(1 for r in reqs if r.op == o) for o in ("gaussian", "sobel", "median", "filter2d")}
    in_total = sum(r.pixels * r.channels for r in reqs)
    out_total = sum(r.pixels * r.channels * (4 if r.op == "sobel" else 1) for r in reqs)
    line = {
        "metric": METRIC, "value": c["mpix_s"], "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": 1,
        "ms_per_step": round(c["span_s"] * 1e3, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8", "data": "synthetic (seeded uniform 0-255)",
        "config": {"workload": f"served stream: {len(reqs)} requests, Poisson arrivals at {args.serve_rate}/s; area "
                               "lognormal median 1 MP log-sd 1 clipped 0.01-33 MP; aspect U[0.5,2]; C in {1,3}; "
                               "gaussianBlur 45% (sigma~U[0.5,4]) / sobel 20% (ksize 3, f32 out) / medianBlur 5x5 "
                               "15% / filter2D 15x15 20%; 40 GiB device budget", "seed": args.serve_seed,
                   "ops": ops, "h2d_bytes": in_total, "d2h_bytes": out_total,
                   "latency": "completion - scheduled arrival, host clock", "host_memory": "pinned"},
        "latency_ms": {"p50": c["p50_ms"], "p99": c["p99_ms"]},
        "continuous": c, "plain": p,
        "speedup_vs_plain_mpix": round(c["mpix_s"] / p["mpix_s"], 3),
        "capacity_speedup_vs_plain": round(c["capacity_mpix_s"] / p["capacity_mpix_s"], 3),
        "e2e": {"value": c["mpix_s"], "unit": UNIT, "h2d_bytes_per_step": in_total, "d2h_bytes_per_step": out_total},
        "clocks": c["clocks"],
    }
    if quiet:
        return line
    print(json.dumps(line), flush=True)
    return 0


def run_filter2d(args):
    """Dense filter2D on 4096x4096x1 (uint8 uniform 0-255 and float U[0,1)),
    seeded N(0,1) taps normalised to sum 1, 15x15 and 31x31, Reflect101: the
    FP32 CUDA-core form against the split-precision tcgen05 form, each timed
    with CUDA events over `steps` launches on resident images (inputs larger
    than L2 are not needed: the op is compute-bound; two image pairs rotate).
    Errors against the FP64 oracle are measured on a 1024x512 crop of the same
    kind of image with the same taps."""
    results, tf, tc_peak, tc_peak_source = filter2d_cases(args, (("u8", 15), ("u8", 31), ("f32", 15), ("f32", 31)),
                                                          args.steps)
    head = tf[("u8", 31)]
    line = {
        "metric": METRIC, "value": head["split"]["mpix_s"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["split"]["ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8 pixels exact in f16, taps f16 hi+lo, f32 accumulate",
        "data": "synthetic (seeded uniform)",
        "config": {"workload": "filter2D 4096x4096x1, dense N(0,1) taps normalised to sum 1, Reflect101; FP32 "
                               "CUDA-core form vs split-precision tcgen05 form", "value_is": "u8 31x31 split Mpix/s",
                   "flops_per_launch": "2*W*H*kw*kh (counted once, not per hi/lo product)"},
        "cases": results,
        "roofline": {"bound": "tensor", "achieved": head["split"]["tflops"], "peak": tc_peak, "unit": "TFLOP/s",
                     "frac": head["split"]["frac_of_bf16_peak"], "traffic": None,
                     "peak_source": tc_peak_source},
        "gpu_launches": (args.steps + args.warmup) * 8,
    }
    print(json.dumps(line), flush=True)
    return 0


def filter2d_cases(args, cases, steps):
    """Times the FP32 and split forms of filter2D on 4096x4096x1 for each
    (dtype, k) of `cases`; returns (rows, rows by case, tensor peak, its source)."""
    import numpy as np
    import torch

    import imageprocessingflex_b200 as ipf
    import oracle
    from imageprocessingflex_b200 import _lib, mix

    lib = _lib.load()
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.Stream(dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    N = 4096
    tf = {}
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    tc_peak = float(peaks.get("bf16_tflops", 1590.0))
    tc_peak_source = ("MEASURED_PEAKS.json bf16_tflops (dense, burst)" if "bf16_tflops" in peaks
                      else "fallback 1.59 PFLOP/s (MEASURED_PEAKS.json absent)")
    fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12  # FP32 FMA pipe, TFLOP/s at the max clock
    orc = oracle.restatement()
    results = []
    for dt in ("u8", "f32"):
        if not any(c[0] == dt for c in cases):
            continue
        g = torch.Generator(device=dev)
        g.manual_seed(3)
        if dt == "u8":
            srcs = [torch.randint(0, 256, (N, N), generator=g, device=dev, dtype=torch.int32).to(torch.uint8)
                    for _ in range(2)]
            code, es = 0, 1
        else:
            srcs = [torch.rand((N, N), generator=g, device=dev, dtype=torch.float32) for _ in range(2)]
            code, es = 4, 4
        dsts = [torch.empty_like(x) for x in srcs]
        views = [(_lib.IpfcImage(x.data_ptr(), N, N, 1, code, N * es, 1), _lib.IpfcImage(y.data_ptr(), N, N, 1, code,
                                                                                           N * es, 1))
                 for x, y in zip(srcs, dsts)]
        crop = oracle.random_image(1024, 512, 1, np.uint8 if dt == "u8" else np.float32, 11)
        for kk in (15, 31):
            if (dt, kk) not in cases:
                continue
            taps = mix.filter2d_taps(kk, seed=1000 + kk)
            tp = taps.ctypes.data
            row = {"dtype": dt, "taps": f"{kk}x{kk}"}
            for form, fn in (("fp32", lib.ipfc_filter2d_fp32), ("split", lib.ipfc_filter2d_split)):
                def step(i):
                    sv, dv = views[i % 2]
                    rc = fn(ctypes.byref(sv), ctypes.byref(dv), tp, kk, kk, -1, -1, BORDER_REFLECT101, 0.0, 0.0, sptr)
                    if rc:
                        raise RuntimeError(lib.ipfc_last_error().decode())
                nsteps = max(2, steps if form == "split" else min(steps, 5))
                for i in range(args.warmup):
                    step(i)
                stream.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for i in range(nsteps):
                    step(i)
                e1.record(stream)
                e1.synchronize()
                ms = e0.elapsed_time(e1) / nsteps
                flops = 2.0 * N * N * kk * kk
                row[form] = {"ms": round(ms, 4), "mpix_s": round(N * N / (ms / 1e3) / 1e6, 1),
                             "tflops": round(flops / (ms / 1e3) / 1e12, 2)}
            row["speedup_split_vs_fp32"] = round(row["fp32"]["ms"] / row["split"]["ms"], 3)
            row["split"]["frac_of_bf16_peak"] = round(row["split"]["tflops"] / tc_peak, 4)
            row["fp32"]["frac_of_fp32_fma_peak"] = round(row["fp32"]["tflops"] / fp32_peak, 4)
            # errors against the FP64 oracle (crop)
            ref = orc.filter2d(crop, taps, 3, 0.0, (-1, -1), 0.0, np.float64)
            for form in ("fp32", "split"):
                got = ipf.filter2D(crop, taps, form=form, dtype=np.float32).astype(np.float64)
                err = np.abs(got - ref)
                row[form]["err_vs_fp64_max"] = float(f"{err.max():.4g}")
                row[form]["err_vs_fp64_mean"] = float(f"{err.mean():.4g}")
            if dt == "u8":
                want = orc.filter2d(crop, taps, 3)
                got = ipf.filter2D(crop, taps, form="split")
                d = np.abs(got.astype(int) - want.astype(int))
                row["split"]["u8_max_lsb"] = int(d.max())
                row["split"]["u8_mismatch_rate"] = float(f"{(d > 0).mean():.4g}")
                row["saturated_fraction"] = float(f"{((want == 0) | (want == 255)).mean():.4g}")
            results.append(row)
            tf[(dt, kk)] = row
    return results, tf, tc_peak, tc_peak_source


def run_sep_sweep(args):
    """The separable sweep: 3840x2160x1 float32 U[0,1), sepFilter2D with seeded
    random taps normalised to sum 1, lengths 3, 7, 15, 31 on both axes, each
    under the five borders; and Sobel (dx, dy) = (1, 0), (0, 1), ksize 3 and 5,
    on 3840x2160x1 uint8 -> int16.  Each case: `steps` C-ABI calls on resident
    device images (two pairs rotating, 66 MB per float image pair), captured
    in a CUDA graph where the call captures (the fast kernels: taps travel in
    the kernel parameters) and replayed, else issued back to back; timed with
    CUDA events on the launching stream.  Parity for every
    case is in the tests (full-size float sweep and exact int16 Sobel)."""
    import numpy as np
    import torch

    from imageprocessingflex_b200 import _lib

    lib = _lib.load()
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.Stream(dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    W, H = 3840, 2160
    peak, peak_kind = measured_peak()
    g = torch.Generator(device=dev)
    g.manual_seed(2)
    fsrc = [torch.rand((H, W), generator=g, device=dev) for _ in range(2)]
    fdst = [torch.empty_like(x) for x in fsrc]
    usrc = [torch.randint(0, 256, (H, W), generator=g, device=dev, dtype=torch.int32).to(torch.uint8) for _ in range(2)]
    idst = [torch.empty((H, W), dtype=torch.int16, device=dev) for _ in range(2)]

    def view(t, code, esize):
        return _lib.IpfcImage(t.data_ptr(), W, H, 1, code, W * esize, 1)

    fv = [(view(a, 4, 4), view(b, 4, 4)) for a, b in zip(fsrc, fdst)]
    uv = [(view(a, 0, 1), view(b, 2, 2)) for a, b in zip(usrc, idst)]
    steps = max(3, args.steps)

    def timed(call):
        """(ms per call, method): a CUDA graph of `steps` calls where the call
        can be captured (no host-side launch overhead), else plain calls."""
        for i in range(3):
            call(i % 2)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        graph = torch.cuda.CUDAGraph()
        try:
            with torch.cuda.graph(graph, stream=stream, capture_error_mode="thread_local"):
                for i in range(steps):
                    call(i % 2)
        except Exception:
            graph = None
            torch.cuda.synchronize(dev)
            lib.ipfc_last_error()
        if graph is not None:
            with torch.cuda.stream(stream):  # replay() launches on the current stream
                graph.replay()
            stream.synchronize()
            e0.record(stream)
            with torch.cuda.stream(stream):
                graph.replay()
            e1.record(stream)
            e1.synchronize()
            del graph
            return e0.elapsed_time(e1) / steps, "graph"
        e0.record(stream)
        for i in range(steps):
            call(i % 2)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / steps, "calls"

    rng = np.random.default_rng(2024)
    cases = []
    border_names = ["constant", "replicate", "reflect", "reflect101", "wrap"]
    with ClockSampler(dev.index) as clk:
        for k in (3, 7, 15, 31):
            kx = rng.uniform(0.1, 1.0, size=k)
            ky = rng.uniform(0.1, 1.0, size=k)
            kx, ky = kx / kx.sum(), ky / ky.sum()
            for b in range(5):
                def call(i, kx=kx, ky=ky, b=b):
                    sv, dv = fv[i]
                    rc = lib.ipfc_sep_filter2d(ctypes.byref(sv), ctypes.byref(dv), kx.ctypes.data, k,
                                               ky.ctypes.data, k, -1, -1, b, 0.0, 0.25, sptr)
                    if rc:
                        raise RuntimeError(lib.ipfc_last_error().decode())
                ms, how = timed(call)
                gbs = 2 * 4 * W * H / (ms / 1e3) / 1e9
                cases.append({"op": "sepFilter2D f32", "taps": k, "border": border_names[b], "timing": how,
                              "ms": round(ms, 4),
                              "mpix_s": round(W * H / (ms / 1e3) / 1e6, 1), "gb_s": round(gbs, 1),
                              "frac_hbm": round(gbs / peak, 4)})
        for ksz in (3, 5):
            for dx, dy in ((1, 0), (0, 1)):
                def call(i, ksz=ksz, dx=dx, dy=dy):
                    sv, dv = uv[i]
                    rc = lib.ipfc_sobel(ctypes.byref(sv), ctypes.byref(dv), dx, dy, ksz, 1.0, 3, sptr)
                    if rc:
                        raise RuntimeError(lib.ipfc_last_error().decode())
                ms, how = timed(call)
                gbs = (1 + 2) * W * H / (ms / 1e3) / 1e9
                cases.append({"op": "sobel u8->i16", "ksize": ksz, "dx": dx, "dy": dy, "timing": how,
                              "ms": round(ms, 4),
                              "mpix_s": round(W * H / (ms / 1e3) / 1e6, 1), "gb_s": round(gbs, 1),
                              "frac_hbm": round(gbs / peak, 4)})
    head = next(c for c in cases if c["op"].startswith("sep") and c["taps"] == 15 and c["border"] == "reflect101")
    line = {
        "metric": METRIC, "value": head["mpix_s"], "unit": UNIT, "n_gpus": 1, "steps": steps, "warmup": 3,
        "ms_per_step": head["ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (sepFilter2D), u8->i16 (sobel)", "data": "synthetic (seeded uniform)",
        "config": {"workload": "separable sweep: 3840x2160x1 f32 sepFilter2D, taps 3/7/15/31 x 5 borders; "
                               "sobel 3840x2160x1 u8->int16, ksize 3/5, dx/dy",
                   "value_is": "f32 15+15 taps Reflect101 Mpix/s",
                   "timing": "CUDA events around a CUDA graph of the C-ABI calls where they capture, else the calls",
                   "l2_policy": "two 66 MB image pairs rotating (inputs larger than L2 per pair of calls)"},
        "cases": cases,
        "roofline": {"bound": "hbm", "achieved": head["gb_s"], "peak": peak, "unit": "GB/s", "frac": head["frac_hbm"],
                     "traffic": None, "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                     else "fallback 6.65 TB/s"},
        "gpu_launches": len(cases) * (steps + 3),
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    return 0


def launches_only(n, workload="headline"):
    """n plain launches of a workload's main kernel on resident data, no
    timing: the programs profiled by the ncu captures summarised under
    profiles/.
      headline -- gaussianBlur(sigma=2) on one 3840x2160x3 uint8 image;
      filter2d -- the split-precision tcgen05 filter2D, 31x31 seeded N(0,1)
                  taps, on one 4096x4096 uint8 image;
      batch    -- the 512-image uneven mix as one batch (plan, then n runs);
      erode    -- erode by the 3x3 rectangle on one 3840x2160x3 uint8 image;
      median3, median5 -- medianBlur 3x3 / 5x5 on that image."""
    import torch

    import imageprocessingflex_b200 as ipf

    if workload == "filter2d":
        from imageprocessingflex_b200 import mix

        g = torch.Generator(device="cuda")
        g.manual_seed(3)
        x = torch.randint(0, 256, (4096, 4096), generator=g, device="cuda", dtype=torch.int32).to(torch.uint8)
        taps = mix.filter2d_taps(31, seed=1031)
        for _ in range(n):
            y = ipf.filter2D(x, taps, form="split")
    elif workload == "batch":
        from imageprocessingflex_b200 import batch as B
        from imageprocessingflex_b200 import mix

        items = mix.uneven_mix(512, seed=2024)
        b = B.Batch()
        keep = []
        for it in items:
            shape = (it.height, it.width, it.channels) if it.channels > 1 else (it.height, it.width)
            s_ = torch.empty(shape, dtype=torch.uint8, device="cuda")
            mix.fill_uniform_u8(s_, it.seed)
            d_ = torch.empty_like(s_)
            keep += [s_, d_]
            if it.op == "gaussian":
                b.add_gaussianBlur(s_, d_, it.sigma)
            elif it.op == "median":
                b.add_medianBlur(s_, d_, it.ksize)
            elif it.op == "erode":
                b.add_erode(s_, d_)
            else:
                b.add_dilate(s_, d_)
        for _ in range(n):
            b.run()
        y = keep[-1]
    elif workload in ("erode", "median3", "median5"):
        x = torch.from_numpy(seeded_image(W_IMG, H_IMG, C_IMG)).cuda()
        se = ipf.getStructuringElement(ipf.MorphShape.Rect, 3)
        for _ in range(n):
            y = ipf.erode(x, se) if workload == "erode" else ipf.medianBlur(x, 3 if workload == "median3" else 5)
    else:
        x = torch.from_numpy(seeded_image(W_IMG, H_IMG, C_IMG)).cuda()
        for _ in range(n):
            y = ipf.gaussianBlur(x, SIGMA)
    torch.cuda.synchronize()
    print(f"{n} launches done ({workload}), checksum {int(y.to(torch.int64).sum().item())}")
    return 0


def run_neighbourhood_op(args):
    """erode 3x3, medianBlur 3x3 or 5x5 on 3840x2160x3 uint8 device images
    through the C ABI: `images_per_step` calls over `buffers` rotating
    source/destination pairs (working set > L2), captured in a CUDA graph;
    CUDA events around `steps` replays.  Roofline: 2*W*H*C bytes per image
    against the measured HBM copy bandwidth."""
    import numpy as np
    import torch

    from imageprocessingflex_b200 import _lib

    if not torch.cuda.is_available():
        print(f"bench.py: --workload {args.workload} needs a GPU", file=sys.stderr)
        return 2
    lib = _lib.load()
    dev = torch.device("cuda", torch.cuda.current_device())
    host = seeded_image(W_IMG, H_IMG, C_IMG)
    nbuf = max(2, args.buffers)
    srcs = [torch.roll(torch.from_numpy(host).to(dev), shifts=i * 7, dims=1).contiguous() for i in range(nbuf)]
    dsts = [torch.empty_like(srcs[0]) for _ in range(nbuf)]
    views = [(_lib.IpfcImage(a.data_ptr(), W_IMG, H_IMG, C_IMG, 0, W_IMG * C_IMG, 1),
              _lib.IpfcImage(b.data_ptr(), W_IMG, H_IMG, C_IMG, 0, W_IMG * C_IMG, 1)) for a, b in zip(srcs, dsts)]
    se = np.ones((3, 3), np.uint8)
    stream = torch.cuda.Stream(dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)

    def one_step():
        for i in range(args.images_per_step):
            sv, dv = views[i % nbuf]
            if args.workload == "erode":
                rc = lib.ipfc_erode(ctypes.byref(sv), ctypes.byref(dv), se.ctypes.data, 3, 3, 1, sptr)
            else:
                k = 3 if args.workload == "median3" else 5
                rc = lib.ipfc_median_blur(ctypes.byref(sv), ctypes.byref(dv), k, BORDER_REFLECT101, sptr)
            if rc:
                raise RuntimeError(lib.ipfc_last_error().decode())

    with torch.cuda.stream(stream):
        one_step()
    stream.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream, capture_error_mode="thread_local"):
        one_step()
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize(dev)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk:
        with torch.cuda.stream(stream):
            start.record(stream)
            for _ in range(args.steps):
                graph.replay()
            end.record(stream)
        end.synchronize()
    ms = start.elapsed_time(end)
    per = ms / (args.steps * args.images_per_step)
    alg = 2.0 * W_IMG * H_IMG * C_IMG
    peak, peak_kind = measured_peak()
    achieved = alg / (per / 1e3) / 1e9
    mpix = W_IMG * H_IMG * args.images_per_step * args.steps / (ms / 1e3) / 1e6
    names = {"erode": "erode 3x3 rect", "median3": "medianBlur 3x3 Reflect101", "median5": "medianBlur 5x5 Reflect101"}
    line = {"metric": METRIC, "value": round(mpix, 1), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded uniform 0-255)",
            "config": {"workload": f"{names[args.workload]}, 3840x2160x3 uint8 -> uint8, device images",
                       "images_per_step": args.images_per_step, "resident_buffers": nbuf,
                       "l2_policy": "rotating buffer pairs, working set > 126 MB",
                       "timing": "CUDA graph replay, CUDA events on the launching stream"},
            "us_per_image": round(per * 1e3, 2),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": None,
                         "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else "fallback 6.65 TB/s", "alg_bytes_per_launch": int(alg)},
            "gpu_launches": args.images_per_step * args.steps, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse_args()
    if args.launches_only > 0:
        return launches_only(args.launches_only, args.workload)
    if args.workload in ("erode", "median3", "median5"):
        return run_neighbourhood_op(args)
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "sep_sweep":
        return run_sep_sweep(args)
    if args.workload == "filter2d":
        return run_filter2d(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
