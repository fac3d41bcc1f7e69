#!/usr/bin/env python3
"""Benchmark: 1080p YUV420P16 DFTTest frames/s on B200.

Workload (the production-size configuration): YUV420P16, 1920x1080 luma and
960x540 chroma, 64 frames per GPU, sbsize 16 / sosize 12 / tbsize 3,
ftype 0 (Wiener), frequency-dependent sigma from slocation (4 knots, 12 at DC
to 4 at Nyquist), zero-mean, all three planes.  Synthetic input: seeded
drifting sinusoids + Gaussian noise (sigma 4*257 codes) + 1% salt-and-pepper.

A step filters the whole 64-frame clip (192 planes) once.
* value: device-resident path (dfttest2_b200_process_planes, inputs already
  in HBM, 398 MB > L2), CUDA events on the launching stream, max over ranks.
* e2e:   the C ABI's host path (dfttest2_b200_process_clip_host) from pinned
  host memory, uploads and downloads inside the timed region.
* roofline: FP32 CUDA-core bound; algorithmic FLOPs per block from the
  reference codelet counts (26,385 for 16x16x3) over the measured step time,
  against FP32 SGEMM throughput measured in the same run.
* cpu_baseline: the reference's CPU math (oracle/_ref) on host threads over a
  bounded sample of the same workload (N=1, rank 0).

``--impl reference`` times only the reference CPU implementation (rank 0).
Multi-GPU (torchrun): each rank filters its own 64 frames of a longer clip
(frame-range sharding, no data-path collective), scaling "weak".
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "vs-dfttest2_b200")]

import numpy as np  # noqa: E402

FRAMES = 64
W, H = 1920, 1080
SLOCATION = [0.0, 12.0, 1 / 3, 28 / 3, 2 / 3, 20 / 3, 1.0, 4.0]
FLOP_PER_BLOCK = {1: 9473, 3: 26385, 5: 47329, 7: 74033}  # B = 16, reference codelet counts
METRIC = "1080p YUV420P16 frames/s (DFTTest sbsize16 sosize12 tbsize3, all planes)"
# DRAM bytes (read + write) of the unit kernel per 1080p YUV420P16 frame, from one ncu capture of a
# 24-frame launch of this workload; traffic grows with the frames processed
DRAM_BYTES_PER_FRAME = 18_942_637


def workload_args():
    from dfttest2_b200.frontend import DFTTest, plugin_arguments
    import dfttest2_b200.frontend as fe

    # run the user-level translation (DFTTest -> DFTTest2) to get the plugin arguments
    captured = {}

    def grab(**k):
        captured.update(k)

    real = fe.DFTTest2
    fe.DFTTest2 = grab
    try:
        from dfttest2_b200 import YUV420P16, Clip
        dummy = Clip([np.zeros((1, H, W), np.uint16), np.zeros((1, H // 2, W // 2), np.uint16),
                      np.zeros((1, H // 2, W // 2), np.uint16)], YUV420P16)
        DFTTest(dummy, ftype=0, sbsize=16, sosize=12, tbsize=3, slocation=SLOCATION)
    finally:
        fe.DFTTest2 = real
    for k in ("clip", "planes", "backend"):
        captured.pop(k)
    return plugin_arguments(**captured)


def workload_config(frames_per_gpu, world, bytes_in):
    """The `config` object both arms print (same workload, same keys)."""
    frame_bytes = (W * H + 2 * (W // 2) * (H // 2)) * 2
    return {"workload": "YUV420P16 1920x1080 + 960x540 chroma, 64 frames/GPU, sbsize16 sosize12 tbsize3, "
                        "ftype0, slocation 12->4, zero-mean, all planes",
            "frames_per_gpu": frames_per_gpu,
            "l2": f"inputs {(bytes_in or frame_bytes * frames_per_gpu) / 1e6:.0f} MB/GPU > 126 MB L2, no flush",
            "parallelism": f"frame shards x{world}"}


def blocks_per_frame():
    from dfttest2_b200.clip import YUV420P16, plane_dims

    def pn(n):
        B, S = 16, 4
        ps = n + ((n % B) and B - n % B) + 2 * max(B - S, S)
        return (ps - B) // S + 1

    total = 0
    for p in range(3):
        pw, ph = plane_dims(YUV420P16, W, H, p)
        total += pn(pw) * pn(ph)
    return total


def make_planes(rank: int, frames: int, radius: int):
    """Synthetic YUV420P16 planes for this rank's frame range plus halo."""
    from dfttest2_b200 import YUV420P16
    from dfttest2_b200.synth import make_clip

    noisy, _ = make_clip(YUV420P16, W, H, frames, seed=1000 + rank, noise_sigma=4 * 257 / 65535, salt_pepper=0.01)
    return noisy.planes


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[4:8]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def fp32_peak_tflops(device) -> float:
    """FP32 (non-tensor) GEMM throughput measured now with cuBLAS SGEMM."""
    import torch

    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        torch.backends.cuda.matmul.fp32_precision = "ieee"
    except AttributeError:
        pass
    n = 8192
    a = torch.randn(n, n, device=device)
    b = torch.randn(n, n, device=device)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    torch.cuda.empty_cache()
    return best


def measured_peaks():
    """Peaks measured on this pool's B200s (MEASURED_PEAKS.json, written next
    to this file by the machine's set-up); without that file, the pool's
    earlier measurement (6.65 TB/s copy, 1.59 PFLOP/s bf16), marked as such."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
            d.setdefault("source", "measured (MEASURED_PEAKS.json)")
            return d
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback (no MEASURED_PEAKS.json)"}


def cpu_reference_fps(args, planes, seconds_target=15.0, threads=None):
    """Reference CPU math (oracle/_ref, else the FP64 port) over a bounded
    sample of output frames, frames in parallel over host threads."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle as O

    threads = threads or os.cpu_count() or 1
    kind = "reference" if O.ref_available() else "port"
    full = dict(args)
    isa = O.ref_isa() if kind == "reference" else "scalar C (FP64 port)"

    def one(n):
        for p in range(3):
            fr = O.clip_frames(planes[p], n, args["radius"])
            if kind == "reference":
                O.ref_plane(fr, full, 16)
            else:
                O.fp64_plane(fr, full, 16)

    nf = planes[0].shape[0]
    t0 = time.perf_counter()
    one(0)
    single = time.perf_counter() - t0
    # frames per batch so that the sample takes about seconds_target
    sample = max(threads, int(seconds_target / max(single, 1e-3) * threads))
    sample = min(sample, 4 * threads, 256)
    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(one, [i % nf for i in range(sample)]))
    dt = time.perf_counter() - t0
    return {"value": sample / dt, "unit": "frames/s", "cores": threads, "kind": kind, "isa": isa,
            "cpu_model": O.cpu_model(),
            "sample": f"{sample} output frames (3 planes each) of the 1080p YUV420P16 workload, "
                      f"frames in parallel over {threads} threads"}


def run_reference(opts, rank, world):
    if rank != 0:
        return
    args = workload_args()
    planes = make_planes(0, 8, args["radius"])
    for _ in range(opts.warmup):  # pages, caches and thread pool warmed on a short sample
        cpu_reference_fps(args, planes, seconds_target=1.0)
    vals = []
    base = None
    for _ in range(opts.steps):
        base = cpu_reference_fps(args, planes, seconds_target=max(2.0, 60.0 / max(opts.steps, 1)))
        vals.append(base["value"])
    v = statistics.median(vals)
    base["value"] = v
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "frames/s", "n_gpus": world,
        "steps": opts.steps, "warmup": opts.warmup, "ms_per_step": 1000.0 / v, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(FRAMES, world, 0),
        "cpu_baseline": base, "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0,
                                       "d2h_bytes_per_step": 0}}))


def run_batch(opts):
    """Prints the multi-clip batching workload's line (batch_measure)."""
    print(json.dumps(batch_measure(opts.seed, opts.workload == "batch_small", opts.steps, opts.warmup)))


def batch_measure(seed, small, steps, warmup):
    """Multi-clip batching workload: 32 seeded clips of mixed resolution,
    length, format and block parameters (synth.batch_specs), filtered by one
    graph launch of a tuned batch vs 32 sequential plain calls (one
    dfttest2_b200_process_planes call per clip, all its frames and planes).
    Inputs are built on the device; both arms write separate outputs, which
    must agree (integers within 1 LSB, float within 2e-5)."""
    import ctypes

    import torch

    from types import SimpleNamespace
    opts = SimpleNamespace(seed=seed, workload="batch_small" if small else "batch", steps=steps, warmup=warmup)

    from dfttest2_b200 import _lib, frontend as fe, synth
    from dfttest2_b200.autograd import frame_planes
    from dfttest2_b200.batch import Batch
    from dfttest2_b200.plugin import Filter

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    lib = _lib.load()
    specs = synth.batch_specs(opts.seed, small=opts.workload == "batch_small")
    items, calls, pairs = [], [], []
    total_frames = 0
    flops = 0.0
    for sp in specs:
        args = fe.plugin_arguments(ftype=sp["ftype"], sigma=sp["sigma"], sbsize=sp["sbsize"], sosize=sp["sosize"],
                                   tbsize=sp["tbsize"])
        flt = Filter(device_id=0, **args)
        fmt = sp["fmt"]
        planes = synth.make_clip_device(fmt, sp["width"], sp["height"], sp["frames"], sp["seed"], 0.03, device)
        arrs = []
        for src in planes:
            ob, os_ = torch.empty_like(src), torch.empty_like(src)
            items.append((flt, src, ob, fmt.sample_type, fmt.bits_per_sample))
            arrs.append(frame_planes(src[None], os_[None], args["radius"]))
            pairs.append((ob, os_, fmt.sample_type))
            B, S = args["block_size"], args["block_step"]
            pn = [(n + ((B - n % B) if n % B else 0) + 2 * max(B - S, S) - B) // S + 1 for n in src.shape[1:]]
            T = 2 * args["radius"] + 1
            flops += src.shape[0] * pn[0] * pn[1] * 2.5 * B * B * T * np.log2(B * B * T) * 2
        arr = (_lib.Plane * sum(len(a) for a in arrs))()
        k = 0
        for a in arrs:
            for pl in a:
                arr[k] = pl
                k += 1
        calls.append((flt, arr, k, fmt.sample_type, fmt.bits_per_sample))
        total_frames += sp["frames"]
    stream = torch.cuda.current_stream(device)

    def sequential():
        for flt, arr, k, st, bits in calls:
            _lib.check(lib.dfttest2_b200_process_planes(flt.handle, arr, k, st, bits, ctypes.c_void_p(stream.cuda_stream)))

    t0 = time.perf_counter()
    batch = Batch(items, tune=True)
    tune_s = time.perf_counter() - t0
    launches, desc = batch.describe()

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        out = []
        for _ in range(reps):
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1))
        return statistics.median(out)

    for _ in range(opts.warmup):
        sequential()
        batch.run()
    clocks = ClockSampler(0).__enter__()
    time.sleep(0.3)
    seq_ms = timed(sequential, opts.steps)
    bat_ms = timed(batch.run, opts.steps)
    time.sleep(0.2)
    clocks.__exit__(None, None, None)
    worst_int, worst_float = 0, 0.0
    for ob, os_, st in pairs:
        a, b2 = (x.to(torch.int32) & 0xFFFF if x.dtype == torch.int16 else x for x in (ob, os_))
        d = (a.to(torch.float32) - b2.to(torch.float32)).abs().max().item()
        if st == 1:
            worst_float = max(worst_float, d)
        else:
            worst_int = max(worst_int, d)
    result = {
        "metric": "32-clip mixed batch, frames/s (all clips, one graph launch)", "value": total_frames / (bat_ms * 1e-3),
        "unit": "frames/s", "n_gpus": 1, "steps": opts.steps, "warmup": opts.warmup, "ms_per_step": bat_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded sinusoids + gaussian 0.03, built on the device)",
        "config": {"workload": f"32 clips (synth.batch_specs seed {opts.seed}"
                               f"{', small' if opts.workload == 'batch_small' else ''}): "
                               f"{'640x360' if opts.workload == 'batch_small' else '640x360..3840x2160'}, 4..32 frames, "
                               "GRAYS/YUV420P8/YUV420P16, sbsize 8/16/32 sosize 3/4, tbsize 1/3/5, ftype 0/1",
                   "frames": total_frames, "l2": "inputs of several GB > L2, no flush"},
        "sequential_ms": seq_ms, "batch_ms": bat_ms, "speedup": seq_ms / bat_ms, "tune_seconds": tune_s,
        "gpu_launches": launches, "groups": desc.strip().split("\n"),
        "parity": {"max_abs_int_lsb": worst_int, "max_abs_float": worst_float},
        "fft_flop_estimate_tflops": flops / (bat_ms * 1e-3) / 1e12,
        "clocks": clocks.summary(),
    }
    batch.close()
    for flt, *_ in calls:
        flt.close()
    return result


def autograd_measure(steps=10, warmup=3):
    """Differentiation workload: 8 GRAYS float32 clips of 256x256 x 9 frames
    (seeded sinusoids; noisy = clean + Gaussian noise, sigma ~ U[0.02, 0.08]
    per clip), Wiener, sbsize 16 / sosize 12 / tbsize 3, learnable sigma array
    (3, 16, 9) initialised to 0.05, MSE to the clean clips.  Times the forward
    pass alone and forward + backward (adjoint kernel) with CUDA events."""
    import torch

    from dfttest2_b200 import GRAYS
    from dfttest2_b200.autograd import DFTTestModule
    from dfttest2_b200.frontend import plugin_arguments
    from dfttest2_b200.synth import make_clip

    device = torch.device("cuda", 0)
    rng = np.random.default_rng(4)
    noisy, clean = [], []
    for c in range(8):
        _, cl = make_clip(GRAYS, 256, 256, 9, seed=400 + c, noise_sigma=0.0)
        x = cl.planes[0]
        clean.append(x)
        noisy.append(x + rng.standard_normal(x.shape).astype(np.float32) * np.float32(rng.uniform(0.02, 0.08)))
    x = torch.from_numpy(np.stack(noisy)).to(device)
    target = torch.from_numpy(np.stack(clean)).to(device)
    mod = DFTTestModule(plugin_arguments(ftype=0, sbsize=16, sosize=12, tbsize=3), 0.05, device="cuda:0")
    stream = torch.cuda.current_stream(device)

    def fwd():
        with torch.no_grad():
            return mod(x)

    def fwd_bwd():
        xg = x.detach().requires_grad_(True)
        loss = (mod(xg) - target).pow(2).mean()
        loss.backward()
        return loss

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    f_ms = timed(fwd)
    fb_ms = timed(fwd_bwd)
    mod.flt.close()
    return {"fwd_ms": f_ms, "fwd_bwd_ms": fb_ms, "ratio": fb_ms / f_ms, "steps": steps,
            "workload": "8 GRAYS float32 clips 256x256 x 9 frames, sbsize16 sosize12 tbsize3, learnable sigma "
                        "(3,16,9) = 0.05, MSE to clean; forward vs forward + backward (adjoint kernel)"}


def strip_form_flops(planes_hw, frames, B=16, S=4, T=3):
    """Tensor-core FLOPs (2 M N K per MMA, as issued: padded rows and the
    Toeplitz columns included) of one launch of the strip form over `frames`
    frames of planes of sizes `planes_hw`: per block row of a strip of up to
    16 blocks, the y products (T planes x 3 split products, 128 x 16 x 16),
    the x products (per 8-block tile, cos and sin parts, ceil((16 + 7 S) / 16)
    K steps x 3, 128 x 16T x 16) and the inverse-y products (per tile, 3,
    128 x 16 x 16)."""
    def pad_num(n):
        pad = n + ((B - n % B) if n % B else 0) + 2 * max(B - S, S)
        return (pad - B) // S + 1

    nks = (B + 7 * S + 15) // 16
    per_mma = lambda n: 2 * 128 * n * 16
    total = 0
    for h, w in planes_hw:
        pnx, pny = pad_num(w), pad_num(h)
        nsx = (pnx + 15) // 16
        tiles = 0
        for sx in range(nsx):
            nb = (sx + 1) * pnx // nsx - sx * pnx // nsx
            tiles += 1 if nb <= 8 else 2
        row = T * 3 * per_mma(16) * nsx + tiles * (2 * nks * 3 * per_mma(16 * T) + 3 * per_mma(16))
        total += row * pny
    return total * frames


def reference_parity(args, host_planes, outs, frames, r):
    """Max LSB and exact-match fraction of device outputs against the
    reference's CPU math (oracle/_ref) on sampled output frames, all planes.
    `outs` are (N, H, W) int16 CUDA tensors indexed like host_planes' output
    frames (output frame n reads host frames n-r..n+r)."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle as O

    if not O.ref_available():
        return None
    jobs = [(p, n) for p in range(3) for n in frames]

    def one(job):
        p, n = job
        return O.ref_plane(O.clip_frames(host_planes[p], n, r), args, 16)

    with ThreadPoolExecutor(min(len(jobs), os.cpu_count() or 1)) as ex:
        refs = list(ex.map(one, jobs))
    worst, exact, total = 0, 0, 0
    for (p, n), ref in zip(jobs, refs):
        got = outs[p][n].cpu().numpy().view(np.uint16)
        d = np.abs(got.astype(np.int64) - ref.astype(np.int64))
        worst = max(worst, int(d.max()))
        exact += int((d == 0).sum())
        total += d.size
    return {"max_lsb": worst, "exact": exact / total, "frames": list(frames), "checker": "oracle/_ref (reference CPU math)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=FRAMES)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-peak", action="store_true", help="skip the SGEMM peak measurement (profiling runs)")
    ap.add_argument("--workload", default="yuv1080p", choices=["yuv1080p", "batch", "batch_small", "autograd"],
                    help="batch: the 32-clip multi-clip batching workload (one GPU); batch_small: the same with "
                         "640x360 clips only; autograd: forward vs forward + backward of the differentiable path")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--fbf-frames", type=int, default=32,
                    help="frames filtered frame by frame through the cached per-plane host path (0 skips)")
    ap.add_argument("--tc-steps", type=int, default=10,
                    help="steps timed for each tensor-core precision mode (0 skips the comparison)")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "tc_fp16x3", "tc_bf16x3", "tc_tf32", "tc_bf16"],
                    help="arithmetic of the timed steps (profiling runs of the tensor-core form)")
    ap.add_argument("--extras", type=int, default=1,
                    help="0 skips the parity, differentiation and batching keys (profiling runs)")
    opts = ap.parse_args()
    if opts.workload == "autograd":
        if opts.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no gradient"}))
            return
        print(json.dumps(autograd_measure(opts.steps, opts.warmup)))
        return
    if opts.workload in ("batch", "batch_small"):
        if opts.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no multi-clip batch"}))
            return
        return run_batch(opts)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch

    pg = False
    if world > 1:
        import datetime

        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = True
    if opts.impl == "reference":
        run_reference(opts, rank, world)
        if pg:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    from dfttest2_b200.plugin import Filter
    from dfttest2_b200.shard import frame_shard, max_over_ranks

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    args = workload_args()
    r = args["radius"]
    nf = opts.frames
    # this rank's output frames [lo, hi) of a world*nf-frame clip and the input frames it needs
    lo, hi, in_lo, in_hi = frame_shard(world * nf, rank, world, r)
    host_planes = make_planes(rank, in_hi - in_lo, r)
    dev_in = [torch.from_numpy(p.view(np.int16)).to(device) for p in host_planes]
    dev_out = [torch.empty((hi - lo,) + tuple(p.shape[1:]), dtype=torch.int16, device=device) for p in host_planes]
    flt = Filter(device_id=local, **args)
    planes = []
    total_clip = world * nf
    for p in range(3):
        src, dst = dev_in[p], dev_out[p]
        ph, pw = src.shape[1], src.shape[2]
        for n in range(lo, hi):
            ptrs = [src[min(max(n - r + t, 0), total_clip - 1) - in_lo].data_ptr() for t in range(2 * r + 1)]
            planes.append(dict(src=ptrs, src_stride=pw * 2, dst=dst[n - lo].data_ptr(), dst_stride=pw * 2,
                               width=pw, height=ph))
    stream = torch.cuda.current_stream(device)

    def step():
        flt.process_planes_device(planes, 0, 16, stream.cuda_stream)

    if opts.precision != "fp32":
        flt.set_precision(opts.precision)

    clocks = ClockSampler(local).__enter__()  # started early: nvidia-smi takes a moment to produce samples
    for _ in range(opts.warmup):
        step()
    torch.cuda.synchronize()
    time.sleep(0.5)
    if pg:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n_before = len(clocks.lines)
    start.record(stream)
    for _ in range(opts.steps):
        step()
    stop.record(stream)
    torch.cuda.synchronize()
    time.sleep(0.2)
    clocks.__exit__(None, None, None)
    clocks.lines = clocks.lines[n_before:] or clocks.lines
    ms = start.elapsed_time(stop)
    if pg:
        torch.distributed.barrier()
    ms = max_over_ranks(ms, pg)
    frames_done = world * (hi - lo) * opts.steps
    value = frames_done / (ms * 1e-3)
    ms_per_step = ms / opts.steps
    flt.check()  # raises if a kernel reported a failure during the timed steps
    extras = opts.extras and world == 1 and opts.precision == "fp32"
    # parity of the timed outputs against the reference's CPU math on two sampled frames
    sample_frames = (0, (hi - lo) // 2 + 1)
    parity = {}
    if extras:
        parity["fp32"] = reference_parity(args, host_planes, dev_out, sample_frames, r)

    # ---- tensor-core form of the transforms on the same workload, against the plain FP32 output
    tc_results = {}
    if opts.tc_steps > 0 and opts.precision == "fp32":
        plain_out = [o.clone() for o in dev_out]
        for mode in ("tc_fp16x3", "tc_bf16x3", "tc_tf32"):
            flt.set_precision(mode)
            for _ in range(2):
                step()
            torch.cuda.synchronize()
            flt.check()
            if extras and mode in ("tc_fp16x3", "tc_bf16x3"):
                parity[mode] = reference_parity(args, host_planes, dev_out, sample_frames, r)
            t_start, t_stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t_start.record(stream)
            for _ in range(opts.tc_steps):
                step()
            t_stop.record(stream)
            torch.cuda.synchronize()
            ms_tc = max_over_ranks(t_start.elapsed_time(t_stop), pg) / opts.tc_steps
            worst, exact, total = 0, 0, 0
            for a_, b_ in zip(dev_out, plain_out):
                d = ((a_.to(torch.int32) & 0xFFFF) - (b_.to(torch.int32) & 0xFFFF)).abs()
                worst = max(worst, int(d.max().item()))
                exact += int((d == 0).sum().item())
                total += d.numel()
            tc_results[mode] = {"value": world * (hi - lo) / (ms_tc * 1e-3), "unit": "frames/s", "ms_per_step": ms_tc,
                                "speedup_vs_fp32": ms_per_step / ms_tc, "max_lsb_vs_fp32": worst,
                                "exact_vs_fp32": exact / max(total, 1), "steps": opts.tc_steps}
            if mode in ("tc_fp16x3", "tc_bf16x3"):
                # the strip form's tensor-core work against the measured dense 16-bit peak
                fl = strip_form_flops([tuple(p.shape[1:]) for p in host_planes], hi - lo)
                peak_tc = measured_peaks().get("bf16_tflops")
                tc_results[mode]["tensor"] = {
                    "tflop_per_step": fl / 1e12, "achieved_tflops": fl / (ms_tc * 1e-3) / 1e12,
                    "peak_tflops": peak_tc, "frac": (fl / (ms_tc * 1e-3) / 1e12 / peak_tc) if peak_tc else None,
                    "peak_source": measured_peaks().get("source") + ", bf16_tflops burst (fp16 runs at the same dense rate)",
                    "note": "FLOPs as issued (2 M N K per tcgen05.mma, padded rows and Toeplitz columns included)"}
        flt.set_precision("fp32")

    # ---- end to end through the C ABI host path (pinned host buffers)
    pinned_in = [torch.from_numpy(p.view(np.int16)).pin_memory() for p in host_planes]
    pinned_out = [torch.empty((in_hi - in_lo,) + tuple(p.shape[1:]), dtype=torch.int16).pin_memory()
                  for p in host_planes]
    _lib = __import__("dfttest2_b200._lib", fromlist=["load"])
    lib = _lib.load()

    hp = (_lib.HostPlane * 3)()
    for p in range(3):
        src, dst = pinned_in[p], pinned_out[p]
        n, ph, pw = src.shape
        hp[p].src, hp[p].src_stride, hp[p].src_frame_bytes = src.data_ptr(), pw * 2, ph * pw * 2
        hp[p].dst, hp[p].dst_stride, hp[p].dst_frame_bytes = dst.data_ptr(), pw * 2, ph * pw * 2
        hp[p].width, hp[p].height = pw, ph

    def e2e_step():
        # the three planes through one host pipeline (one call per step)
        rc = lib.dfttest2_b200_process_clip_planes_host(flt.handle, hp, 3, pinned_in[0].shape[0], 0, 16)
        if rc:
            raise RuntimeError(lib.dfttest2_b200_last_error().decode())

    if opts.e2e_steps > 0:
        e2e_step()
    if pg:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(opts.e2e_steps):
        e2e_step()
    e2e_s = max(max_over_ranks(time.perf_counter() - t0, pg), 1e-9)
    e2e_frames = world * (in_hi - in_lo) * opts.e2e_steps
    bytes_in = sum(p.nbytes for p in host_planes)

    # kernels per step: the unit kernel, plus the fix-up kernel unless every unit is a
    # full-height strip (strips of 16 blocks reach 4 x SMs units), when seams are summed in-kernel
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    pn = [(n + ((16 - n % 16) if n % 16 else 0) + 24 - 16) // 4 + 1 for n in (W, W // 2)]
    strips = (hi - lo) * ((pn[0] + 15) // 16 + 2 * ((pn[1] + 15) // 16))
    launches_per_step = 1 if strips >= 4 * sms else 2

    # ---- frame by frame, as a VapourSynth GetFrame drives the library: one cached per-plane
    # host call per plane of each output frame, source planes cached on the device by frame number
    fbf = {}
    nfb = min(opts.fbf_frames, (in_hi - in_lo) // 2)  # the other half of the clip warms the cache up
    if nfb > 0 and world == 1:
        import ctypes
        from concurrent.futures import ThreadPoolExecutor

        fbf_flt = Filter(device_id=local, num_streams=4, **args)
        reqs = []
        for n in range(2 * nfb):
            for p in range(3):
                src = host_planes[p]
                N, ph, pw = src.shape
                pl = _lib.Plane()
                ids = [min(max(n - r + t, 0), N - 1) for t in range(2 * r + 1)]
                for t, k in enumerate(ids):
                    pl.src[t] = src[k].ctypes.data
                # touched once, as the pooled frames of a frame server are (a first write
                # into fresh pages would time page faults, not the library)
                out = np.zeros((ph, pw), src.dtype)
                out.fill(1)
                pl.src_stride = pw * 2
                pl.dst = out.ctypes.data
                pl.dst_stride = pw * 2
                pl.width, pl.height = pw, ph
                reqs.append((n, pl, (ctypes.c_int * len(ids))(*ids), p, out))

        pidx = (ctypes.c_int * 3)(0, 1, 2)
        frame_planes_arr = []
        for n in range(2 * nfb):
            arr = (_lib.Plane * 3)()
            for k, (_, pl, _, _, _) in enumerate(reqs[3 * n:3 * n + 3]):
                arr[k] = pl
            frame_planes_arr.append(arr)

        def frame(n, cached=True):
            if cached:  # the three planes of the frame in one call, sources cached on the device
                rc = lib.dfttest2_b200_process_frame_host_cached(fbf_flt.handle, frame_planes_arr[n], 3, pidx,
                                                                 reqs[3 * n][2], 0, 16)
                return lib.dfttest2_b200_last_error().decode() if rc else ""
            for rn, pl, ids, p, _ in reqs[3 * n:3 * n + 3]:
                # every call uploads its 2r+1 source planes, as the reference does per output frame
                rc = lib.dfttest2_b200_process_plane_host(fbf_flt.handle, ctypes.byref(pl), 0, 16)
                if rc:
                    return lib.dfttest2_b200_last_error().decode()
            return ""

        uncached = {}
        for threads in (1, 4):
            for cached, into in ((True, fbf), (False, uncached)):
                with ThreadPoolExecutor(threads) as pool:
                    # warm-up on frames nfb .. 2 nfb - 1: allocations, the cache's working set
                    list(pool.map(lambda k: frame(k, cached), range(nfb, 2 * nfb)))
                    t0 = time.perf_counter()
                    errs = [e for e in pool.map(lambda k: frame(k, cached), range(nfb)) if e]
                    dt = time.perf_counter() - t0
                if errs:
                    raise RuntimeError(errs[0])
                into[f"threads_{threads}"] = nfb / dt
        fbf_flt.close()
        fbf = {"value_by_threads": fbf, "uncached_by_threads": uncached, "unit": "frames/s", "frames": nfb,
               "path": "dfttest2_b200_process_frame_host_cached, one call per frame for its three planes (pageable "
                       "host frames), source planes cached on the device by frame number; uncached = "
                       "dfttest2_b200_process_plane_host (2r+1 source planes uploaded per call)"}

    # ---- roofline
    blocks = blocks_per_frame() * (hi - lo)
    flops_step = blocks * FLOP_PER_BLOCK[2 * r + 1]
    achieved = flops_step / (ms_per_step * 1e-3) / 1e12
    peak = float("nan") if opts.no_peak else fp32_peak_tflops(device)
    algo_bytes = sum(p.nbytes for p in host_planes) / (in_hi - in_lo) * (hi - lo) * 2

    result = {
        "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": opts.steps,
        "warmup": opts.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded sinusoids + gaussian + 1% salt-pepper)",
        "config": workload_config(hi - lo, world, bytes_in),
        "e2e": {"value": e2e_frames / e2e_s, "unit": "frames/s", "h2d_bytes_per_step": bytes_in,
                "d2h_bytes_per_step": bytes_in, "path": "dfttest2_b200_process_clip_planes_host (3 planes, one pipeline), pinned host memory"},
        "gpu_launches": launches_per_step * opts.steps,
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": DRAM_BYTES_PER_FRAME * (hi - lo),
                     "traffic_note": "dram__bytes_read.sum + dram__bytes_write.sum per launch, scaled from an ncu "
                                     "capture of a 24-frame launch",
                     "peak_source": "cuBLAS FP32 SGEMM (TF32 off) measured in this run; nominal 148 SM x 128 x 2 x "
                                    "1.965 GHz = 74.4",
                     "flop_per_step": flops_step, "hbm_algorithmic_gbs": algo_bytes / (ms_per_step * 1e-3) / 1e9,
                     "hbm_peak_gbs": measured_peaks().get("hbm_gbs"),
                     "hbm_peak_source": measured_peaks().get("source")},
        "clocks": clocks.summary(),
        "tc": tc_results,
        "parity": parity or None,
        "e2e_frame_by_frame": fbf or None,
    }
    if extras:
        result["fwd_bwd_over_fwd"] = autograd_measure()
        bm = batch_measure(0, True, 5, 2)
        result["batch_speedup"] = {"value": bm["speedup"], "sequential_ms": bm["sequential_ms"],
                                   "batch_ms": bm["batch_ms"], "gpu_launches": bm["gpu_launches"],
                                   "parity": bm["parity"], "workload": bm["config"]["workload"]}
    if world == 1 and rank == 0 and not opts.no_cpu_baseline:
        result["cpu_baseline"] = cpu_reference_fps(args, host_planes)
    flt.close()
    if rank == 0:
        print(json.dumps(result))
    if pg:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
