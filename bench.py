#!/usr/bin/env python
"""ELAS stereo benchmark on B200.

Workload (one "step" = one stereo pair through the whole hot path:
descriptors, support matching, Delaunay, plane prior, dense matching of both
views, L/R check, post-filters): a seeded synthetic 1242x375 pair with
disparity range 0-255 (the KITTI-shaped configuration).  `value` is pairs/s
with the inputs resident in HBM, timed with CUDA events on the launch stream,
L2 flushed (256 MiB write) before every step outside the timed events.
`e2e` is the same metric through the C-ABI host-buffer call (pinned host
inputs, host->device copy, pipeline, device->host copy of both maps).

Multi-GPU: pairs are independent, so N ranks run N replicas on their own
pairs (weak scaling, no collective on the data path); the timed region is
bracketed by barriers and the max over ranks is reported.

`--impl reference` times the CPU implementation of the path (the oracle's
restatement of the reference kernels with the reference's own Triangle) on
the host cores for the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "cuda-stereo-matching_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))

import elas_b200 as eb  # noqa: E402

METRIC = "pairs/s, ELAS 1242x375 disparity 0-255"
PRESET = 1
L2_FLUSH_BYTES = 256 << 20


def peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name):
    """dram bytes per launch recorded from an ncu capture (profiles/<name>.txt)."""
    path = os.path.join(REPO, "profiles", name + ".txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("traffic_bytes_per_launch:"):
            return float(line.split(":")[1])
    return None


class ClockSampler:
    """SM clock and throttle reasons sampled during a timed region.  NVML is
    polled from a thread about every millisecond (a 20-step region of a
    1242x375 pair lasts about 10 ms); nvidia-smi, whose period is 100 ms, is
    the fallback.  Read-only: no clock or other setting is changed."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, index):
        self.index = index
        self.samples = []          # (sm_mhz, reasons mask)
        self.max_mhz = None
        self.nvml = None
        self.proc = None
        self.lines = []
        self._stop = threading.Event()
        self.thread = None

    def start(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self.nvml = (pynvml, h)
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            fields = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                      "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                      "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + fields,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _poll(self):
        pynvml, h = self.nvml
        while not self._stop.is_set():
            try:
                mhz = float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                mask = int(pynvml.nvmlDeviceGetCurrentClocksEventReasons(h))
                self.samples.append((mhz, mask))
            except Exception:
                break
            time.sleep(0.001)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        self._stop.set()
        if self.nvml:
            self.thread.join(timeout=5)
            pynvml = self.nvml[0]
            reasons = set()
            for _, mask in self.samples:
                for name, attr in self.REASONS:
                    if mask & getattr(pynvml, attr, 0):
                        reasons.add(name)
            sm = [m for m, _ in self.samples]
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                    "reasons": sorted(reasons), "samples": len(sm), "source": "nvml, ~1 ms polling"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no clock source"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = [n for n, _ in self.REASONS]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi, 100 ms period"}


def replica_seed(rank):
    """Seed of the pair rank `rank` processes: every replica works on its own pair."""
    return 1000 + rank


def aggregate_rate(units_per_rank, max_seconds, world):
    """Whole-job throughput: the units all ranks processed over the slowest rank's time."""
    return units_per_rank * world / max_seconds


def dist_setup(args, backend=None):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = backend or ("nccl" if args.impl == "ours" else "gloo")
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(x, world, device=None):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def quality(D, gt):
    valid_gt = np.isfinite(gt) & (gt > 0)
    bad = (np.abs(D - gt) > 2) | (D < 0)
    return {"bad2px": float(bad[valid_gt].mean()), "density": float((D >= 0).mean())}


def time_pipeline(e, L, R, steps, warmup, torch, flush, stream, stage_steps=5):
    """Device-resident timing: per step flush L2, then CUDA events around one
    pair.  The timed steps run without the per-stage event marks (recording
    them inside the pipeline costs time); the stage breakdown comes from a
    separate pass of `stage_steps` pairs with the marks on."""
    H, W = L.shape
    dl = torch.from_numpy(L).cuda()
    dr = torch.from_numpy(R).cuda()
    o1 = torch.empty((H, W), dtype=torch.float32, device="cuda")
    o2 = torch.empty_like(o1)
    s = stream.cuda_stream
    e.set_timing(False)
    for _ in range(warmup):
        flush.zero_()
        e.process_device(dl.data_ptr(), dr.data_ptr(), o1.data_ptr(), o2.data_ptr(), W, H, stream=s)
    torch.cuda.synchronize()
    start = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    end = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    l0 = e.launch_count
    for k in range(steps):
        flush.zero_()
        start[k].record(stream)
        e.process_device(dl.data_ptr(), dr.data_ptr(), o1.data_ptr(), o2.data_ptr(), W, H, stream=s)
        end[k].record(stream)
    torch.cuda.synchronize()
    launches = e.launch_count - l0
    total_ms = sum(a.elapsed_time(b) for a, b in zip(start, end))
    # stage breakdown (diagnostic, outside the timed steps)
    e.set_timing(True)
    stage_ms = {k: 0.0 for k in e.TIME_STAGES}
    for k in range(stage_steps + 2):
        flush.zero_()
        e.process_device(dl.data_ptr(), dr.data_ptr(), o1.data_ptr(), o2.data_ptr(), W, H, stream=s)
        t = e.timing()                        # waits for this pair
        if k >= 2:                            # the first calls with the marks run eagerly and capture
            for name, ms in t.items():
                stage_ms[name] += ms / stage_steps
    e.set_timing(False)
    torch.cuda.synchronize()
    return total_ms, stage_ms, launches, o1.cpu().numpy()


def time_e2e(e, L, R, steps, torch, flush, warmup=3):
    """Through the host-buffer C-ABI call from pinned memory (blocking call).
    The first calls size the workspace and capture the pair's graph; they
    run before the timed calls."""
    H, W = L.shape
    pl = torch.from_numpy(L).pin_memory()
    pr = torch.from_numpy(R).pin_memory()
    d1 = torch.empty((H, W), dtype=torch.float32).pin_memory()
    d2 = torch.empty_like(d1).pin_memory()
    dims = np.array([W, H, W], np.int32)
    lib = eb.library()
    import ctypes

    def call():
        rc = lib.elas_b200_process(e._h, ctypes.c_void_p(pl.data_ptr()), ctypes.c_void_p(pr.data_ptr()),
                                   ctypes.c_void_p(d1.data_ptr()), ctypes.c_void_p(d2.data_ptr()),
                                   dims.ctypes.data_as(ctypes.c_void_p), None)
        e._check(rc)

    for _ in range(max(3, warmup)):
        call()
    total = 0.0
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        call()
        total += time.perf_counter() - t0
    return total, {"h2d_bytes_per_step": 2 * W * H, "d2h_bytes_per_step": 2 * W * H * 4}


def cpu_baseline(L, R, p, budget_s=12.0):
    import oracle

    threads = os.cpu_count() or 1
    oracle.process(L, R, p, threads=threads)   # warm-up
    n, t0 = 0, time.perf_counter()
    while True:
        oracle.process(L, R, p, threads=threads)
        n += 1
        el = time.perf_counter() - t0
        if el >= budget_s or n >= 200:
            break
    return {"value": n / el, "unit": "pairs/s", "cores": threads, "kind": "port",
            "sample": f"{n} full {L.shape[1]}x{L.shape[0]} pairs (disparity 0-{p.disp_max}) through the oracle "
                      f"(C++ restatement of the reference kernels + the reference's Triangle), {threads} threads"}


def reference_gpu(L, R, runs=5):
    """The reference's own Elas::process -- its CUDA kernels built for
    sm_100a from the reference tree into oracle/_ref, host buffers, its
    per-call allocations and CPU Triangle -- timed on the same GPU: a
    comparator beside the CPU baseline, not the target.  Its kernels are
    compiled with the disparity range 0-255 (KernelsCommon.h)."""
    import ctypes

    import oracle

    if not oracle.have_ref_elas():
        return {"unavailable": "the reference pipeline was not built (oracle/_ref/libelasref.so)"}
    libc = ctypes.CDLL(None)
    sys.stdout.flush()
    saved, devnull = os.dup(1), os.open(os.devnull, os.O_WRONLY)
    ts = []
    try:
        os.dup2(devnull, 1)              # the reference prints a per-stage profile to stdout
        oracle.ref_elas_process(L, R)
        for _ in range(runs):
            t0 = time.perf_counter()
            oracle.ref_elas_process(L, R)
            ts.append(time.perf_counter() - t0)
    finally:
        libc.fflush(None)
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)
    ms = 1e3 * statistics.median(ts)
    return {"value": 1e3 / ms, "unit": "pairs/s", "ms_per_pair": ms, "runs": runs,
            "what": "reference Elas::process built for sm_100a, host buffers, median of the runs"}


def run_ours(args):
    import torch

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    W, H, D = eb.synth_dims(PRESET)
    L, R, gt, _ = eb.synth_pair(PRESET, replica_seed(rank))
    p = eb.params_config(D)
    e = eb.Elas(p, device=local)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    total_ms, stage_ms, launches, D1 = time_pipeline(e, L, R, args.steps, args.warmup, torch, flush, stream)
    barrier(world)
    torch.cuda.synchronize()
    clk = clocks.stop()
    max_ms = max_over_ranks(total_ms, world, device="cuda")
    pairs = args.steps * world
    value = aggregate_rate(args.steps, max_ms / 1e3, world)
    ms_per_step = max_ms / args.steps

    e2e_s, e2e_bytes = time_e2e(e, L, R, args.steps, torch, flush, args.warmup)
    e2e_s = max_over_ranks(e2e_s, world, device="cuda")
    e2e_value = pairs / e2e_s

    hbm, peak_kind = peaks()
    dense_bytes = 80.0 * W * H          # algorithmic bytes per launch (both views)
    dense_ms = stage_ms["dense"]
    dominant = max(stage_ms, key=stage_ms.get)
    roof = {"kernel": "k_dense (dense matching, both views)", "bound": "hbm",
            "achieved": dense_bytes / (dense_ms / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
            "frac": dense_bytes / (dense_ms / 1e3) / 1e9 / hbm, "peak_kind": peak_kind,
            "algorithmic_bytes_per_launch": dense_bytes,
            "traffic": profile_traffic("k_dense_1242x375"), "dominant_stage": dominant}
    out = {
        "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8",
        "data": "synthetic: seeded slanted textured planes, z-buffered right view, noise sigma 2",
        "config": {"workload": "elas_pair_1242x375_disp0-255", "width": W, "height": H, "disp_max": D,
                   "pairs_per_step_per_gpu": 1, "l2": "flushed before every step (256 MiB write)",
                   "parallelism": f"replicas x{world}", "params": "reference kernel constants + post-filters"},
        "gpix_disp_per_s": value * W * H * (D + 1) / 1e9,
        "e2e": {"value": e2e_value, "unit": "pairs/s", **e2e_bytes},
        "roofline": roof,
        "stages_ms": stage_ms,
        "clocks": clk,
        "gpu_launches": launches,
        "quality": quality(D1, gt),
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(L, R, p, args.cpu_seconds)
    if rank == 0 and world == 1 and not args.no_ref_gpu:
        out["reference_gpu"] = reference_gpu(L, R)
    if rank == 0 and world == 1 and not args.no_large:
        out["large"] = run_large(torch, args, flush, stream, hbm, peak_kind)
    if rank == 0 and world == 1 and not args.no_batch:
        out["batch"] = run_batch(torch, args, flush, stream)
    if rank == 0 and world == 1 and not args.no_learned:
        out["learned"] = run_learned(torch)
    e.close()
    del flush
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def run_large(torch, args, flush, stream, hbm, peak_kind):
    """The 5.7 MP configuration (2880x1988, disparity 0-511) on one GPU."""
    W, H, D = eb.synth_dims(2)
    L, R, gt, _ = eb.synth_pair(2, 1)
    p = eb.params_config(D)
    e = eb.Elas(p)
    steps = max(3, min(args.steps, 10))
    total_ms, stage_ms, launches, D1 = time_pipeline(e, L, R, steps, 3, torch, flush, stream)
    e.close()
    dense_bytes = 80.0 * W * H
    v = steps / (total_ms / 1e3)
    ref = reference_gpu(L, R) if not args.no_ref_gpu else None
    return {"workload": "elas_pair_2880x1988_disp0-511", "steps": steps, "value": v, "unit": "pairs/s",
            "reference_gpu_disp0-255": ref,
            "ms_per_step": total_ms / steps, "gpix_disp_per_s": v * W * H * (D + 1) / 1e9, "stages_ms": stage_ms,
            "roofline_dense": {"achieved": dense_bytes / (stage_ms["dense"] / 1e3) / 1e9, "peak": hbm,
                               "unit": "GB/s", "frac": dense_bytes / (stage_ms["dense"] / 1e3) / 1e9 / hbm,
                               "peak_kind": peak_kind, "traffic": profile_traffic("k_dense_2880x1988")},
            "gpu_launches": launches, "quality": quality(D1, gt)}


def run_learned(torch, n1=10, n2=3):
    """Plain ELAS against the learned support-point proposal on held-out
    seeds (the first n1 of the 1242x375 set, the first n2 of the 2880x1988
    set), with the trained weights shipped in the package."""
    if not os.path.exists(eb.PN_WEIGHTS):
        return {"unavailable": "no trained proposal weights in the package"}
    import proposal

    theta = eb.load_proposal()
    return [proposal.evaluate(torch, theta, 1, list(range(proposal.EVAL_SEED0_1242, proposal.EVAL_SEED0_1242 + n1))),
            proposal.evaluate(torch, theta, 2, list(range(proposal.EVAL_SEED0_2880, proposal.EVAL_SEED0_2880 + n2)))]


def batch_workload(n=64, seed=7):
    """Heterogeneous batch: widths 320-1920, heights 240-1080 (multiples of
    16), disparity ranges 64/128/256, drawn from a fixed seed."""
    rng = np.random.default_rng(seed)
    shapes = []
    for _ in range(n):
        w = int(rng.integers(20, 121)) * 16
        h = int(rng.integers(15, 68)) * 16
        d = int(rng.choice([64, 128, 256]))
        shapes.append((w, h, d))
    return shapes


def run_batch(torch, args, flush, stream):
    """64 independent pairs per step through the batched device call: one
    worker stream per pair, the whole batch replayed as one CUDA graph."""
    shapes = batch_workload()
    n = len(shapes)
    bufs, pix = [], 0
    for i, (w, h, d) in enumerate(shapes):
        L, R, _, _ = eb.synth_pair(3, 5000 + i, width=w, height=h, disp_max=d, gt=False)
        bufs.append([torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda(),
                     torch.empty((h, w), dtype=torch.float32, device="cuda"),
                     torch.empty((h, w), dtype=torch.float32, device="cuda")])
        pix += w * h
    dims = [(w, h) for (w, h, _) in shapes]
    dmax = [d for (_, _, d) in shapes]
    ptrs = [[b[k].data_ptr() for b in bufs] for k in range(4)]
    e = eb.Elas(eb.params_config(64))
    s = stream.cuda_stream
    out = {"workload": f"batch_{n}_pairs_w320-1920_h240-1080_disp64-256", "pairs_per_step": n,
           "megapixels_per_step": pix / 1e6}
    steps = max(3, min(args.steps, 10))
    for mode, graphs in (("graph", True), ("eager", False)):
        e.set_graphs(graphs)
        l0 = e.launch_count
        for _ in range(3):
            flush.zero_()
            e.process_batch_device(*ptrs, dims, dmax, stream=s)
        torch.cuda.synchronize()
        lat = []
        total = 0.0
        for _ in range(steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            e.process_batch_device(*ptrs, dims, dmax, stream=s)
            b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
            lat.extend(e.batch_latency(n).tolist())
        v = steps * n / (total / 1e3)
        out[mode] = {"value": v, "unit": "pairs/s", "ms_per_step": total / steps,
                     "megapixels_per_s": v * pix / n / 1e6,
                     "latency_ms_p50": float(np.percentile(lat, 50)), "latency_ms_p99": float(np.percentile(lat, 99)),
                     "steps": steps}
    out["dense_shapes"] = sorted({f"{(w + 127) // 128 * 128}/{d}:{e.dense_shape(w, d)}" for (w, _, d) in shapes})
    e.close()
    return out


def run_only(args):
    import torch

    torch.cuda.set_device(0)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    hbm, peak_kind = peaks()
    if args.only == "large":
        out = run_large(torch, args, flush, stream, hbm, peak_kind)
    elif args.only == "learned":
        out = run_learned(torch, n1=3, n2=2)
    else:
        out = run_batch(torch, args, flush, stream)
    print(json.dumps(out))


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle   # the generator and presets come from the oracle library: no product library is loaded

    W, H, D = oracle.synth_dims(PRESET)
    L, R, _, _ = oracle.synth_pair(PRESET, 1000)
    p = oracle.params_config(D)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        oracle.process(L, R, p, threads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.process(L, R, p, threads=threads)
    el = time.perf_counter() - t0
    value = args.steps / el
    out = {
        "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic", "impl": "reference",
        "config": {"workload": "elas_pair_1242x375_disp0-255", "width": W, "height": H, "disp_max": D,
                   "pairs_per_step_per_gpu": 1, "parallelism": "host cores"},
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full pairs through the CPU restatement of the reference "
                                   f"kernels with the reference's Triangle, {threads} threads"},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-large", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--only", choices=["large", "batch", "learned"], default=None,
                    help="run one secondary workload alone (for profiling) and print its block")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.only:
        run_only(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
