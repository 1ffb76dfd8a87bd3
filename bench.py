"""Benchmark of the resample hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Workload (N=1 default): thumbnail of one 8192x8192x3 u8 image to 400 px width
(in-memory plan: ShrinkH 19 -> ShrinkV 19 -> ReduceH/ReduceV 1.0779 Lanczos3).
A step is one execution of the plan on device-resident input; the 201 MB
input exceeds the 126 MB L2, so no flush is needed between steps.

Prints one JSON line.  `value` is input Mpix/s over all ranks (each rank runs
its own replica: the single-image workload does not shard).  `e2e` is the same
metric through the public plan API with host buffers (pinned host -> device
copy of the input and device -> host copy of the thumbnail inside the timed
region).  `roofline` is the shrink kernel's algorithmic HBM bytes per launch
divided by its CUDA-event launch time, against the measured copy bandwidth.
`cpu_baseline` is the CPU restatement of viprs on this host's cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0


def measured_hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, 0
    import datetime

    import torch
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    return rank, ws, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, ws):
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline_thumbnail(img_np, target_w, seconds=10.0):
    """The CPU restatement of viprs (oracle port) on all host cores, on the same image."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    O.thumbnail(img_np, "width", target_w, 0, threads=threads)  # warm
    n = 0
    t0 = time.perf_counter()
    while True:
        O.thumbnail(img_np, "width", target_w, 0, threads=threads)
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    mpix = img_np.shape[0] * img_np.shape[1] / 1e6
    return {"value": round(mpix * n / el, 3), "unit": "Mpix/s", "cores": threads, "kind": "port",
            "sample": f"{n} thumbnails of the same {img_np.shape[1]}x{img_np.shape[0]}x{img_np.shape[2]} u8 "
                      f"image in {el:.1f} s"}


def run_thumbnail(args, rank, ws, local):
    import numpy as np
    import torch

    from viprs_b200 import api, synth

    H = W = 8192
    B = 3
    TW = 400
    torch.cuda.set_device(local)
    img = synth.smooth_u8(H, W, B, 0x5EED0001 + rank)
    plan = api.thumbnail_plan(W, H, B, torch.uint8, "width", TW)
    out = torch.empty(plan.out_shape, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        plan(img, out)
    torch.cuda.synchronize()
    n_st = plan.launches
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    barrier(ws)
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for k in range(args.steps):
        e0, e1, e2 = ev[k]
        e0.record(stream)
        plan.run_stages(img, out, 0, 1)
        e1.record(stream)
        plan.run_stages(img, out, 1, n_st - 1)
        e2.record(stream)
    end.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clocks = sampler.stop()
    total_ms = start.elapsed_time(end)
    total_ms = max_over_ranks(total_ms, ws)
    shrink_ms = statistics.mean(e0.elapsed_time(e1) for e0, e1, _ in ev)
    mpix = H * W / 1e6
    value = mpix * args.steps * ws / (total_ms / 1e3)

    # algorithmic bytes of the shrink launch: the 8189x8189 source pixels the
    # 19x19 box shrink needs, read once, plus the shrunk plane written once
    fh = 19
    need = (W // fh) * fh
    shrink_bytes = need * need * B + (W // fh) * (H // fh) * B
    achieved = shrink_bytes / (shrink_ms / 1e3) / 1e9
    peak, peak_kind = measured_hbm_peak()

    # end to end through the public API from pinned host memory
    host_in = img.cpu().pin_memory()
    host_out = torch.empty(plan.out_shape, dtype=torch.uint8).pin_memory()
    for _ in range(max(1, args.warmup)):
        plan.execute_host(host_in, host_out)
    barrier(ws)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        plan.execute_host(host_in, host_out)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, ws)
    e2e_value = mpix * args.steps * ws / e2e_s

    ok = np.array_equal(out.cpu().numpy(), host_out.numpy())
    line = {
        "metric": "thumbnail input Mpix/s (8192x8192x3 u8 -> 400 px, bit-exact vs viprs CPU path)",
        "value": round(value, 2), "unit": "Mpix/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded smooth sinusoids + noise, generated on device)",
        "config": {"workload": "thumbnail 8192x8192x3 u8 -> 400x400 (shrink 19 + Lanczos3 reduce 1.0779)",
                   "parallelism": f"replicas x{ws}", "l2": "input 201 MB > 126 MB L2 (no flush needed)"},
        "gpu_launches": n_st * args.steps,
        "e2e": {"value": round(e2e_value, 2), "unit": "Mpix/s", "h2d_bytes_per_step": H * W * B,
                "d2h_bytes_per_step": int(np.prod(plan.out_shape))},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None, "peak_kind": peak_kind,
                     "kernel": "shrink2d_kernel<u8,HV>", "kernel_ms": round(shrink_ms, 4),
                     "algorithmic_bytes": shrink_bytes},
        "clocks": clocks,
        "parity": "device result equals host-path result" if ok else "MISMATCH",
    }
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline_thumbnail(img.cpu().numpy(), TW, args.cpu_seconds)
    return line


def run_reference(args, rank, ws):
    """Reference arm: viprs's CPU path restated in C (viprs itself needs a Rust
    toolchain that this image lacks), on all host cores, same workload."""
    import numpy as np
    if rank != 0:
        return None
    from oracle import oracle as O
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    rng = np.random.default_rng(0x5EED0001)
    # a host-generated image of the workload's shape and distribution
    from gpu_helpers import smooth_image
    img = smooth_image(rng, 8192, 8192, 3)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        O.thumbnail(img, "width", 400, 0, threads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.thumbnail(img, "width", 400, 0, threads=threads)
    el = time.perf_counter() - t0
    v = 8192 * 8192 / 1e6 * args.steps / el
    return {
        "metric": "thumbnail input Mpix/s (8192x8192x3 u8 -> 400 px, bit-exact vs viprs CPU path)",
        "value": round(v, 3), "unit": "Mpix/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(el * 1e3 / args.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded smooth sinusoids + noise)",
        "config": {"workload": "thumbnail 8192x8192x3 u8 -> 400x400 (shrink 19 + Lanczos3 reduce 1.0779)",
                   "parallelism": "host threads"},
        "impl": "reference",
        "cpu_baseline": {"value": round(v, 3), "unit": "Mpix/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} thumbnails of one 8192x8192x3 u8 image"},
        "e2e": {"value": round(v, 3), "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        ws = int(os.environ.get("WORLD_SIZE", "1"))
        line = run_reference(args, rank, ws)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    rank, ws, local = dist_setup()
    line = run_thumbnail(args, rank, ws, local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
