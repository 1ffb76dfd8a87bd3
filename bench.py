"""Benchmark of the resample hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--no-cpu] [--no-others] [--split]
                    [--images N] [--only NAME]

Headline workload (the metric "input Mpix/s batched vs per-image GPU (bit-exact
u8); fwd+bwd GB/s vs HBM"): thumbnails of 512 u8 images of uneven size (width
log-uniform in 256..6000, aspect w/h uniform in 0.5..2, 3 or 4 bands with
p = 0.5) to a 256 px FitBox with Lanczos3 — per image the in-memory thumbnail
chain (premultiply for 4 bands, box shrink, residual Lanczos3 reduce,
unpremultiply).  A step is one run of the whole batch: a few persistent
launches over a device work list, one per stage level and kind (the shrinks of
every image, then the fused reduces), captured in a CUDA graph, inputs resident in
HBM (about 9.4 GB, far above the 126 MB L2: no flush needed).  The plain
per-image GPU path (each image's plan launched in turn) is timed on the same
images, and the batch output is checked bit-exact against it.

Every rank runs its own 512-image batch (different seeds): `value` is the
input Mpix/s of all ranks over the max-over-ranks time, scaling "weak"; no
data crosses between GPUs.  With `--split` the ranks divide ONE batch by byte
weight (api.partition_batch, computed identically on every rank), scaling
"strong".

`e2e` is the same batch through ThumbnailBatch.run_host: pinned host images
copied in, the graph run, thumbnails copied out, every step.  `roofline` is the
batch kernel's algorithmic bytes (each image's input read once + output written
once) over its CUDA-event time per launch, against MEASURED_PEAKS.json.
`cpu_baseline` is the oracle (the C restatement of viprs's CPU path) on all
host cores over the whole batch once; its thumbnails are compared byte for
byte with the GPU batch's (`parity`).  `others` holds the remaining
configurations: the 8192x8192x3 thumbnail, the 1024x768x3 reduce, the f32
6000x4000x4 resize, and the fwd+bwd GB/s of the reduce+affine and mapim
gradient workloads.

`--impl reference` times the reference arm: viprs's CPU path as restated in C
(viprs itself needs a Rust toolchain this image lacks), all host cores, the
whole batch -- the same shapes and seeded generator as the GPU arm -- per step.
"""
import argparse
import ctypes
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
# DRAM bytes (read + write) of one batch step over its algorithmic bytes, from
# an ncu capture of one step's persistent launches on the first 64 images
# (`ncu --clock-control none --metrics dram__bytes_read.sum,dram__bytes_write.sum
# -k regex:^batch_ -c 5 python bench.py --images 64 --steps 1 --warmup 3 --no-cpu
# --no-others --no-autotune`, the step's four launches for these images:
# 1,174,348,288 B against 1,156,046,596 B); every image adds its input once and
# its shrunk intermediate once, so the ratio carries over to the 512-image step
BATCH_TRAFFIC_RATIO = 1174348288 / 1156046596
METRIC = "input Mpix/s batched vs per-image GPU (bit-exact u8); fwd+bwd GB/s vs HBM"
BATCH_N = 512
BATCH_SEED = 0x5EED0003
BATCH_BOX = 256
WORKLOAD = f"{BATCH_N} uneven u8 images (w logU[256,6000], w/h U[0.5,2], 3|4 bands) -> thumbnail FitBox {BATCH_BOX} Lanczos3"


def batch_config(shapes):
    """The `config` of both arms: the workload and its exact size (identical
    for the GPU arm and the reference arm, which process the same images)."""
    return {"workload": WORKLOAD if len(shapes) == BATCH_N else f"first {len(shapes)} of: {WORKLOAD}",
            "images": len(shapes), "seed": BATCH_SEED,
            "input_mpix": round(sum(h * w for h, w, _ in shapes) / 1e6, 2),
            "input_bytes": sum(h * w * b for h, w, b in shapes)}


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
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
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


def _rank_device():
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(x, ws):
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_rank_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, ws):
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_rank_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def timed(fn, steps, warmup, stream):
    """Mean CUDA-event ms of fn() over `steps` launches after `warmup`."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for a, b in evs:
        a.record(stream)
        fn()
        b.record(stream)
    torch.cuda.synchronize()
    return statistics.mean(a.elapsed_time(b) for a, b in evs)


def graph_timed(fn, steps):
    """Mean CUDA-event ms of one replay of fn() captured in a CUDA graph: the
    device time of its launches without the host's gaps between them.  fn must
    read the current stream at call time.  Returns (ms, None) or (None, why)
    when fn does not capture."""
    import torch
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        fn()  # tables cached, allocations settled before the capture
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    try:
        with torch.cuda.graph(g):
            fn()
    except Exception as e:  # reported, never hidden
        torch.cuda.synchronize()
        return None, f"{type(e).__name__}: {e}"[:200]
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    cur = torch.cuda.current_stream()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for a, b in evs:
        a.record(cur)
        g.replay()
        b.record(cur)
    torch.cuda.synchronize()
    ms = statistics.mean(a.elapsed_time(b) for a, b in evs)
    del g
    return ms, None


# ----------------------------------------------------------------------------- headline: batched thumbnails

def make_batch_images(seed, n=BATCH_N, device="cuda", indices=None):
    """Shapes and pixels of the batch (its first n images, or the images
    `indices` of them), each image seeded by its index in the batch."""
    from viprs_b200 import synth
    shapes = synth.uneven_batch_shapes(BATCH_N, seed)[:n]
    if indices is None:
        indices = range(len(shapes))
    imgs = [synth.smooth_u8(*shapes[i], seed * 1000 + i, device=device) for i in indices]
    return [shapes[i] for i in indices], imgs


def cpu_batch_step(host_imgs, threads, outs=None):
    """One step of the CPU arm: the oracle (the C restatement of viprs's CPU
    path) thumbnails every image of the batch in order, each on `threads`
    host threads.  Returns the thumbnails when `outs` is a list."""
    from oracle import oracle as O
    for img in host_imgs:
        r = O.thumbnail(img, "fitbox", BATCH_BOX, BATCH_BOX, threads=threads)
        if outs is not None:
            outs.append(r)


def cpu_baseline_batch(srcs, dsts):
    """The oracle on all host cores over the whole batch, once, timed; every
    thumbnail it makes is compared byte for byte with the GPU batch's."""
    import numpy as np
    threads = os.cpu_count() or 1
    host_imgs = [s.cpu().numpy() for s in srcs]
    mpix = sum(im.shape[0] * im.shape[1] for im in host_imgs) / 1e6
    outs = []
    cpu_batch_step(host_imgs[:1], threads)  # warm
    t0 = time.perf_counter()
    cpu_batch_step(host_imgs, threads, outs)
    el = time.perf_counter() - t0
    same = sum(int(o.shape == tuple(d.shape) and np.array_equal(o, d.cpu().numpy())) for o, d in zip(outs, dsts))
    line = {"value": round(mpix / el, 3), "unit": "Mpix/s", "cores": threads, "kind": "port",
            "sample": f"the whole batch ({len(host_imgs)} images, {mpix:.1f} Mpix) once, image after image, "
                      f"each on all {threads} threads, {el:.1f} s"}
    return line, same, len(outs)


def run_batch(args, rank, ws, local):
    import numpy as np
    import torch

    from viprs_b200 import api

    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    if args.split and ws > 1:
        # one batch divided over the ranks by byte weight (strong scaling)
        from viprs_b200 import synth
        every = synth.uneven_batch_shapes(BATCH_N, BATCH_SEED)[:args.images]
        shapes, srcs = make_batch_images(BATCH_SEED, args.images, indices=api.partition_batch(every, ws)[rank])
    else:
        # an independent batch per rank (weak scaling)
        shapes, srcs = make_batch_images(BATCH_SEED + 7919 * rank, args.images)
    batch = api.ThumbnailBatch(shapes, "fitbox", BATCH_BOX, BATCH_BOX)
    dsts = batch.alloc_outputs()
    in_bytes = sum(h * w * b for h, w, b in shapes)
    out_bytes = sum(h * w * b for h, w, b in batch.out_shapes)
    mpix = sum(h * w for h, w, _ in shapes) / 1e6

    split = bool(args.split and ws > 1)
    # the project's autotuner picks the ring size, work-list lag and blocks per SM
    tuned = batch.autotune(srcs, dsts, repeats=2)[0] if not args.no_autotune else batch.config()
    items, stages, grid = batch.work()

    # plain per-image GPU path, timed on the same images
    per = batch.alloc_outputs()
    per_ms = timed(lambda: batch.run_per_image(srcs, per), max(3, args.steps // 4), 2, stream)
    batched_launches, per_launches = batch.launches()

    # batched: warm-up (captures the graph), then K timed graph launches
    for _ in range(args.warmup):
        batch.run(srcs, dsts, graph=True)
    torch.cuda.synchronize()
    assert batch.status() == 0, "batch kernel reported an error"
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.25)
    barrier(ws)
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for a, b in evs:
        a.record(stream)
        batch.run(srcs, dsts, graph=True)
        b.record(stream)
    end.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clocks = sampler.stop()
    assert batch.status() == 0, "batch kernel reported an error"
    total_ms = max_over_ranks(start.elapsed_time(end), ws)
    kernel_ms = statistics.mean(a.elapsed_time(b) for a, b in evs)
    all_mpix = sum_over_ranks(mpix, ws)
    value = all_mpix * args.steps / (total_ms / 1e3)
    per_value = mpix / (per_ms / 1e3)

    same = all(torch.equal(a, b) for a, b in zip(dsts, per))

    # end to end from pinned host memory through ThumbnailBatch.run_host
    host_srcs = [s.cpu().pin_memory() for s in srcs]
    host_dsts = [torch.empty(s, dtype=torch.uint8).pin_memory() for s in batch.out_shapes]
    e2e_steps = max(3, min(args.steps, 10))
    batch.run_host(host_srcs, host_dsts, srcs, dsts)
    barrier(ws)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        batch.run_host(host_srcs, host_dsts, srcs, dsts)
    e2e_s = max_over_ranks(time.perf_counter() - t0, ws)
    e2e_value = all_mpix * e2e_steps / e2e_s
    same = same and all(torch.equal(h, d.cpu()) for h, d in zip(host_dsts, dsts))

    peak, peak_kind = measured_hbm_peak()
    alg = in_bytes + out_bytes
    achieved = alg / (kernel_ms / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "Mpix/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "strong" if split else "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded smooth sinusoids + uniform noise, generated on device)",
        "config": batch_config(every if split else shapes),
        "batch_plan": {"persistent_launches_per_step": batched_launches,
                       "parallelism": (f"one batch split over {ws} GPUs by byte weight" if split
                                       else f"independent batch per GPU x{ws}"),
                       "l2": f"inputs {in_bytes / 1e9:.1f} GB >> 126 MB L2 (no flush needed)",
                       "autotuned": tuned, "work_items": items, "stages": stages, "grid": grid},
        "gpu_launches": args.steps * batched_launches,
        "per_image": {"value": round(per_value, 2), "unit": "Mpix/s", "ms_per_step": round(per_ms, 4),
                      "launches_per_step": per_launches},
        "batched_over_per_image": round(value / ws / per_value, 3),
        "e2e": {"value": round(e2e_value, 2), "unit": "Mpix/s", "h2d_bytes_per_step": in_bytes,
                "d2h_bytes_per_step": out_bytes, "path": "ThumbnailBatch.run_host (pinned host buffers)"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": round(alg * BATCH_TRAFFIC_RATIO),
                     "traffic_source": "ncu capture of the first 64 images, scaled by algorithmic bytes",
                     "peak_kind": peak_kind,
                     "kernel": "batch_kernel", "kernel_ms": round(kernel_ms, 4), "algorithmic_bytes": alg},
        "clocks": clocks,
        "parity": "batched == per-image path (bit-exact)" if same else "MISMATCH batched vs per-image",
    }
    del host_srcs, host_dsts
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"], n_same, n_cpu = cpu_baseline_batch(srcs, dsts)
        line["parity"] = (f"oracle bit-exact on {n_same}/{n_cpu} images; " + line["parity"]
                          if n_same == n_cpu else f"MISMATCH oracle on {n_cpu - n_same}/{n_cpu} images; "
                          + line["parity"])
    return line


# ----------------------------------------------------------------------------- the other configurations

def other_thumbnail_8192(stream, steps):
    import torch

    from viprs_b200 import api, synth
    H = W = 8192
    img = synth.smooth_u8(H, W, 3, 0x5EED0001)
    plan = api.thumbnail_plan(W, H, 3, torch.uint8, "width", 400)
    out = torch.empty(plan.out_shape, dtype=torch.uint8, device="cuda")
    total = timed(lambda: plan(img, out), steps, 3, stream)
    shrink = timed(lambda: plan.run_stages(img, out, 0, 1), steps, 3, stream)
    g_total, why = graph_timed(lambda: plan(img, out), steps)
    g_shrink, _ = graph_timed(lambda: plan.run_stages(img, out, 0, 1), steps)
    need = (W // 19) * 19
    sb = need * need * 3 + (W // 19) * (H // 19) * 3
    peak, _ = measured_hbm_peak()
    r = {"workload": "thumbnail 8192x8192x3 u8 -> 400 px (shrink 19 + Lanczos3 1.0779)",
         "mpix_per_s": round(H * W / 1e6 / (total / 1e3), 1), "ms": round(total, 4), "launches": plan.launches,
         "shrink_kernel": {"ms": round(shrink, 4), "algorithmic_bytes": sb,
                           "gbs": round(sb / (shrink / 1e3) / 1e9, 1),
                           "frac": round(sb / (shrink / 1e3) / 1e9 / peak, 4)}}
    if g_total is not None:
        r["graph"] = {"ms": round(g_total, 4), "mpix_per_s": round(H * W / 1e6 / (g_total / 1e3), 1),
                      "shrink_ms": round(g_shrink, 4), "shrink_gbs": round(sb / (g_shrink / 1e3) / 1e9, 1),
                      "shrink_frac": round(sb / (g_shrink / 1e3) / 1e9 / peak, 4)}
    else:
        r["graph"] = {"unavailable": why}
    return r


def other_reduce_1024(stream, steps):
    import torch

    from viprs_b200 import api, synth
    img = synth.smooth_u8(768, 1024, 3, 0x5EED0000)
    plan = api.PipelineBuilder(1024, 768, 3, torch.uint8).reduce_h(4.0).reduce_v(4.0).build()
    out = torch.empty(plan.out_shape, dtype=torch.uint8, device="cuda")
    ms = timed(lambda: plan(img, out), steps, 3, stream)
    gms, why = graph_timed(lambda: plan(img, out), steps)
    b = 1024 * 768 * 3 + 256 * 192 * 3
    r = {"workload": "reduce_h(4)+reduce_v(4) Lanczos3 1024x768x3 u8 (single launch, latency-bound)",
         "mpix_per_s": round(0.786432 / (ms / 1e3), 1), "us": round(ms * 1e3, 2), "algorithmic_bytes": b,
         "gbs": round(b / (ms / 1e3) / 1e9, 1)}
    r["graph"] = {"us": round(gms * 1e3, 2), "gbs": round(b / (gms / 1e3) / 1e9, 1)} if gms else {"unavailable": why}
    return r


def other_reduce_1024_batch(stream, steps, n=256):
    """The reduce_h(4)+reduce_v(4) workload of the 1024x768x3 case on n images
    at once: one persistent launch over the batch's work list (ChainBatch), and
    the same n images as n per-image plan launches."""
    import torch

    from viprs_b200 import api, synth
    imgs = [synth.smooth_u8(768, 1024, 3, 0x5EED0000 + i) for i in range(n)]
    builder = api.PipelineBuilder(1024, 768, 3, torch.uint8).reduce_h(4.0).reduce_v(4.0)
    batch = api.ChainBatch([(768, 1024, 3)] * n, builder)
    outs = batch.alloc_outputs()
    ms = timed(lambda: batch.run(imgs, outs, graph=True), steps, 3, stream)
    plan = builder.build()
    pouts = [torch.empty(plan.out_shape, dtype=torch.uint8, device="cuda") for _ in range(n)]

    def per_image():
        for i in range(n):
            plan(imgs[i], pouts[i])
    pms = timed(per_image, steps, 3, stream)
    b = n * (1024 * 768 * 3 + 256 * 192 * 3)
    peak, kind = measured_hbm_peak()
    gbs = b / (ms / 1e3) / 1e9
    return {"workload": f"{n} x reduce_h(4)+reduce_v(4) Lanczos3 1024x768x3 u8, one persistent launch (ChainBatch)",
            "images": n, "mpix_per_s": round(n * 0.786432 / (ms / 1e3), 1), "ms": round(ms, 4),
            "algorithmic_bytes": b, "gbs": round(gbs, 1), "frac": round(gbs / peak, 4), "peak_kind": kind,
            "per_image_ms": round(pms, 4), "batched_vs_per_image": round(pms / ms, 2),
            "launches": batch.launches()[0], "per_image_launches": n * plan.launches}


def other_resize_f32(stream, steps):
    import torch

    from viprs_b200 import api, synth
    img = synth.uniform_f32(4000, 6000, 4, 0x5EED0002)
    plan = api.resize_plan(6000, 4000, 4, torch.float32, 0.37)
    out = torch.empty(plan.out_shape, dtype=torch.float32, device="cuda")
    ms = timed(lambda: plan(img, out), steps, 3, stream)
    b = 6000 * 4000 * 16 + out.numel() * 4
    peak, _ = measured_hbm_peak()
    return {"workload": "resize 0.37 Lanczos3 6000x4000x4 f32 (ReduceV+ReduceH 2.7027 fused)",
            "mpix_per_s": round(24.0 / (ms / 1e3), 1), "ms": round(ms, 4), "algorithmic_bytes": b,
            "gbs": round(b / (ms / 1e3) / 1e9, 1), "frac": round(b / (ms / 1e3) / 1e9 / peak, 4),
            "launches": plan.launches}


def other_resize_up(stream, steps):
    """resize 2.0 of 4096x3072x3 u8 (one Zoom(2, 2) node) and resize 2.5 of
    1024x768x3 u8 (Zoom(2, 2) + the Copy-extend Lanczos3 affine tail)."""
    import torch

    from viprs_b200 import api, synth
    img = synth.smooth_u8(3072, 4096, 3, 0x5EED000B)
    plan = api.resize_plan(4096, 3072, 3, torch.uint8, 2.0)
    out = torch.empty(plan.out_shape, dtype=torch.uint8, device="cuda")
    ms = timed(lambda: plan(img, out), steps, 3, stream)
    b = img.numel() + out.numel()
    small = synth.smooth_u8(768, 1024, 3, 0x5EED000C)
    plan2 = api.resize_plan(1024, 768, 3, torch.uint8, 2.5)
    out2 = torch.empty(plan2.out_shape, dtype=torch.uint8, device="cuda")
    ms2 = timed(lambda: plan2(small, out2), steps, 3, stream)
    sim_b = api.PipelineBuilder(1024, 768, 3, torch.uint8).similarity(1.25, 30.0, "bicubic")
    plan3 = sim_b.build()
    out3 = torch.empty(plan3.out_shape, dtype=torch.uint8, device="cuda")
    ms3 = timed(lambda: plan3(small, out3), steps, 3, stream)
    peak, _ = measured_hbm_peak()
    return {"workload": "resize 2.0 of 4096x3072x3 u8 (Zoom 2x2, 16-byte stores)",
            "mpix_per_s": round(out.numel() / 3 / 1e6 / (ms / 1e3), 1), "ms": round(ms, 4),
            "algorithmic_bytes": b, "gbs": round(b / (ms / 1e3) / 1e9, 1),
            "frac": round(b / (ms / 1e3) / 1e9 / peak, 4), "launches": plan.launches,
            "resize_2_5_1024x768": {"workload": "resize 2.5 Lanczos3 1024x768x3 u8 (Zoom 2x2 + affine 1.25)",
                                    "ms": round(ms2, 4), "launches": plan2.launches,
                                    "mpix_per_s": round(out2.numel() / 3 / 1e6 / (ms2 / 1e3), 1)},
            "similarity_1024x768": {"workload": "similarity scale 1.25 angle 30 bicubic 1024x768x3 u8 (auto canvas)",
                                    "ms": round(ms3, 4), "launches": plan3.launches,
                                    "out": list(plan3.out_shape),
                                    "mpix_per_s": round(out3.numel() / 3 / 1e6 / (ms3 / 1e3), 1)}}


def other_reduce_affine_grad(stream, steps):
    """16 x 1024^2 x 4 f32: reduce_h(2)+reduce_v(2) -> affine bilinear 512^2 (alpha path), fwd + bwd."""
    import torch

    from viprs_b200 import _native as N
    from viprs_b200 import api, synth
    n, S = 16, 4
    xs = [synth.uniform_f32(1024, 1024, 4, 0x5EED0004 + i) for i in range(n)]
    gys = [torch.randn((512, 512, 4), device="cuda") for _ in range(n)]
    # the 16 images run on S streams (one plan per stream: a plan's executions
    # must not overlap), so that their small launches overlap on the GPU
    plans = [api.PipelineBuilder(1024, 1024, 4, torch.float32).reduce_h(2.0).reduce_v(2.0).build()
             for _ in range(S)]
    plan = plans[0]
    streams = [torch.cuda.Stream() for _ in range(S)]
    zs = [torch.empty(plan.out_shape, device="cuda") for _ in range(n)]
    ys = [torch.empty((512, 512, 4), device="cuda") for _ in range(n)]
    gzs = [torch.empty(plan.out_shape, device="cuda") for _ in range(n)]
    gxs = [torch.empty((1024, 1024, 4), device="cuda") for _ in range(n)]
    gms = torch.empty((n, 6), dtype=torch.float64, device="cuda")
    mats = []
    for M, tx, ty in synth.rotation_matrices(n, 0x5EED0004):
        bm, btx, bty = api.forward_affine_to_backward(M, tx, ty)
        mats.append(((ctypes.c_double * 4)(*bm), btx, bty))
    L = N.lib()

    def fan_out(work):
        """work(k, i) for image i on stream k = i % S; every stream starts after
        and ends before the current stream's position."""
        main = torch.cuda.current_stream()
        ev = main.record_event()
        for k, st in enumerate(streams):
            st.wait_event(ev)
            with torch.cuda.stream(st):
                for i in range(k, n, S):
                    work(k, i)
        for st in streams:
            main.wait_stream(st)

    def fwd_one(k, i):
        plans[k](xs[i], zs[i])
        m, btx, bty = mats[i]
        N.check(L.viprs_affine_backward_matrix(api.image(zs[i]), api.image(ys[i]), m, btx, bty, 1, 2, 0.0, 0,
                                               0, 0, api._stream()), "affine")

    def bwd_one(k, i):
        m, btx, bty = mats[i]
        sp = api._stream()
        N.check(L.viprs_affine_grad(api.image(zs[i]), api.image(gys[i]), api.image(gzs[i]), m, btx, bty, 1, 2,
                                    0.0, 0, 0, 0, 0, ctypes.c_void_p(gms[i].data_ptr()), sp), "affine_grad")
        N.check(L.viprs_reduce_hv_adjoint(api.image(gzs[i]), api.image(gxs[i]), 2.0, 2.0, 9, sp),
                "reduce_hv_adjoint")

    def fwd():
        fan_out(fwd_one)

    def bwd():
        fan_out(bwd_one)

    fwd_ms = timed(fwd, steps, 3, stream)
    bwd_ms = timed(bwd, steps, 3, stream)
    g_fwd, why = graph_timed(fwd, steps)
    g_bwd, why_b = graph_timed(bwd, steps)
    alg = 738197504
    peak, _ = measured_hbm_peak()
    gbs = alg / ((fwd_ms + bwd_ms) / 1e3) / 1e9
    r = {"workload": "16 x 1024^2x4 f32: reduce_h(2)+reduce_v(2) L3 -> affine(s R(theta), t) bilinear 512^2, "
                     "fwd + bwd (image and matrix gradients, f32-atomic scatter), images over 4 streams",
         "fwd_ms": round(fwd_ms, 4), "bwd_ms": round(bwd_ms, 4), "algorithmic_bytes_fwd_bwd": alg,
         "gbs": round(gbs, 1), "frac": round(gbs / peak, 4)}
    if g_fwd is not None and g_bwd is not None:
        gg = alg / ((g_fwd + g_bwd) / 1e3) / 1e9
        r["graph"] = {"fwd_ms": round(g_fwd, 4), "bwd_ms": round(g_bwd, 4), "gbs": round(gg, 1),
                      "frac": round(gg / peak, 4)}
    else:
        r["graph"] = {"unavailable": why or why_b}
    return r


def other_mapim_grad(stream, steps):
    """4096^2 f32 source, identity grid + smooth displacement (max 8 px), bicubic, fwd + bwd."""
    import torch

    from viprs_b200 import _native as N
    from viprs_b200 import api, synth
    S = 4096
    src = synth.uniform_f32(S, S, 1, 0x5EED0005)
    index = synth.displacement_index(S, 0x5EED0005)
    out = torch.empty((S, S, 1), device="cuda")
    gy = torch.randn((S, S, 1), device="cuda")
    gs = torch.empty_like(src)
    gi = torch.empty_like(index)
    L = N.lib()

    def fwd():
        N.check(L.viprs_mapim(api.image(src), api.image(index), api.image(out), 2, 0, 0.0, 0, api._stream()), "mapim")

    def bwd(det):
        N.check(L.viprs_mapim_grad(api.image(src), api.image(index), api.image(gy), api.image(gs), api.image(gi),
                                   2, 0, 0.0, 0, det, api._stream()), "mapim_grad")

    fwd_ms = timed(fwd, steps, 3, stream)
    bwd_ms = timed(lambda: bwd(0), steps, 3, stream)
    det_ms = timed(lambda: bwd(1), steps, 3, stream)
    alg = 738197504
    peak, _ = measured_hbm_peak()
    gbs = alg / ((fwd_ms + bwd_ms) / 1e3) / 1e9
    return {"workload": "mapim bicubic 4096^2x1 f32, index = identity + Gaussian(sigma 32)-smoothed displacement "
                        "(max 8 px), fwd + bwd (image and coordinate gradients)",
            "fwd_ms": round(fwd_ms, 4), "bwd_ms_atomic": round(bwd_ms, 4), "bwd_ms_deterministic": round(det_ms, 4),
            "algorithmic_bytes_fwd_bwd": alg, "gbs": round(gbs, 1), "frac": round(gbs / peak, 4),
            "forward_only_gbs": round(268435456 / (fwd_ms / 1e3) / 1e9, 1)}


OTHERS = (("thumbnail_8192", other_thumbnail_8192), ("reduce_1024x768", other_reduce_1024),
          ("reduce_1024x768_x256", other_reduce_1024_batch),
          ("resize_f32_6000x4000", other_resize_f32), ("resize_up", other_resize_up),
          ("reduce_affine_fwd_bwd", other_reduce_affine_grad),
          ("mapim_fwd_bwd", other_mapim_grad))


def run_others(steps, only=None):
    import torch
    stream = torch.cuda.current_stream()
    out = {}
    for name, fn in OTHERS:
        if only is not None and name != only:
            continue
        try:
            out[name] = fn(stream, steps)
        except Exception as e:  # reported, never hidden
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        torch.cuda.empty_cache()
    return out


# ----------------------------------------------------------------------------- reference arm

def run_reference(args, rank, ws):
    """Reference arm: viprs's CPU path restated in C (viprs itself needs a Rust
    toolchain that this image lacks), on all host cores.  Each step is the
    whole batch -- the same 512 images, shapes and seeds as the GPU arm,
    generated on the host -- each image's thumbnail on all threads."""
    if rank != 0:
        return None
    from viprs_b200 import synth
    shapes = synth.uneven_batch_shapes(BATCH_N, BATCH_SEED)[:args.images]
    imgs = [synth.smooth_u8(*shapes[i], BATCH_SEED * 1000 + i, device="cpu").numpy() for i in range(len(shapes))]
    mpix = sum(im.shape[0] * im.shape[1] for im in imgs) / 1e6
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_batch_step(imgs, threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cpu_batch_step(imgs, threads)
    el = time.perf_counter() - t0
    v = mpix * args.steps / el
    sample = f"the whole batch ({len(imgs)} images, {mpix:.1f} Mpix) per step, image after image, each on all " \
             f"{threads} threads"
    return {
        "metric": METRIC, "value": round(v, 3), "unit": "Mpix/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(el * 1e3 / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded smooth sinusoids + noise)",
        "config": batch_config(shapes),
        "impl": "reference",
        "cpu_baseline": {"value": round(v, 3), "unit": "Mpix/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": round(v, 3), "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-others", action="store_true")
    ap.add_argument("--images", type=int, default=BATCH_N, help="first N images of the batch (profiling cases)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default kernel configuration")
    ap.add_argument("--split", action="store_true",
                    help="with several GPUs: divide ONE batch over them by byte weight (strong scaling) instead of "
                         "giving each GPU its own batch")
    ap.add_argument("--only", default=None, choices=[n for n, _ in OTHERS],
                    help="run one of the other configurations alone, --steps timed steps (profiling cases)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    args.steps = max(args.steps, 1)
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        ws = int(os.environ.get("WORLD_SIZE", "1"))
        line = run_reference(args, rank, ws)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    if args.only is not None:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps({"only": args.only, **run_others(args.steps, args.only)}), flush=True)
        return
    rank, ws, local = dist_setup()
    line = run_batch(args, rank, ws, local)
    if rank == 0 and not args.no_others:
        line["others"] = run_others(10)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
