"""The multi-GPU bench path on CPU: two ranks over gloo (127.0.0.1).

bench.py runs one rank per GPU: each rank takes its own images, no data
crosses between ranks, and only the timing is combined (max of the ranks'
times, sum of their megapixels).  These tests run that plumbing with two CPU
processes: the byte-weighted split of one batch over the ranks, the rank
reductions the bench reports, and a split batch whose per-rank thumbnails
(computed with the CPU restatement of viprs on each rank) together equal the
single-process result.
"""
import zlib

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, result_dir):
    import datetime

    import bench
    from viprs_b200 import api, synth
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        shapes = synth.uneven_batch_shapes(512, bench.BATCH_SEED)
        parts = api.partition_batch(shapes, ws)
        mine = parts[rank]
        gathered = [None] * ws
        dist.all_gather_object(gathered, mine)
        # every rank computed the same split on its own
        assert gathered == parts
        mpix = sum(shapes[i][0] * shapes[i][1] for i in mine) / 1e6
        total = bench.sum_over_ranks(mpix, ws)
        slowest = bench.max_over_ranks(10.0 + rank, ws)
        bench.barrier(ws)
        with open(os.path.join(result_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{total!r} {slowest!r} {len(mine)}\n")
    finally:
        dist.destroy_process_group()


SPLIT_SEED = 0x5EED0013


def _split_shapes():
    from viprs_b200 import synth
    return synth.uneven_batch_shapes(24, SPLIT_SEED, wmin=48, wmax=700)


def _thumb_digest(i, shape):
    from oracle import oracle as O
    from viprs_b200 import synth
    img = synth.smooth_u8(*shape, SPLIT_SEED * 1000 + i, device="cpu").numpy()
    out = O.thumbnail(img, "fitbox", 64, 64)
    return out.shape, zlib.crc32(out.tobytes())


def _split_rank_main(rank, ws, port, result_dir):
    import datetime
    import json

    from viprs_b200 import api
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        shapes = _split_shapes()
        mine = api.partition_batch(shapes, ws)[rank]
        local = {i: _thumb_digest(i, shapes[i]) for i in mine}
        gathered = [None] * ws
        dist.all_gather_object(gathered, local)
        if rank == 0:
            union = {}
            for part in gathered:
                assert not set(part) & set(union), "an image was thumbnailed on two ranks"
                union.update(part)
            with open(os.path.join(result_dir, "union.json"), "w") as f:
                json.dump({str(k): [list(v[0]), v[1]] for k, v in union.items()}, f)
    finally:
        dist.destroy_process_group()


def test_split_batch_union_equals_single_process(tmp_path):
    import json
    ws = 2
    mp.spawn(_split_rank_main, args=(ws, _free_port(), str(tmp_path)), nprocs=ws, join=True)
    union = json.load(open(tmp_path / "union.json"))
    shapes = _split_shapes()
    assert sorted(int(k) for k in union) == list(range(len(shapes)))
    for i, shape in enumerate(shapes):
        out_shape, crc = _thumb_digest(i, shape)
        assert union[str(i)] == [list(out_shape), crc], f"image {i} differs between the split and one process"


def test_partition_is_a_balanced_cover():
    from viprs_b200 import api, synth
    shapes = synth.uneven_batch_shapes(512, 0x5EED0003)
    for parts in (1, 2, 3, 8):
        split = api.partition_batch(shapes, parts)
        flat = sorted(i for p in split for i in p)
        assert flat == list(range(len(shapes)))
        loads = [sum(shapes[i][0] * shapes[i][1] * shapes[i][2] for i in p) for p in split]
        biggest = max(h * w * b for h, w, b in shapes)
        # largest-first greedy: parts differ by at most one image's bytes
        assert max(loads) - min(loads) <= biggest
    assert api.partition_batch([], 2) == [[], []]
    with pytest.raises(ValueError):
        api.partition_batch(shapes, 0)


def test_two_ranks_gloo(tmp_path):
    ws = 2
    mp.spawn(_rank_main, args=(ws, _free_port(), str(tmp_path)), nprocs=ws, join=True)
    from viprs_b200 import synth
    import bench
    shapes = synth.uneven_batch_shapes(512, bench.BATCH_SEED)
    want_total = sum(h * w for h, w, _ in shapes) / 1e6
    rows = [open(tmp_path / f"rank{r}.txt").read().split() for r in range(ws)]
    for total, slowest, _ in rows:
        assert float(total) == pytest.approx(want_total, rel=1e-12)
        assert float(slowest) == 11.0
    assert sum(int(r[2]) for r in rows) == len(shapes)
