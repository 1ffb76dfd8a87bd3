"""viprs_reduce_noalloc: the reduce entry point for callers that cannot allocate
device memory (a host framework whose allocator owns the GPU's memory, a
plugin inside another program's processing callback, a loop that must not
let cudaMalloc/cudaFree synchronise the device).  It keeps its tables in one
static device array instead of allocating them.

Checked through the C ABI against viprs_reduce, the allocating entry point,
with the tolerance the parity tests use (u8 bit-exact; f32 floored relative
error <= 1e-5), on calls made back to back on one stream, so that each call
runs on the scratch contents the previous one left.  This file is collected
last on purpose: the first call on a device sets the scratch up.
"""
import numpy as np
import pytest

from gpu_helpers import assert_same, rand_image, to_dev, to_host

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from viprs_b200 import _native as N  # noqa: E402
from viprs_b200 import api  # noqa: E402

SCRATCH_LIMIT = 11  # VIPRS_ERR_SCRATCH_LIMIT

CASES = [
    # (height, width, bands, dtype, hfactor, vfactor, kernel)
    (480, 640, 3, np.uint8, 2.0, 2.0, "lanczos3"),
    (207, 301, 4, np.float32, 2.7027, 1.5, "lanczos3"),
    (700, 900, 3, np.uint8, 3.3, 30.0, "lanczos3"),
    (123, 77, 1, np.uint16, 1.25, 4.0, "bicubic"),
]


def _out_like(t, hf, vf):
    h, w, b = t.shape
    return torch.full((api.reduce_output_len(vf, h), api.reduce_output_len(hf, w), b), 7, dtype=t.dtype,
                      device=t.device)


def _noalloc(t, out, hf, vf, kernel):
    return N.lib().viprs_reduce_noalloc(api.image(t), api.image(out), float(hf), float(vf), api._kernel(kernel),
                                        api._stream())


def test_reduce_noalloc_matches_reduce_on_back_to_back_calls():
    rng = np.random.default_rng(0x5EED)
    inputs = [to_dev(rand_image(rng, h, w, b, dt)) for (h, w, b, dt, _, _, _) in CASES]
    outs = [_out_like(t, c[4], c[5]) for t, c in zip(inputs, CASES)]
    # every call enqueued back to back: each one overwrites the scratch the previous call used
    for t, out, c in zip(inputs, outs, CASES):
        assert _noalloc(t, out, c[4], c[5], c[6]) == 0
    again = _out_like(inputs[0], CASES[0][4], CASES[0][5])
    assert _noalloc(inputs[0], again, CASES[0][4], CASES[0][5], CASES[0][6]) == 0
    for t, out, c in zip(inputs, outs, CASES):
        ref = api.reduce(t, c[4], c[5], c[6])
        assert_same(to_host(out), to_host(ref), c[3])
    assert_same(to_host(again), to_host(outs[0]), CASES[0][3])


def test_reduce_noalloc_intermediate_plane():
    # a 181-tap vertical pass does not fit the fused tile: the call stages the
    # horizontal pass's plane in the scratch after the tables
    h, w, b, dt, hf, vf, k = CASES[2]
    plan = api.PipelineBuilder(w, h, b, torch.uint8).reduce(hf, vf, k).build()
    assert plan.workspace_bytes > 0
    t = to_dev(rand_image(np.random.default_rng(9), h, w, b, dt))
    out = _out_like(t, hf, vf)
    assert _noalloc(t, out, hf, vf, k) == 0
    assert_same(to_host(out), to_host(api.reduce(t, hf, vf, k)), dt)


def test_reduce_noalloc_at_the_scratch_limit():
    # the tables plus the intermediate plane grow with the height: find the
    # tallest image that still fits the array, check its result against
    # viprs_reduce, and that one row more is refused
    w, b, hf, vf, k = 900, 3, 3.3, 30.0, "lanczos3"
    rng = np.random.default_rng(17)

    def status(h):
        t = torch.zeros((h, w, b), dtype=torch.uint8, device="cuda")
        return _noalloc(t, _out_like(t, hf, vf), hf, vf, k)

    lo, hi = 700, 8000
    assert status(lo) == 0 and status(hi) == SCRATCH_LIMIT
    while hi - lo > 1:
        mid = (lo + hi) // 2
        if status(mid) == 0:
            lo = mid
        else:
            hi = mid
    plan = api.PipelineBuilder(w, lo, b, torch.uint8).reduce(hf, vf, k).build()
    assert plan.workspace_bytes > (3 << 20), "the plane dominates the scratch at the limit"
    t = to_dev(rand_image(rng, lo, w, b, np.uint8))
    out = _out_like(t, hf, vf)
    assert _noalloc(t, out, hf, vf, k) == 0
    assert_same(to_host(out), to_host(api.reduce(t, hf, vf, k)), np.uint8)
    assert status(lo + 1) == SCRATCH_LIMIT


def test_reduce_noalloc_rejects_work_beyond_its_scratch():
    # a 2,000,000-pixel-wide row needs ~6.7 MB of position tables: more than the 4 MiB array
    t = torch.zeros((1, 2_000_000, 1), dtype=torch.uint8, device="cuda")
    out = _out_like(t, 1.5, 1.0)
    assert _noalloc(t, out, 1.5, 1.0, "lanczos3") == SCRATCH_LIMIT
    torch.cuda.synchronize()
    assert bool((out == 7).all()), "a rejected call must not touch the output"
    # argument errors are the same statuses as viprs_reduce's
    small = torch.zeros((8, 8, 3), dtype=torch.uint8, device="cuda")
    assert _noalloc(small, _out_like(small, 2.0, 2.0), 0.5, 2.0, "lanczos3") == 1
    assert _noalloc(small, _out_like(small, 2.0, 2.0), 2.0, 2.0, "lbb") == 7
