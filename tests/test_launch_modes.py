"""One frame through every launch mode of the library gives the same bytes.

The transform and clamp classes other than DCT8 run as a chain of
programmatic dependent launches on one side stream, and the EPF and the
clamp's active-block pass are programmatic dependents of the kernels before
them on the main stream. Those launches keep only the orders the kernels'
data need (the classes' blocks are disjoint; the EPF waits for the guide
range before it reads it). They are used kernel by kernel, in graph replay
and in the batch (each frame on one stream, the frames as branches of one
graph). The profiling mode launches every kernel on one stream after the
one before it, with ordinary launches. Results must be bit-identical in
every mode and form: the FP32 form is deterministic, and so are the
tensor-core forms (their sums have a fixed order)."""

import numpy as np
import pytest
import torch

from pik_b200 import native, synthetic

pytestmark = pytest.mark.gpu


def frame_with_every_class():
    f = synthetic.make_frame(1536, 1032, seed=21, qf_median=12.0)
    types = set(int(v) >> 4 for v in np.unique(f.ac_strategy))
    assert types == set(range(9)), types
    return f


def run_context(frame, form, **kw):
    ctx = native.Context(0, form=form, **kw)
    try:
        ctx.begin(frame)
        ctx.set_ac()
        first = ctx.reconstruct(linear=True, srgb8=True)
        second = ctx.reconstruct(linear=True, srgb8=True)
        return first, second, ctx.graph_stats()
    finally:
        ctx.close()


def run_batch(frames, form):
    dev = torch.device("cuda", 0)
    b = native.Batch(len(frames), 0, form=form)
    try:
        for c, f in zip(b.frames, frames):
            c.begin(f)
            c.set_ac()
        outs = [torch.empty((3, f.ysize, f.xsize), device=dev) for f in frames]
        b.reconstruct_device([o.data_ptr() for o in outs],
                             [f.xsize for f in frames])
        torch.cuda.synchronize()
        return [o.cpu().numpy() for o in outs]
    finally:
        b.close()


@pytest.mark.parametrize("form", ["fp32", "split_bf16", "split_bf16x3"])
def test_every_launch_mode_gives_the_same_bytes(form):
    frame = frame_with_every_class()
    (lin_d, rgb_d), (lin_g, rgb_g), stats = run_context(frame, form)
    assert stats["last_replayed"], stats
    (lin_p, rgb_p), _, _ = run_context(frame, form, profile=True)
    other = synthetic.make_frame(700, 500, seed=22, qf_median=12.0)
    lin_b, lin_o = run_batch([frame, other], form)
    np.testing.assert_array_equal(lin_g, lin_d)
    np.testing.assert_array_equal(rgb_g, rgb_d)
    np.testing.assert_array_equal(lin_p, lin_d)
    np.testing.assert_array_equal(rgb_p, rgb_d)
    np.testing.assert_array_equal(lin_b, lin_d)
    (want_o, _), _, _ = run_context(other, form, profile=True)
    np.testing.assert_array_equal(lin_o, want_o)
