"""Batched reconstruction (pikgpu_batch_*): frames of uneven sizes run as
the branches of one captured CUDA graph. The graph replays the same kernels
with the same arguments as single-frame reconstruction, so every frame's
output must equal its single-frame output bit for bit, on the capturing
call and on replays; changing a frame must re-capture."""

import numpy as np
import pytest

from pik_b200 import native, synthetic

pytestmark = pytest.mark.gpu

SIZES = [(1030, 530), (256, 256), (8, 8), (600, 1100), (13, 7)]


def single(frame, form):
    ctx = native.Context(0, form=form)
    try:
        ctx.begin(frame)
        ctx.set_ac()
        return ctx.reconstruct(linear=True)[0]
    finally:
        ctx.close()


def gpu_outputs(frames):
    import torch
    return [torch.full((3, f.ysize, f.xsize), float("nan"), device="cuda")
            for f in frames]


@pytest.mark.parametrize("form", ["fp32", "split_bf16"])
def test_batch_equals_single_frames(form):
    frames = [synthetic.make_frame(w, h, seed=40 + i, qf_median=12.0)
              for i, (w, h) in enumerate(SIZES)]
    want = [single(f, form) for f in frames]
    b = native.Batch(len(frames), form=form)
    try:
        for c, f in zip(b.frames, frames):
            c.begin(f)
            c.set_ac()
        outs = gpu_outputs(frames)
        for _ in range(2):  # capture, then replay
            for o in outs:
                o.fill_(float("nan"))
            b.reconstruct_device([o.data_ptr() for o in outs],
                                 [f.xsize for f in frames])
            for o, w in zip(outs, want):
                np.testing.assert_array_equal(o.cpu().numpy(), w)
        assert b.capture_count() == 1
        assert b.launch_count() > len(frames) * 10

        # A new frame in slot 1 re-captures the graph.
        new = synthetic.make_frame(700, 300, seed=99, qf_median=9.0)
        b.frames[1].begin(new)
        b.frames[1].set_ac()
        frames[1] = new
        want[1] = single(new, form)
        outs = gpu_outputs(frames)
        b.reconstruct_device([o.data_ptr() for o in outs],
                             [f.xsize for f in frames])
        assert b.capture_count() == 2
        for o, w in zip(outs, want):
            np.testing.assert_array_equal(o.cpu().numpy(), w)
    finally:
        b.close()


def test_autotuned_batch_equals_single_frames():
    frames = [synthetic.make_frame(w, h, seed=60 + i, qf_median=12.0)
              for i, (w, h) in enumerate(SIZES)]
    want = [single(f, "split_bf16") for f in frames]
    b = native.Batch(len(frames), form="split_bf16")
    try:
        for c, f in zip(b.frames, frames):
            c.begin(f)
            c.set_ac()
        outs = gpu_outputs(frames)
        ptrs = [o.data_ptr() for o in outs]
        strides = [f.xsize for f in frames]
        shape = b.autotune(ptrs, strides)
        assert 1 <= shape["chains"] <= len(frames)
        assert shape["tc_ctas_per_sm"] in (1, 2, 4)
        for o in outs:
            o.fill_(float("nan"))
        b.reconstruct_device(ptrs, strides)
        for o, w in zip(outs, want):
            np.testing.assert_array_equal(o.cpu().numpy(), w)
    finally:
        b.close()


def test_batch_errors():
    b = native.Batch(2)
    try:
        with pytest.raises(native.PikGpuError) as e:
            b.reconstruct_device([0, 0], [8, 8])
        assert e.value.code in (-1, -4)
        f = synthetic.make_frame(64, 64, seed=1)
        for c in b.frames:
            c.begin(f)
            c.set_ac()
        with pytest.raises(native.PikGpuError) as e:
            b.reconstruct_device([0, 0], [64, 64])  # NULL outputs
        assert e.value.code == -1
    finally:
        b.close()
