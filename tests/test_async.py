"""Asynchronous reconstruction (pikgpu_reconstruct_async + pikgpu_wait):
frames alternated over two contexts, so that one frame's copies overlap the
other's kernels, must come out exactly as from the blocking call; a context
with work in flight refuses every call but pikgpu_wait."""

import ctypes

import numpy as np
import pytest

from pik_b200 import native, synthetic

pytestmark = pytest.mark.gpu


def blocking(frame, form):
    ctx = native.Context(0, form=form)
    try:
        ctx.begin(frame)
        ctx.set_ac()
        return ctx.reconstruct(linear=True)[0]
    finally:
        ctx.close()


@pytest.mark.parametrize("form", ["fp32", "split_bf16"])
def test_two_contexts_pipelined_equal_blocking(form):
    import torch
    frames = [synthetic.make_frame(640, 360, seed=30 + i, qf_median=12.0)
              for i in range(5)]
    want = [blocking(f, form) for f in frames]
    ctxs = [native.Context(0, form=form) for _ in range(2)]
    outs = [torch.empty((3, 360, 640), dtype=torch.float32).pin_memory()
            for _ in range(2)]
    acs = [torch.from_numpy(f.quantized_ac).pin_memory() for f in frames]
    got = [None] * len(frames)
    pending = [None, None]
    try:
        for i, f in enumerate(frames):
            k = i % 2
            c = ctxs[k]
            c.wait()
            if pending[k] is not None:
                got[pending[k]] = outs[k].numpy().copy()
            c.begin(f)
            planes = (ctypes.c_void_p * 3)(
                *[acs[i][p].data_ptr() for p in range(3)])
            c._check(c.L.pikgpu_frame_set_ac(c.h, planes, f.xsize // 8 * 64))
            outs[k].fill_(float("nan"))
            c.reconstruct_async([outs[k][p].data_ptr() for p in range(3)],
                                f.xsize)
            pending[k] = i
            # In flight: every call but wait is refused.
            with pytest.raises(native.PikGpuError) as e:
                c.begin(f)
            assert e.value.code == -4
        for k, c in enumerate(ctxs):
            c.wait()
            c.wait()  # nothing pending: returns at once
            got[pending[k]] = outs[k].numpy().copy()
        for g, w in zip(got, want):
            np.testing.assert_array_equal(g, w)
    finally:
        for c in ctxs:
            c.close()
