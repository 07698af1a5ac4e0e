"""pikgpu_frame_set_ac_device: device AC planes in the context's own layout
(stride Bx * 64, consecutive planes) are read in place, others are copied.
Both give the host upload's result bit for bit; in place, a change of the
caller's buffer between calls shows in the next reconstruction, also when
that reconstruction is a graph replay."""

import numpy as np
import pytest

from pik_b200 import native, synthetic

pytestmark = pytest.mark.gpu


def _host_result(frame, ac=None):
    ctx = native.Context(0, form="split_bf16")
    try:
        ctx.begin(frame)
        ctx.set_ac(ac)
        return ctx.reconstruct(linear=True)[0]
    finally:
        ctx.close()


def test_in_place_and_copied_device_ac():
    import torch
    frame = synthetic.make_frame(1030, 530, seed=8)
    by, bx = frame.blocks
    want = _host_result(frame)
    ac = torch.from_numpy(np.ascontiguousarray(frame.quantized_ac)).cuda()
    # A padded layout (stride Bx * 64 + 64): copied.
    padded = torch.zeros((3, by, bx * 64 + 64), dtype=torch.int16,
                         device="cuda")
    padded[:, :, :bx * 64] = ac
    ctx = native.Context(0, form="split_bf16")
    try:
        ctx.begin(frame)
        ctx.set_ac_device([padded[c].data_ptr() for c in range(3)],
                          bx * 64 + 64)
        np.testing.assert_array_equal(ctx.reconstruct(linear=True)[0], want)
        # The context's layout: read in place. Same output buffer each
        # call, so the second call captures a graph and the third replays it.
        ctx.set_ac_device([ac[c].data_ptr() for c in range(3)], bx * 64)
        out = torch.empty((3, frame.ysize, frame.xsize), device="cuda")
        for _ in range(3):
            ctx.reconstruct_device(out.data_ptr(), frame.xsize)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(out.cpu().numpy(), want)
        # Change the caller's buffer: the next (replayed) result follows it.
        changed = frame.quantized_ac.copy()
        changed[:, ::3] = 0
        ac.copy_(torch.from_numpy(changed))
        torch.cuda.synchronize()
        ctx.reconstruct_device(out.data_ptr(), frame.xsize)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(),
                                      _host_result(frame, changed))
    finally:
        ctx.close()
