"""The device's bounded mbarrier waits, made to run out: the tensor-core
kernels' wait on MMA completions and the EPF's wait on its TMA tile copies.

PIKGPU_OPT_TC_WAIT_POLLS = 0 gives every first wait zero polls, so it runs
out at once, as a wait on a completion that never comes would after its
limit. The kernel then drains what is in flight (MMAs, the tile copy) with
a second bounded wait, records the error and stops; nothing hangs and
nothing faults. The host must report PIKGPU_ERR_CUDA, and the context must
stay usable: with the default limit restored, the same frame reconstructs
bit-identically to a fresh context's result. In the FP32 form only the
EPF's TMA wait exists (its interior tiles are copied by the TMA)."""

import numpy as np
import pytest

from pik_b200 import native, synthetic

pytestmark = pytest.mark.gpu


def _frame():
    return synthetic.make_frame(520, 264, seed=11,
                                shares={"DCT32X32": 0.4, "DCT16X16": 0.4,
                                        "DCT": 0.2})


def _reconstruct(ctx, frame):
    ctx.begin(frame)
    ctx.set_ac()
    return ctx.reconstruct(linear=True)[0]


@pytest.mark.parametrize("form", ["split_bf16", "split_bf16x3", "fp32"])
def test_wait_runs_out_then_context_recovers(form):
    frame = _frame()
    fresh = native.Context(0, form=form)
    try:
        want = _reconstruct(fresh, frame)
    finally:
        fresh.close()
    ctx = native.Context(0, form=form)
    try:
        ctx.set_option(native.OPT_TC_WAIT_POLLS, 0)
        with pytest.raises(native.PikGpuError) as e:
            _reconstruct(ctx, frame)
        assert e.value.code == -3 and "timed out" in str(e.value)
        if form == "fp32":
            assert "TMA" in str(e.value)
        ctx.set_option(native.OPT_TC_WAIT_POLLS, -1)
        got = _reconstruct(ctx, frame)
        np.testing.assert_array_equal(got, want)
    finally:
        ctx.close()


def test_poll_option_rejects_negative_values():
    ctx = native.Context(0)
    try:
        with pytest.raises(native.PikGpuError) as e:
            ctx.set_option(native.OPT_TC_WAIT_POLLS, -2)
        assert e.value.code == -1
    finally:
        ctx.close()
