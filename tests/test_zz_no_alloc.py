"""The allocation-free DC entry point (pikgpu_dc_reconstruct_noalloc)
against the DC stage of the context path (pikgpu_reconstruct), through the C
ABI. It runs the FP32 form's DC kernels in the same order, so its contract
with an FP32-form context is bit-equality. The tensor-core forms' DC EPF uses
fused multiply-adds; against a split-BF16 context the bound is 2e-6 on the
DC scale, the tolerance the parity tests use for the DC stage. Named to run
after the other GPU tests, and it also passes alone in a fresh process."""

import numpy as np
import pytest

from pik_b200 import native, synthetic

pytestmark = pytest.mark.gpu

TOL = 2e-6


def _context_dc(frame, form="fp32"):
    ctx = native.Context(0, keep_stages=True, form=form)
    try:
        ctx.begin(frame)
        ctx.set_ac()
        ctx.reconstruct(linear=True)
        return ctx.stage("dc")
    finally:
        ctx.close()


def _dc_dequant(frame):
    return np.array([frame.dequant_table[frame.dequant_offsets[c]]
                     for c in range(3)], np.float32)


@pytest.mark.parametrize("size", [(1030, 530), (64, 40), (4096, 4096)])
def test_noalloc_dc_matches_context_twice(size):
    import torch
    w, h = size
    frame = synthetic.make_frame(w, h, seed=w + 3 * h, qf_median=12.0)
    by, bx = frame.blocks
    want = _context_dc(frame)
    qdc = torch.from_numpy(np.ascontiguousarray(frame.quantized_dc)).cuda()
    outs = []
    for _ in range(2):  # two calls in a row on fresh output buffers
        out = torch.full((3, by, bx), float("nan"), device="cuda")
        native.dc_reconstruct_noalloc(
            qdc.data_ptr(), bx, by, frame.global_scale, frame.quant_dc,
            _dc_dequant(frame), frame.ytox_dc, frame.ytob_dc, out.data_ptr())
        torch.cuda.synchronize()
        outs.append(out.cpu().numpy())
    split = _context_dc(frame, "split_bf16")
    for got in outs:
        assert np.isfinite(got).all()
        np.testing.assert_array_equal(got, want)
        assert np.abs(got - split).max() <= TOL


def test_noalloc_rejects_oversized_and_bad_arguments():
    import torch
    qdc = torch.zeros((3, 513, 8), dtype=torch.int16, device="cuda")
    out = torch.zeros((3, 513, 8), device="cuda")
    mul = np.ones(3, np.float32)
    with pytest.raises(native.PikGpuError) as e:
        native.dc_reconstruct_noalloc(qdc.data_ptr(), 8, 513, 3065, 16, mul,
                                      128, 0, out.data_ptr())
    assert e.value.code == -1 and "limit" in str(e.value)
    host = np.zeros((3, 8, 8), np.int16)
    with pytest.raises(native.PikGpuError) as e:
        native.dc_reconstruct_noalloc(host.ctypes.data, 8, 8, 3065, 16, mul,
                                      128, 0, out.data_ptr())
    assert e.value.code == -1
    with pytest.raises(native.PikGpuError) as e:
        native.dc_reconstruct_noalloc(qdc.data_ptr(), 8, 8, 0, 16, mul,
                                      128, 0, out.data_ptr())
    assert e.value.code == -1


def test_noalloc_calls_take_no_device_memory():
    """After the first call, further calls leave the free device memory
    unchanged."""
    import torch
    frame = synthetic.make_frame(512, 512, seed=9)
    by, bx = frame.blocks
    qdc = torch.from_numpy(np.ascontiguousarray(frame.quantized_dc)).cuda()
    out = torch.empty((3, by, bx), device="cuda")
    args = (qdc.data_ptr(), bx, by, frame.global_scale, frame.quant_dc,
            _dc_dequant(frame), frame.ytox_dc, frame.ytob_dc, out.data_ptr())
    native.dc_reconstruct_noalloc(*args)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        native.dc_reconstruct_noalloc(*args)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
