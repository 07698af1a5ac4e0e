"""Parity of high-quality frames with highlights, the frames of the
8192x8192 workload (pik_b200.synthetic.make_highlight_frame: distance 0.5,
quant field up to 64, AC doubled, 1% of the area at 4x light), through the
C ABI at 1030x530 (ragged blocks and groups).

The FP32 form is bit-identical to the FP32 oracle at every stage. The
split-BF16 form is held to the bounds of the other tensor-core tests, on
the FP32 form's EPF and clamp decisions: max-abs 2e-5 against FP64 on the
[0,1]-normalised linear output (reference value / 255) and 8-bit sRGB
within 1 LSB."""

import pytest

from pik_b200 import synthetic
from tests.test_gpu_parity import assert_bitexact_vs_oracle, run_gpu
from tests.test_split_bf16 import check_against_fp64

pytestmark = pytest.mark.gpu


def frame():
    return synthetic.make_highlight_frame(1030, 530, seed=5)


def test_highlight_frame_fp32_bitexact():
    f = frame()
    assert_bitexact_vs_oracle(f, run_gpu(f))


def test_highlight_frame_split_bf16_vs_fp64():
    check_against_fp64(frame(), "split_bf16")
