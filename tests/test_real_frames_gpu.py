"""Reference-encoded frames heavy in DCT32X32, through the C ABI.

The committed fixtures are encoded at distance 1, where the reference
encoder picks no DCT32X32. These cases encode generator images (12
sinusoids, 20 rectangles, noise sigma 3) at distance 0.5 (37% of the cells
in DCT32X32) and 3.0 (72%) with the reference compiled here. The
reference's scalar build decodes them to the reconstruction boundary and
runs its own stages. The GPU then gives:
- DC and dequantised AC bit for bit; IDCT and the guide source within 2e-6;
- every stage bit-identical to the FP32 oracle;
- linear output within 2e-5 of the reference on the [0,1] scale (reference
  value / 255) given the reference's EPF decisions, and 8-bit sRGB within
  1 LSB of the exact encoding of the reference's output;
- with its own decisions, u8 guide flips on at most 2e-4 of the bytes and
  no per-block sigma flips."""

import os

import numpy as np
import pytest

from oracle import decisions, refpy
from pik_b200 import synthetic
from tests import golden_cases
from tests.test_gpu_parity import assert_bitexact_vs_oracle, run_gpu
from tests.test_split_bf16 import check_against_fp64

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not (refpy.available("scalar")
                            and refpy.available("avx2")),
                       reason="reference build (oracle/_ref) not present"),
]


@pytest.mark.parametrize("w,h,distance,seed", [(512, 384, 0.5, 7),
                                               (384, 256, 3.0, 8)])
def test_dct32_heavy_reference_frame(w, h, distance, seed):
    img = synthetic.srgb8_to_linear255(synthetic.make_image(
        w, h, seed=seed, sinusoids=12, rectangles=20, noise_sigma=3.0))
    bs = refpy.encode(img, distance, flavour="avx2",
                      threads=os.cpu_count() or 1)
    fz = refpy.Frozen(bs, flavour="scalar")
    ref, _ = fz.run_stages(threads=1, want=("dc", "dequant_ac", "idct",
                                            "smoothed", "linear"))
    frame = fz.frame()
    assert ((frame.ac_strategy >> 4) == 5).mean() >= 0.3  # DCT32X32 cells
    gpu = run_gpu(frame)
    np.testing.assert_array_equal(gpu["dc"], ref["dc"])
    np.testing.assert_array_equal(gpu["dequant_ac"], ref["dequant_ac"])
    assert np.abs(gpu["idct"] - ref["idct"]).max() <= 2e-6
    assert np.abs(gpu["smoothed"] - ref["smoothed"]).max() <= 2e-6
    assert_bitexact_vs_oracle(frame, gpu)
    g, s = decisions.frame_decisions(ref["smoothed"], frame.raw_quant_field,
                                     frame.ac_strategy,
                                     frame.ar_sigma_lut_ids)
    np.testing.assert_array_equal(gpu["sigma"], s)
    assert (gpu["guide"] != g).mean() <= 2e-4
    gpu2 = run_gpu(frame, guide=g, sigma=s, keep=False)
    assert np.abs(gpu2["linear"] - ref["linear"]).max() / 255 <= 2e-5
    lsb = np.abs(gpu2["srgb8"].transpose(2, 0, 1).astype(np.int32) -
                 golden_cases.srgb8_exact(ref["linear"]))
    assert lsb.max() <= 1
    # The tensor-core forms, whose DCT32X32 transforms and clamp run on
    # tcgen05, against FP64 on the FP32 form's decisions.
    for form in ("split_bf16", "split_bf16x3"):
        check_against_fp64(frame, form)


def test_fixed_sigma_reference_frame():
    """A reference-encoded frame decoded with the decoder's fixed-sigma EPF
    override (DecompressParams::epf_sigma, pik/pik_frame.cc:112-115): the
    GPU on the reference's guide is within 2e-5 of the reference's own
    full decode with the override, and bit-identical to the FP32 oracle."""
    sigma = 120
    img = synthetic.srgb8_to_linear255(synthetic.make_image(
        400, 264, seed=12, sinusoids=12, rectangles=20, noise_sigma=3.0))
    bs = refpy.encode(img, 1.0, flavour="avx2", threads=os.cpu_count() or 1)
    fz = refpy.Frozen(bs, flavour="scalar")
    fz.set_fixed_sigma(sigma)
    ref, _ = fz.run_stages(threads=1, want=("smoothed", "linear"))
    full = refpy.decode(bs, fz.xsize, fz.ysize, threads=1, epf_sigma=sigma)
    np.testing.assert_array_equal(full, ref["linear"])
    frame = fz.frame()
    gpu = run_gpu(frame)
    assert np.all(gpu["sigma"] == sigma)
    assert_bitexact_vs_oracle(frame, gpu)
    g, _ = decisions.guide_and_stretch(ref["smoothed"])
    by, bx = frame.blocks
    gpu2 = run_gpu(frame, guide=g, sigma=np.full((by, bx), sigma, np.int32),
                   keep=False)
    assert np.abs(gpu2["linear"] - full).max() / 255 <= 2e-5
