"""The oracle against the reference compiled from its own sources, run live
on fresh bitstreams. CPU only.

Generator images of ragged sizes are encoded by the reference encoder at
distances 0.5 to 3, which gives mixed blocks, adaptive quant fields, CfL and
the EPF. The reference's scalar build decodes each bitstream to the
reconstruction boundary and runs its own stages on it. The FP32
restatement must then give:
- DC and the dequantised AC bit for bit;
- IDCT and the gaborish guide source within 2e-6;
- linear output within 2e-5 on the [0,1] scale (reference value / 255),
  given the reference's EPF decisions (u8 guide, per-block sigma).

With its own decisions, only rounding-boundary flips of the u8 guide are
allowed (the guide sources agree to 2e-6). They are at most 2e-4 of the
guide bytes, and no per-block sigma flips."""

import numpy as np
import pytest

from oracle import decisions, oraclepy, refpy
from pik_b200 import synthetic

pytestmark = pytest.mark.skipif(
    not (oraclepy.available() and refpy.available("scalar")
         and refpy.available("avx2")),
    reason="oracle or reference build (oracle/_ref) not built")

CASES = [(200, 136, 0.5, 1), (333, 201, 2.0, 2), (129, 67, 3.0, 3),
         (520, 72, 1.0, 4)]


@pytest.mark.parametrize("w,h,distance,seed", CASES)
def test_oracle_matches_live_reference(w, h, distance, seed):
    img = synthetic.srgb8_to_linear255(synthetic.make_image(w, h, seed=seed))
    bs = refpy.encode(img, distance, flavour="avx2")
    fz = refpy.Frozen(bs, flavour="scalar")
    stages = ("dc", "dequant_ac", "idct", "smoothed", "linear")
    ref, _ = fz.run_stages(threads=1, want=stages)
    frame = fz.frame()
    assert frame.have_ar
    o = oraclepy.run(frame, precision=32, want=stages, export_decisions=True)
    np.testing.assert_array_equal(o["dc"], ref["dc"])
    np.testing.assert_array_equal(o["dequant_ac"], ref["dequant_ac"])
    assert np.abs(o["idct"] - ref["idct"]).max() <= 2e-6
    assert np.abs(o["smoothed"] - ref["smoothed"]).max() <= 2e-6
    g, s = decisions.frame_decisions(ref["smoothed"], frame.raw_quant_field,
                                     frame.ac_strategy,
                                     frame.ar_sigma_lut_ids)
    np.testing.assert_array_equal(o["sigma"], s)
    assert (o["guide"] != g).mean() <= 2e-4
    o2 = oraclepy.run(frame, precision=32, want=("linear",), guide=g, sigma=s)
    assert np.abs(o2["linear"] - ref["linear"]).max() / 255 <= 2e-5


def _transform(fn, t, inv, x, istride, shape_out, ostride):
    out = np.zeros(shape_out, np.float32)
    xx = np.ascontiguousarray(x, np.float32)
    assert fn(t, inv, xx.ctypes.data, istride, out.ctypes.data, ostride) == 0
    return out


@pytest.mark.parametrize("t", range(9))
def test_transforms_match_live_reference(t):
    """TransformToPixels / TransformFromPixels (pik/ac_strategy.cc:531-848)
    of all nine types on seeded random blocks, magnitudes 1e-3 to 1e3,
    against the reference's scalar build. The reference computes the DCTs
    with butterflies, the restatement with dense matrices: within 2e-6 of
    the block's largest value. IDENTITY and DCT2X2 are sums and
    differences in the same order: bit for bit."""
    L, R = oraclepy.lib(), refpy.lib("scalar")
    rng = np.random.default_rng(100 + t)
    cov = {4: 2, 5: 4}.get(t, 1)
    n = 8 * cov
    for _ in range(20):
        scale = 10.0 ** rng.uniform(-3, 3)
        coef = (rng.standard_normal((cov, 64 * cov)) * scale).astype(
            np.float32)
        pix = (rng.standard_normal((n, n)) * scale).astype(np.float32)
        for inv, x, istride, shape, ostride in (
                (1, coef, 64 * cov, (n, n), n),
                (0, pix, n, (cov, 64 * cov), 64 * cov)):
            got = _transform(L.pikoracle_transform_f32, t, inv, x, istride,
                             shape, ostride)
            ref = _transform(R.pikref_transform, t, inv, x, istride, shape,
                             ostride)
            if t in (1, 2):  # IDENTITY, DCT2X2
                np.testing.assert_array_equal(got, ref)
            else:
                assert np.abs(got - ref).max() <= 2e-6 * float(
                    np.abs(ref).max())


def test_epf_weights_match_live_reference():
    """WeightFast + MulTable (pik/epf_target.cc:300-413) for every sigma
    the filter uses (kMinSigma 16 to kMaxSigma 672) and patch SADs from 0
    to 3060 in steps of 7, against the reference's scalar build: bit for
    bit."""
    L, R = oraclepy.lib(), refpy.lib("scalar")
    for sigma in range(16, 673):
        for sad in range(0, 3061, 7):
            assert (L.pikoracle_epf_weight(sigma, sad) ==
                    R.pikref_epf_weight(sigma, sad)), (sigma, sad)


@pytest.mark.parametrize("t", range(9))
@pytest.mark.parametrize("which", range(4))
def test_lf_helpers_match_live_reference(t, which):
    """LowestFrequenciesFromDC, DC2x2FromLowestFrequencies,
    DC2x2FromLowFrequencies and LowFrequenciesFromDC2x2
    (pik/ac_strategy.cc:850-1056) on seeded random 8x32 inputs, against the
    reference's scalar build: within 2e-6 of the largest output value."""
    L, R = oraclepy.lib(), refpy.lib("scalar")
    rng = np.random.default_rng(1000 + 10 * t + which)
    for _ in range(5):
        src = (rng.standard_normal((8, 32)) *
               10.0 ** rng.uniform(-2, 3)).astype(np.float32)
        got = np.zeros_like(src)
        ref = np.zeros_like(src)
        L.pikoracle_lf_helper_f32(t, which, src.ctypes.data, 32,
                                  got.ctypes.data, 32)
        R.pikref_lf_helper(t, which, src.ctypes.data, 32, ref.ctypes.data,
                           32)
        assert np.abs(got - ref).max() <= 2e-6 * max(
            1e-30, float(np.abs(ref).max()))


@pytest.mark.parametrize("sigma", [16, 90, 672])
def test_fixed_sigma_epf_matches_live_reference(sigma):
    """The decoder's fixed-sigma EPF (DecompressParams::epf_sigma,
    pik/pik_frame.cc:112-115; Filter, pik/epf_target.cc:1342-1386): every
    block filtered with one sigma. The restatement on the reference's guide
    must give its EPF output and linear output within 2e-5 (the bounds of
    the adaptive case), and the reference's own full decode with the
    override must equal its stage-by-stage run."""
    img = synthetic.srgb8_to_linear255(synthetic.make_image(200, 136,
                                                            seed=sigma))
    bs = refpy.encode(img, 1.5, flavour="avx2")
    fz = refpy.Frozen(bs, flavour="scalar")
    fz.set_fixed_sigma(sigma)
    ref, _ = fz.run_stages(threads=1, want=("smoothed", "epf", "linear"))
    frame = fz.frame()
    assert frame.epf_enable_adaptive == 0 and frame.epf_sigma == sigma
    g, _ = decisions.guide_and_stretch(ref["smoothed"])
    by, bx = frame.blocks
    s = np.full((by, bx), sigma, np.int32)
    o = oraclepy.run(frame, precision=32, want=("epf", "linear"), guide=g,
                     sigma=s)
    assert np.abs(o["epf"] - ref["epf"]).max() <= 2e-6
    assert np.abs(o["linear"] - ref["linear"]).max() / 255 <= 2e-5
    # Without injected decisions the restatement takes the same sigma.
    o2 = oraclepy.run(frame, precision=32, want=("linear",),
                      export_decisions=True)
    np.testing.assert_array_equal(o2["sigma"], s)
    full = refpy.decode(bs, frame.xsize, frame.ysize, threads=1,
                        epf_sigma=sigma)
    np.testing.assert_array_equal(full, ref["linear"])
