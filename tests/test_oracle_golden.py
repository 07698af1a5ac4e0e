"""The oracle (C++ restatement, oracle/pik_oracle.cc) against golden outputs
of the reference compiled from its own sources. CPU only."""

import numpy as np
import pytest

from oracle import decisions, oraclepy
from tests import golden_cases

pytestmark = pytest.mark.skipif(not oraclepy.available(),
                                reason="oracle library not built")


def _transform(fn, t, inv, x, istride, shape_out, ostride, dtype):
    out = np.zeros(shape_out, dtype)
    xx = np.ascontiguousarray(x, dtype)
    rc = fn(t, inv, xx.ctypes.data, istride, out.ctypes.data, ostride)
    assert rc == 0
    return out


@pytest.mark.parametrize("t", range(9))
def test_transforms_match_reference(t):
    """AcStrategy::TransformToPixels / TransformFromPixels for all nine
    types (pik/ac_strategy.cc:531-848)."""
    p = golden_cases.probes()
    L = oraclepy.lib()
    cov = {4: 2, 5: 4}.get(t, 1)
    n = 8 * cov
    for i in range(4):
        ref = p[f"tr{t}_inv"][i]
        for fn, dt, tol in ((L.pikoracle_transform_f64, np.float64, 2e-6),
                            (L.pikoracle_transform_f32, np.float32, 2e-6)):
            got = _transform(fn, t, 1, p[f"tr{t}_coef"][i], 64 * cov, (n, n),
                             n, dt)
            scale = max(1.0, float(np.abs(ref).max()))
            assert np.abs(got - ref).max() <= tol * scale
            ref_f = p[f"tr{t}_fwd"][i]
            got_f = _transform(fn, t, 0, p[f"tr{t}_pix"][i], n,
                               (cov, 64 * cov), 64 * cov, dt)
            scale = max(1.0, float(np.abs(ref_f).max()))
            assert np.abs(got_f - ref_f).max() <= tol * scale


@pytest.mark.parametrize("t", range(9))
@pytest.mark.parametrize("which", range(4))
def test_lf_helpers_match_reference(t, which):
    """LowestFrequenciesFromDC, DC2x2FromLowestFrequencies,
    DC2x2FromLowFrequencies, LowFrequenciesFromDC2x2
    (pik/ac_strategy.cc:850-1056)."""
    p = golden_cases.probes()
    L = oraclepy.lib()
    src = p[f"lf{t}_{which}_in"]
    ref = p[f"lf{t}_{which}_out"]
    got = np.zeros_like(ref)
    if which == 2:
        # The reference reads the block's coefficient layout (rows of 8c).
        cov = {4: 2, 5: 4}.get(t, 1)
        blk = np.ascontiguousarray(src.reshape(-1)[:64 * cov * cov])
        blk = np.ascontiguousarray(src)
        L.pikoracle_lf_helper_f32(t, which, blk.ctypes.data, 32,
                                  got.ctypes.data, 32)
    else:
        s = np.ascontiguousarray(src)
        L.pikoracle_lf_helper_f32(t, which, s.ctypes.data, 32,
                                  got.ctypes.data, 32)
    assert np.abs(got - ref).max() <= 2e-6 * max(1.0, np.abs(ref).max())


def test_epf_weights_exact():
    """WeightFast + MulTable (pik/epf_target.cc:300-413) bit for bit."""
    p = golden_cases.probes()
    L = oraclepy.lib()
    got = np.array([[L.pikoracle_epf_weight(int(s), int(d))
                     for d in p["epf_sad"]] for s in p["epf_sigma"]],
                   np.float32)
    np.testing.assert_array_equal(got, p["epf_weight"])
    # Known answers the reference tests assert (pik/epf_target.cc:467-478):
    # weight 1 at SAD 0 and ~0.5 at SAD = sigma / 4.
    for i, s in enumerate(p["epf_sigma"]):
        if s % 4 == 0:
            assert abs(got[i, 0] - 1.0) <= 0.02


def test_opsin_inverse_matrix_exact():
    p = golden_cases.probes()
    got = np.zeros(9, np.float32)
    oraclepy.lib().pikoracle_opsin_inverse_matrix(got.ctypes.data)
    np.testing.assert_array_equal(got, p["opsin_inverse"])


def test_c1_dct8_epf_off():
    """Config-1 shape: all-DCT8, EPF off, gaborish on."""
    frame, ref = golden_cases.load("c1_256_dct8")
    o = oraclepy.run(frame, precision=32, want=("dc", "idct", "linear"))
    np.testing.assert_array_equal(o["dc"], ref["dc"])
    assert np.abs(o["idct"] - ref["idct"]).max() <= 2e-6
    # Float planes on the [0,1]-normalised scale (reference value / 255).
    assert np.abs(o["linear"] - ref["linear"]).max() / 255 <= 2e-5


def test_c2_mixed_epf_on():
    """Config-2 shape at 256x256: mixed blocks, adaptive qf, CfL, EPF."""
    frame, ref = golden_cases.load("c2_256_d1")
    o = oraclepy.run(frame, precision=32,
                     want=("dc", "idct", "smoothed", "linear"))
    np.testing.assert_array_equal(o["dc"], ref["dc"])
    assert np.abs(o["idct"] - ref["idct"]).max() <= 2e-6
    assert np.abs(o["smoothed"] - ref["smoothed"]).max() <= 2e-6
    # With the reference's own EPF decisions the arithmetic agrees to 2e-5.
    g, s = decisions.frame_decisions(ref["smoothed"], frame.raw_quant_field,
                                     frame.ac_strategy,
                                     frame.ar_sigma_lut_ids)
    o2 = oraclepy.run(frame, precision=32, want=("linear",), guide=g, sigma=s)
    assert np.abs(o2["linear"] - ref["linear"]).max() / 255 <= 2e-5
    # Own decisions: isolated guide-rounding flips only.
    d = np.abs(o["linear"] - ref["linear"]) / 255
    assert np.quantile(d, 0.999) <= 2e-5
    assert (d > 2e-5).mean() <= 1e-3


def test_fp64_oracle_close_to_fp32():
    """The FP64 restatement on the same EPF decisions stays within FP32
    rounding of the FP32 restatement (the accuracy oracle is sane)."""
    frame, _ = golden_cases.load("c1_256_dct8")
    o32 = oraclepy.run(frame, precision=32, want=("linear",))
    o64 = oraclepy.run(frame, precision=64, want=("linear",))
    assert np.abs(o32["linear"] - o64["linear"]).max() / 255 <= 1e-5
