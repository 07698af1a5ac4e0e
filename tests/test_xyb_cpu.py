"""pik_b200.xyb.linear_to_xyb (the encoder's opsin transform, used to build
adjoint targets from a source image) against the reference's own
LinearToXyb (pik/opsin_image.cc:34-47, compiled from its sources): bit for
bit, on random values (including negatives, which the transform clamps)
and on a generator image, for both reference builds."""

import numpy as np
import pytest

from oracle import refpy
from pik_b200 import synthetic, xyb


@pytest.mark.parametrize("flavour", ["scalar", "avx2"])
def test_linear_to_xyb_bit_exact(flavour):
    if not refpy.available(flavour):
        pytest.skip("reference build (oracle/_ref) not present")
    rng = np.random.default_rng(3)
    lin = rng.uniform(-20.0, 300.0, (3, 64, 97)).astype(np.float32)
    lin[:, 0, :8] = np.array([0.0, -0.0, 1e-30, 1e-6, 0.5, 255.0, 254.9,
                              1.0], np.float32)
    np.testing.assert_array_equal(xyb.linear_to_xyb(lin),
                                  refpy.linear_to_xyb(lin, flavour))
    img = synthetic.srgb8_to_linear255(
        synthetic.make_image(128, 96, seed=4, sinusoids=12, rectangles=20,
                             noise_sigma=3))
    np.testing.assert_array_equal(xyb.linear_to_xyb(img),
                                  refpy.linear_to_xyb(img, flavour))
