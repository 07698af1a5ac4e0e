"""Linear sRGB -> XYB, as the reference encoder forms the opsin image it
compresses (OpsinDynamicsImage / LinearToXyb, pik/opsin_image.cc:25-47,
with OpsinAbsorbance, pik/opsin_image.h:23-30, the constants of
pik/opsin_params.h:18-49 and ApproxCubeRoot, pik/approx_cube_root.h:18-51).

An encoder that tunes a frame against its source with pikgpu_adjoint needs
the source in the domain the decoder reconstructs before OpsinToLinear;
this is that transform, in float32 with each operation rounded in the
reference's order (the reference is compiled without contraction), so the
result is bit-identical to the reference's (checked against it in
tests/test_xyb_cpu.py)."""

from __future__ import annotations

import numpy as np

_F = np.float32
# kOpsinAbsorbanceMatrix / kOpsinAbsorbanceBias: double constants divided by
# kScale = 255 in double, then rounded to float.
_MIX = np.array([0.29956550340058319, 0.63373087833825936,
                 0.077705617820981968, 0.22158691104574774,
                 0.68491388044116142, 0.096254234043612538,
                 0.20062661225219422, 0.070366199217588729,
                 0.5571760754215358], np.float64) / 255.0
_MIX = _MIX.astype(_F)
_BIAS = (np.array([0.26786006338144885, 0.24494032763907073,
                   0.14255999980363571], np.float64) / 255.0).astype(_F)
_SCALE_R = _F(1.0)
_SCALE_G = _F(2.0) - _SCALE_R
_ONE_THIRD = _F(1.0) / _F(3.0)


def _cube_root(y: np.ndarray) -> np.ndarray:
    """ApproxCubeRoot: the bit-pattern initial guess 0x2a50f200 + bits / 3
    (integer division; y >= 0 here) and two Newton steps."""
    bits = y.view(np.int32)
    x = (np.int32(0x2a50f200) + bits // np.int32(3)).astype(np.int32)
    x = x.view(_F)
    for _ in range(2):
        x = _ONE_THIRD * (_F(2.0) * x + y / (x * x))
    return x


def linear_to_xyb(linear: np.ndarray) -> np.ndarray:
    """(3, H, W) linear sRGB on the 0..255 scale -> (3, H, W) XYB float32."""
    r, g, b = (np.asarray(p, dtype=_F) for p in linear)
    mixed = []
    for k in range(3):
        m = _MIX[3 * k] * r + _MIX[3 * k + 1] * g
        m = m + _MIX[3 * k + 2] * b
        m = m + _BIAS[k]
        mixed.append(_cube_root(np.maximum(_F(0.0), m).astype(_F)))
    x = (_SCALE_R * mixed[0] - _SCALE_G * mixed[1]) * _F(0.5)
    y = (_SCALE_R * mixed[0] + _SCALE_G * mixed[1]) * _F(0.5)
    return np.stack([x, y, mixed[2]]).astype(_F)
