"""Loading of the golden fixtures (tests/golden/, generated from the
reference by tests/golden/make_fixtures.py)."""

from __future__ import annotations

import os

import numpy as np

from pik_b200 import layout

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name: str):
    """Returns (Frame, {ref_stage: array}) for a golden case."""
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    kw = {}
    for k in z.files:
        if k.startswith("frame_"):
            v = z[k]
            kw[k[6:]] = v if v.ndim > 0 else int(v)
    frame = layout.Frame(**kw)
    refs = {k[4:]: z[k] for k in z.files if k.startswith("ref_")}
    if "bitstream" in z.files:
        refs["bitstream"] = z["bitstream"].tobytes()
    return frame, refs


def probes():
    return np.load(os.path.join(GOLDEN, "probes.npz"))


def srgb8_exact(linear255: np.ndarray) -> np.ndarray:
    """IEC 61966-2-1 encoding of linear samples (0..255 scale) to 8 bits,
    in float64: the value the reference's rational-polynomial TF_SRGB
    approximates."""
    x = np.clip(np.asarray(linear255, np.float64) / 255.0, 0.0, 1.0)
    e = np.where(x <= 0.0031308, 12.92 * x, 1.055 * x ** (1 / 2.4) - 0.055)
    return np.floor(np.clip(e, 0, 1) * 255.0 + 0.5).astype(np.int32)
