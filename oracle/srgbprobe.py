"""ctypes access to the sRGB probe (oracle/_ref/libsrgbprobe_{scalar,avx2}.so,
built from oracle/srgb_probe.cc): the reference's own TF_SRGB, compiled from
its source text, with ExternalImage::CopyTo's clamping and rounding.

Test infrastructure only: the checker of the device's sRGB output, never
the measured product.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_libs: dict[str, ctypes.CDLL] = {}


def lib_path(flavour: str) -> str:
    return os.path.join(_HERE, "_ref", f"libsrgbprobe_{flavour}.so")


def available(flavour: str = "scalar") -> bool:
    return os.path.exists(lib_path(flavour))


def encode(linear: np.ndarray, bits: int = 8,
           flavour: str = "scalar") -> np.ndarray:
    """(3, H, W) linear planes on the 0..255 scale -> (H, W, 3) sRGB
    samples (uint8 for 8 bits, uint16 for 16)."""
    if flavour not in _libs:
        L = ctypes.CDLL(lib_path(flavour), mode=ctypes.RTLD_LOCAL)
        L.srgbprobe_encode.argtypes = [ctypes.c_void_p, ctypes.c_size_t,
                                       ctypes.c_size_t, ctypes.c_int,
                                       ctypes.c_void_p]
        _libs[flavour] = L
    lin = np.ascontiguousarray(linear, np.float32)
    _, h, w = lin.shape
    out = np.zeros((h, w, 3), np.uint8 if bits == 8 else np.uint16)
    rc = _libs[flavour].srgbprobe_encode(lin.ctypes.data, w, h, bits,
                                         out.ctypes.data)
    if rc != 0:
        raise RuntimeError("srgbprobe_encode failed")
    return out
