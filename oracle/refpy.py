"""ctypes access to the reference decoder built from google/pik's own
sources (oracle/_ref/libpikref_{avx2,scalar}.so, see oracle/Makefile).

Test infrastructure only: used by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference leg of bench.py as the checker and the baseline,
never as the measured product.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from pik_b200 import layout

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")

_libs: dict[str, ctypes.CDLL] = {}

STAGES = ("dc", "dequant_ac", "idct", "smoothed", "epf", "ar", "pre_opsin",
          "linear")


def lib_path(flavour: str) -> str:
    return os.path.join(REF_DIR, f"libpikref_{flavour}.so")


def available(flavour: str = "scalar") -> bool:
    return os.path.exists(lib_path(flavour))


def lib(flavour: str = "scalar") -> ctypes.CDLL:
    if flavour in _libs:
        return _libs[flavour]
    L = ctypes.CDLL(lib_path(flavour), mode=ctypes.RTLD_LOCAL)
    P = ctypes.c_void_p
    L.pikref_last_error.restype = ctypes.c_char_p
    L.pikref_flavour.restype = ctypes.c_char_p
    L.pikref_encode.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, ctypes.POINTER(P),
                                ctypes.POINTER(ctypes.c_size_t)]
    L.pikref_free.argtypes = [P]
    L.pikref_decode.argtypes = [P, ctypes.c_size_t, ctypes.c_int, P,
                                ctypes.c_size_t]
    L.pikref_linear_to_xyb.argtypes = [P, ctypes.c_size_t, P]
    L.pikref_frozen_from_bitstream.restype = P
    L.pikref_frozen_from_bitstream.argtypes = [P, ctypes.c_size_t,
                                               ctypes.c_int, ctypes.c_int]
    L.pikref_frozen_free.argtypes = [P]
    L.pikref_frozen_scalars.argtypes = [P, P, P]
    L.pikref_frozen_copy.argtypes = [P, ctypes.c_char_p, P, ctypes.c_size_t]
    L.pikref_run_stages.argtypes = [P, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_void_p),
                                    ctypes.POINTER(ctypes.c_double)]
    L.pikref_frozen_set_ac.argtypes = [P, P, ctypes.c_size_t]
    L.pikref_frozen_set_fixed_sigma.argtypes = [P, ctypes.c_int]
    L.pikref_encode_pnm.argtypes = [P, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, P,
                                    ctypes.c_size_t,
                                    ctypes.POINTER(ctypes.c_size_t)]
    L.pikref_decode_epf_sigma.argtypes = [P, ctypes.c_size_t, ctypes.c_int,
                                          ctypes.c_int, P, ctypes.c_size_t]
    L.pikref_frozen_encode_dct8.restype = P
    L.pikref_frozen_encode_dct8.argtypes = [P, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_float, ctypes.c_int]
    L.pikref_opsin_inverse_matrix.argtypes = [P]
    L.pikref_transform.argtypes = [ctypes.c_int, ctypes.c_int, P,
                                   ctypes.c_size_t, P, ctypes.c_size_t]
    L.pikref_lf_helper.argtypes = [ctypes.c_int, ctypes.c_int, P,
                                   ctypes.c_size_t, P, ctypes.c_size_t]
    L.pikref_epf_weight.restype = ctypes.c_float
    L.pikref_epf_weight.argtypes = [ctypes.c_int, ctypes.c_int]
    L.pikref_opsin_inverse_matrix.argtypes = [P]
    L.pikref_gaborish.argtypes = [ctypes.c_int, P, ctypes.c_int, ctypes.c_int,
                                  P]
    _libs[flavour] = L
    return L


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def encode(linear: np.ndarray, distance: float, *, ar: int = -1,
           gaborish: int = -1, fast: bool = False, threads: int = 0,
           flavour: str = "avx2") -> bytes:
    """Reference encoder on a (3, H, W) linear-sRGB image (0..255 scale)."""
    L = lib(flavour)
    img = np.ascontiguousarray(linear, dtype=np.float32)
    out = ctypes.c_void_p()
    n = ctypes.c_size_t()
    rc = L.pikref_encode(_ptr(img), img.shape[2], img.shape[1],
                         float(distance), ar, gaborish, int(fast), threads,
                         ctypes.byref(out), ctypes.byref(n))
    if rc != 0:
        raise RuntimeError(L.pikref_last_error().decode())
    data = ctypes.string_at(out, n.value)
    L.pikref_free(out)
    return data


def linear_to_xyb(linear: np.ndarray, flavour: str = "scalar") -> np.ndarray:
    """The reference's LinearToXyb on (3, H, W) linear planes (0..255)."""
    L = lib(flavour)
    lin = np.ascontiguousarray(linear, dtype=np.float32)
    out = np.empty_like(lin)
    L.pikref_linear_to_xyb(_ptr(lin), lin[0].size, _ptr(out))
    return out


def decode(bitstream: bytes, xsize: int, ysize: int, *, threads: int = 0,
           flavour: str = "scalar", epf_sigma: int = 0) -> np.ndarray:
    """Full reference PikToPixels to (3, H, W) linear planes; epf_sigma > 0
    is the decoder's fixed-sigma EPF override (DecompressParams)."""
    L = lib(flavour)
    out = np.zeros((3, ysize, xsize), np.float32)
    buf = ctypes.create_string_buffer(bitstream, len(bitstream))
    rc = L.pikref_decode_epf_sigma(ctypes.cast(buf, ctypes.c_void_p),
                                   len(bitstream), threads, epf_sigma,
                                   _ptr(out), out.size)
    if rc != 0:
        raise RuntimeError(L.pikref_last_error().decode())
    return out


def encode_pnm(linear: np.ndarray, bits: int, srgb: bool = True,
               flavour: str = "scalar") -> bytes:
    """The reference's PNM writer (EncodeImagePNM) on (3, H, W) linear
    planes (0..255): PPM for 8/16 bits, PFM for 32."""
    L = lib(flavour)
    img = np.ascontiguousarray(linear, dtype=np.float32)
    _, h, w = img.shape
    cap = 64 + 3 * w * h * max(1, bits // 8)
    out = np.zeros(cap, np.uint8)
    n = ctypes.c_size_t()
    rc = L.pikref_encode_pnm(_ptr(img), w, h, bits, int(srgb), _ptr(out),
                             cap, ctypes.byref(n))
    if rc != 0:
        raise RuntimeError(L.pikref_last_error().decode())
    return out[:n.value].tobytes()


def encode_dct8(linear: np.ndarray, quant: float, *, gaborish: int = 2,
                flavour: str = "scalar") -> "Frozen":
    """All-DCT8, EPF-off frame from the reference encoder's coefficient stage
    with a uniform quant field (the compressed_image_test route)."""
    L = lib(flavour)
    img = np.ascontiguousarray(linear, dtype=np.float32)
    h = L.pikref_frozen_encode_dct8(_ptr(img), img.shape[2], img.shape[1],
                                    float(quant), gaborish)
    if not h:
        raise RuntimeError(L.pikref_last_error().decode())
    return Frozen(None, flavour=flavour, handle=h)


class Frozen:
    """A bitstream decoded up to the reconstruction boundary by the
    reference's own decoding functions."""

    def __init__(self, bitstream: bytes | None, *, override_ar: int = -1,
                 override_gaborish: int = -1, flavour: str = "scalar",
                 handle=None):
        self.flavour = flavour
        self.L = lib(flavour)
        if handle is not None:
            self.h = handle
        else:
            buf = ctypes.create_string_buffer(bitstream, len(bitstream))
            self.h = self.L.pikref_frozen_from_bitstream(
                ctypes.cast(buf, ctypes.c_void_p), len(bitstream),
                override_ar, override_gaborish)
        if not self.h:
            raise RuntimeError(self.L.pikref_last_error().decode())
        ints = np.zeros(32, np.int64)
        floats = np.zeros(8, np.float32)
        self.L.pikref_frozen_scalars(self.h, _ptr(ints), _ptr(floats))
        self.ints, self.floats = ints, floats
        self.xsize, self.ysize = int(ints[0]), int(ints[1])
        self.bx, self.by = int(ints[2]), int(ints[3])
        self.tx, self.ty = int(ints[19]), int(ints[20])

    def __del__(self):
        if getattr(self, "h", None):
            self.L.pikref_frozen_free(self.h)
            self.h = None

    def _get(self, name: str, shape, dtype) -> np.ndarray:
        a = np.zeros(shape, dtype)
        rc = self.L.pikref_frozen_copy(self.h, name.encode(), _ptr(a),
                                       a.nbytes)
        if rc != 0:
            raise RuntimeError(f"copy {name}: {rc}")
        return a

    def frame(self) -> layout.Frame:
        i = self.ints
        bx, by, tx, ty = self.bx, self.by, self.tx, self.ty
        return layout.Frame(
            xsize=self.xsize, ysize=self.ysize, flags=int(i[4]),
            gaborish=int(i[5]), predict_lf=int(i[6]), predict_hf=int(i[7]),
            have_ar=int(i[8]), epf_enable_adaptive=int(i[9]),
            epf_sigma=int(i[10]), epf_use_sharpened=int(i[11]),
            global_scale=int(i[12]), quant_dc=int(i[13]),
            ytox_dc=int(i[14]), ytob_dc=int(i[15]),
            ytox_map=self._get("ytox_map", (ty, tx), np.int32),
            ytob_map=self._get("ytob_map", (ty, tx), np.int32),
            ac_strategy=self._get("ac_strategy", (by, bx), np.uint8),
            raw_quant_field=self._get("raw_quant_field", (by, bx), np.int32),
            ar_sigma_lut_ids=self._get("ar_sigma_lut_ids", (by, bx),
                                       np.uint8),
            quantized_dc=self._get("quantized_dc", (3, by, bx), np.int16),
            quantized_ac=self._get("quantized_ac", (3, by, bx * 64),
                                   np.int16),
            dequant_table=self._get("dequant_table", (int(i[16]),),
                                    np.float32),
            dequant_offsets=self._get("dequant_offsets",
                                      (int(i[17]) * 7 * 3,), np.uint32),
            dequant_control_field=self._get("dequant_control_field",
                                            (ty, tx), np.uint8),
            dequant_map=self._get("dequant_map", (16, 256), np.uint8))

    def set_fixed_sigma(self, sigma: int) -> None:
        """The decoder's fixed-sigma EPF override (sigma > 0)."""
        if self.L.pikref_frozen_set_fixed_sigma(self.h, sigma) != 0:
            raise ValueError(f"fixed sigma {sigma}")
        self.ints[9], self.ints[10] = 0, sigma

    def dc_smoothed(self) -> np.ndarray:
        return self._get("dc_smoothed", (3, self.by, self.bx), np.float32)

    def set_ac(self, ac: np.ndarray) -> None:
        a = np.ascontiguousarray(ac, np.int16)
        if self.L.pikref_frozen_set_ac(self.h, _ptr(a), a.size) != 0:
            raise ValueError("AC shape mismatch")

    def run_stages(self, threads: int = 0, want=STAGES):
        """Reference reconstruction; returns {stage: (3, h, w) array} and the
        elapsed seconds."""
        px, py = self.bx * 8, self.by * 8
        shapes = {"dc": (3, self.by, self.bx),
                  "dequant_ac": (3, self.by, self.bx * 64),
                  "idct": (3, py, px), "smoothed": (3, py, px),
                  "epf": (3, py, px), "ar": (3, py, px),
                  "pre_opsin": (3, self.ysize, self.xsize),
                  "linear": (3, self.ysize, self.xsize)}
        out = {}
        ptrs = (ctypes.c_void_p * 8)()
        for k, name in enumerate(STAGES):
            if name in want:
                out[name] = np.zeros(shapes[name], np.float32)
                ptrs[k] = out[name].ctypes.data
        secs = ctypes.c_double()
        rc = self.L.pikref_run_stages(self.h, threads, ptrs,
                                      ctypes.byref(secs))
        if rc != 0:
            raise RuntimeError(self.L.pikref_last_error().decode())
        return out, secs.value

    def dictionary_changed(self) -> bool:
        return bool(self.L.pikref_dictionary_changed())
