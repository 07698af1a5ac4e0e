"""ctypes access to the C++ restatement of the reconstruction path
(oracle/_ref/libpikoracle.so built from oracle/pik_oracle.cc).

Test infrastructure only (tests/, __graft_entry__.smoke(), bench.py's CPU
baseline): the checker, never the measured product.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from pik_b200 import abi, layout

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libpikoracle.so")
_lib = None

STAGES = ("dc", "dequant_ac", "idct", "smoothed", "epf", "ar", "pre_opsin",
          "linear", "srgb8")


class Decisions(ctypes.Structure):
    _fields_ = [("guide", ctypes.c_void_p), ("sigma", ctypes.c_void_p),
                ("dc_guide", ctypes.c_void_p), ("dc_sigma", ctypes.c_void_p),
                ("clamp_tape", ctypes.c_void_p)]


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_LOCAL)
        P = ctypes.c_void_p
        for fn in (L.pikoracle_run_f32, L.pikoracle_run_f64):
            fn.argtypes = [P, P, ctypes.POINTER(P), P, P, P]
        L.pikoracle_transform_f64.argtypes = [ctypes.c_int, ctypes.c_int, P,
                                              ctypes.c_size_t, P,
                                              ctypes.c_size_t]
        L.pikoracle_transform_f32.argtypes = [ctypes.c_int, ctypes.c_int, P,
                                              ctypes.c_size_t, P,
                                              ctypes.c_size_t]
        L.pikoracle_lf_helper_f32.argtypes = [ctypes.c_int, ctypes.c_int, P,
                                              ctypes.c_size_t, P,
                                              ctypes.c_size_t]
        L.pikoracle_epf_weight.restype = ctypes.c_float
        L.pikoracle_epf_weight.argtypes = [ctypes.c_int, ctypes.c_int]
        L.pikoracle_opsin_inverse_matrix.argtypes = [P]
        L.pikoracle_dct_table.argtypes = [ctypes.c_int, ctypes.c_int, P]
        L.pikoracle_adjoint_f64.argtypes = [P, P, P, P, P, P, P, P, P]
        _lib = L
    return _lib


def stage_shapes(frame: layout.Frame) -> dict:
    by, bx = frame.blocks
    return {"dc": (3, by, bx), "dequant_ac": (3, by, bx * 64),
            "idct": (3, by * 8, bx * 8), "smoothed": (3, by * 8, bx * 8),
            "epf": (3, by * 8, bx * 8), "ar": (3, by * 8, bx * 8),
            "pre_opsin": (3, frame.ysize, frame.xsize),
            "linear": (3, frame.ysize, frame.xsize),
            "srgb8": (frame.ysize, frame.xsize, 3)}


def run(frame: layout.Frame, *, precision: int = 32, want=STAGES,
        guide=None, sigma=None, dc_guide=None, dc_sigma=None,
        clamp_tape=None, export_decisions: bool = False):
    """Runs the restatement. Returns {stage: array}; with export_decisions,
    also 'guide' (3, H+12, W+12) uint8 and 'sigma' (By, Bx) int32."""
    L = lib()
    packed = abi.PackedFrame(frame)
    ftype = np.float32 if precision == 32 else np.float64
    shapes = stage_shapes(frame)
    out = {}
    ptrs = (ctypes.c_void_p * 9)()
    for k, name in enumerate(STAGES):
        if name in want:
            dt = np.uint8 if name == "srgb8" else ftype
            out[name] = np.zeros(shapes[name], dt)
            ptrs[k] = out[name].ctypes.data
    dec = Decisions()
    keep = []
    for field, arr, dt in (("guide", guide, np.uint8),
                           ("sigma", sigma, np.int32),
                           ("dc_guide", dc_guide, np.uint8),
                           ("dc_sigma", dc_sigma, np.int32),
                           ("clamp_tape", clamp_tape, np.uint8)):
        if arr is not None:
            a = np.ascontiguousarray(arr, dt)
            keep.append(a)
            setattr(dec, field, a.ctypes.data)
    by, bx = frame.blocks
    gout = sout = None
    if export_decisions:
        gout = np.zeros((3, by * 8 + 12, bx * 8 + 12), np.uint8)
        sout = np.zeros((by, bx), np.int32)
    fn = L.pikoracle_run_f32 if precision == 32 else L.pikoracle_run_f64
    rc = fn(packed.ref, packed.ac.ctypes.data, ptrs, ctypes.byref(dec),
            gout.ctypes.data if gout is not None else None,
            sout.ctypes.data if sout is not None else None)
    if rc != 0:
        raise RuntimeError(f"oracle failed: {rc}")
    if export_decisions:
        out["guide"], out["sigma"] = gout, sout
    return out


def adjoint(frame: layout.Frame, target: np.ndarray, *, guide=None,
            sigma=None, dc_guide=None, dc_sigma=None, clamp_tape=None,
            ac_dequant=None, ar_scale=None, grads: bool = True):
    """FP64 adjoint (pik_adjoint.inc): returns (loss, grad_ac, grad_qf);
    grad_ac is (3, By, Bx*64) (dequantised AC, frame layout), grad_qf
    (By, Bx). `target` is (3, ysize, xsize) XYB. EPF decisions should be
    the base point's; `ac_dequant` / `ar_scale` move the forward off the
    integer lattice for finite differences."""
    L = lib()
    packed = abi.PackedFrame(frame)
    by, bx = frame.blocks
    dec = Decisions()
    keep = []
    for field, arr, dt in (("guide", guide, np.uint8),
                           ("sigma", sigma, np.int32),
                           ("dc_guide", dc_guide, np.uint8),
                           ("dc_sigma", dc_sigma, np.int32),
                           ("clamp_tape", clamp_tape, np.uint8)):
        if arr is not None:
            a = np.ascontiguousarray(arr, dt)
            keep.append(a)
            setattr(dec, field, a.ctypes.data)
    t = np.ascontiguousarray(target, np.float64)
    assert t.shape == (3, frame.ysize, frame.xsize)
    acd = None if ac_dequant is None else np.ascontiguousarray(ac_dequant,
                                                               np.float64)
    ars = None if ar_scale is None else np.ascontiguousarray(ar_scale,
                                                             np.float64)
    loss = np.zeros(1, np.float64)
    g_ac = np.zeros((3, by, bx * 64), np.float64) if grads else None
    g_qf = np.zeros((by, bx), np.float64) if grads else None
    rc = L.pikoracle_adjoint_f64(
        packed.ref, packed.ac.ctypes.data, ctypes.byref(dec),
        acd.ctypes.data if acd is not None else None,
        ars.ctypes.data if ars is not None else None, t.ctypes.data,
        loss.ctypes.data, g_ac.ctypes.data if grads else None,
        g_qf.ctypes.data if grads else None)
    if rc != 0:
        raise RuntimeError(f"oracle adjoint failed: {rc}")
    return float(loss[0]), g_ac, g_qf
