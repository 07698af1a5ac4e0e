"""ctypes mirror of the C ABI in include/pikgpu.h."""

from __future__ import annotations

import ctypes

import numpy as np

from . import layout

P = ctypes.c_void_p
U32 = ctypes.c_uint32
I32 = ctypes.c_int32


class FrameParams(ctypes.Structure):
    """struct pikgpu_frame_params."""
    _fields_ = [
        ("xsize", U32), ("ysize", U32),
        ("flags", U32), ("gaborish", U32),
        ("predict_lf", U32), ("predict_hf", U32),
        ("have_adaptive_reconstruction", U32),
        ("epf_enable_adaptive", U32), ("epf_sigma", U32),
        ("epf_use_sharpened", U32),
        ("global_scale", I32), ("quant_dc", I32),
        ("dequant_table", P), ("dequant_table_size", U32),
        ("dequant_offsets", P), ("num_dequant_tables", U32),
        ("dequant_control_field", P), ("dequant_map", P),
        ("ytox_map", P), ("ytob_map", P),
        ("ytox_dc", I32), ("ytob_dc", I32),
        ("ac_strategy", P), ("raw_quant_field", P), ("ar_sigma_lut_ids", P),
        ("quantized_dc", P),
    ]


class PackedFrame:
    """A Frame's arrays made contiguous plus the FrameParams pointing at
    them (keeps the arrays alive as long as the params are used)."""

    def __init__(self, frame: layout.Frame):
        self.frame = frame
        c = np.ascontiguousarray
        self.arrays = dict(
            dequant_table=c(frame.dequant_table, np.float32),
            dequant_offsets=c(frame.dequant_offsets, np.uint32),
            dequant_control_field=c(frame.dequant_control_field, np.uint8),
            dequant_map=c(frame.dequant_map, np.uint8),
            ytox_map=c(frame.ytox_map, np.int32),
            ytob_map=c(frame.ytob_map, np.int32),
            ac_strategy=c(frame.ac_strategy, np.uint8),
            raw_quant_field=c(frame.raw_quant_field, np.int32),
            ar_sigma_lut_ids=c(frame.ar_sigma_lut_ids, np.uint8),
            quantized_dc=c(frame.quantized_dc, np.int16),
        )
        self.ac = c(frame.quantized_ac, np.int16)
        a = self.arrays
        p = FrameParams()
        p.xsize, p.ysize = frame.xsize, frame.ysize
        p.flags = frame.flags
        p.gaborish = frame.gaborish
        p.predict_lf, p.predict_hf = frame.predict_lf, frame.predict_hf
        p.have_adaptive_reconstruction = frame.have_ar
        p.epf_enable_adaptive = frame.epf_enable_adaptive
        p.epf_sigma = frame.epf_sigma
        p.epf_use_sharpened = frame.epf_use_sharpened
        p.global_scale, p.quant_dc = frame.global_scale, frame.quant_dc
        p.dequant_table = a["dequant_table"].ctypes.data
        p.dequant_table_size = a["dequant_table"].size
        p.dequant_offsets = a["dequant_offsets"].ctypes.data
        p.num_dequant_tables = a["dequant_offsets"].size // 21
        for k in ("dequant_control_field", "dequant_map", "ytox_map",
                  "ytob_map", "ac_strategy", "raw_quant_field",
                  "ar_sigma_lut_ids", "quantized_dc"):
            setattr(p, k, a[k].ctypes.data)
        p.ytox_dc, p.ytob_dc = frame.ytox_dc, frame.ytob_dc
        self.params = p

    @property
    def ref(self):
        return ctypes.byref(self.params)
