"""The C ABI library without a GPU: it loads, exports every entry point
include/pikgpu.h declares, and validates frames like pikgpu_frame_begin
(host-side checks only; no device call is made)."""

import ctypes
import os
import re

import numpy as np
import pytest

from pik_b200 import layout, native, synthetic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "pikgpu.h")).read()
    return sorted(set(re.findall(r"\b(pikgpu_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = native.lib()
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
        assert ctypes.cast(getattr(L, n), ctypes.c_void_p).value


def _frame(**over):
    f = synthetic.make_frame(64, 48, seed=5)
    for k, v in over.items():
        setattr(f, k, v)
    return f


def test_valid_frames_pass():
    for seed in range(3):
        f = synthetic.make_frame(200 + 37 * seed, 120 + 11 * seed, seed=seed)
        assert native.validate(f) == (0, "")


@pytest.mark.parametrize("mutate, code", [
    (lambda f: f.ac_strategy.__setitem__((0, 0), 9 << 4), -1),   # type > 8
    (lambda f: f.raw_quant_field.__setitem__((1, 1), 0), -1),    # qf < 1
    (lambda f: f.raw_quant_field.__setitem__((1, 1), 257), -1),  # qf > 256
    (lambda f: f.ar_sigma_lut_ids.__setitem__((0, 1), 2), -1),   # LUT id
    (lambda f: setattr(f, "flags", 4), -2),                      # noise
    # fixed sigma: 0 (copy) or in [kMinSigma, kMaxSigma] = [16, 672]
    (lambda f: (setattr(f, "epf_enable_adaptive", 0),
                setattr(f, "epf_sigma", 15)), -1),
    (lambda f: (setattr(f, "epf_enable_adaptive", 0),
                setattr(f, "epf_sigma", 673)), -1),
    (lambda f: setattr(f, "gaborish", 5), -1),
    (lambda f: setattr(f, "global_scale", 0), -1),
    (lambda f: setattr(f, "quant_dc", 300), -1),
    (lambda f: f.dequant_map.__setitem__((0, 0), 1), -1),        # table id
    (lambda f: f.dequant_control_field.__setitem__((0, 0), 16), -1),
])
def test_invalid_fields_rejected(mutate, code):
    f = _frame()
    mutate(f)
    rc, msg = native.validate(f)
    assert rc == code and msg


@pytest.mark.parametrize("sigma", [0, 16, 100, 672])
def test_fixed_sigma_epf_accepted(sigma):
    f = _frame(epf_enable_adaptive=0, epf_sigma=sigma)
    assert native.validate(f) == (0, "")


def test_misaligned_and_overlapping_transforms_rejected():
    f = _frame()
    acs = np.zeros_like(f.ac_strategy)  # all DCT8
    # DCT16 at an odd block position: unsupported.
    acs[1:3, 1:3] = np.array([[0x40, 0x41], [0x42, 0x43]], np.uint8)
    f.ac_strategy = acs
    rc, msg = native.validate(f)
    assert rc == -2 and "aligned" in msg
    acs = np.zeros_like(f.ac_strategy)
    acs[0, 0] = 0x41  # non-first sub-block without its first block
    f.ac_strategy = acs
    assert native.validate(f)[0] == -1
    f = synthetic.make_frame(64, 40, seed=5)  # 8 x 5 blocks
    acs = np.zeros_like(f.ac_strategy)
    acs[4, 4] = 0x50  # aligned DCT32 that would extend past the image
    f.ac_strategy = acs
    rc, msg = native.validate(f)
    assert rc == -1 and "past" in msg


def test_dequant_offsets_beyond_table_rejected():
    f = _frame()
    off = f.dequant_offsets.copy()
    off[5 * 3] = f.dequant_table.size - 10  # DCT32 needs 1024 floats
    f.dequant_offsets = off
    assert native.validate(f)[0] == -1


def test_empty_image_rejected():
    f = _frame()
    f.xsize = 0
    assert native.validate(f)[0] == -1


def test_default_dequant_table_matches_decoded_frames():
    from tests import golden_cases
    frame, _ = golden_cases.load("c2_256_d1")
    table, offsets = layout.default_dequant_table()
    np.testing.assert_array_equal(frame.dequant_table, table)
    np.testing.assert_array_equal(frame.dequant_offsets, offsets)


def test_frame_save_load_roundtrip(tmp_path):
    f = synthetic.make_frame(40, 24, seed=2)
    p = str(tmp_path / "f.npz")
    f.save(p)
    g = layout.Frame.load(p)
    for k in ("ac_strategy", "raw_quant_field", "quantized_ac",
              "quantized_dc", "ytox_map"):
        np.testing.assert_array_equal(getattr(f, k), getattr(g, k))
    assert g.global_scale == f.global_scale and g.xsize == f.xsize


@pytest.mark.parametrize("size", [(1, 1), (13, 7), (300, 200), (1030, 530)])
def test_highlight_frame_generator(size):
    """The high-quality highlight frames of the 8192x8192 workload: valid at
    the ABI, quant field within [6, 64], the highlight share reached, and
    deterministic for a seed."""
    w, h = size
    f = synthetic.make_highlight_frame(w, h, seed=5)
    assert native.validate(f)[0] == 0
    assert f.raw_quant_field.min() >= 6 and f.raw_quant_field.max() <= 64
    base = synthetic.make_frame(w, h, seed=5, qf_median=36.0, ac_scale=2.0,
                                qf_max=64)
    changed = (f.quantized_dc[1] != base.quantized_dc[1]).mean()
    if f.raw_quant_field.size >= 400:  # else one 2x2 rectangle is > 1%
        assert changed <= 0.05
    g = synthetic.make_highlight_frame(w, h, seed=5)
    np.testing.assert_array_equal(f.quantized_ac, g.quantized_ac)
    np.testing.assert_array_equal(f.quantized_dc, g.quantized_dc)


def test_highlight_frame_encoder_mix():
    """The reference encoder's distance-0.5 transform mix, as the 8192x8192
    workload's `--mix encoder` uses it: valid at the ABI and within 0.02 of
    the target shares."""
    f = synthetic.make_highlight_frame(
        1030, 530, seed=5, shares=synthetic.ENCODER_SHARES_D05)
    assert native.validate(f)[0] == 0
    types = f.ac_strategy >> 4
    for name, share in synthetic.ENCODER_SHARES_D05.items():
        got = float((types == layout.ACS_TYPES[name]).mean())
        assert abs(got - share) <= 0.02, (name, got, share)


def test_run_frame_arguments():
    """The command-line runner takes a frame file or a generated highlight
    frame (not both), optionally cropped."""
    from pik_b200 import run_frame
    a = run_frame.parse_args(["--highlight", "300", "200", "--mix",
                              "encoder", "--crop", "128", "64"])
    f = run_frame.load_frame(a)
    assert (f.xsize, f.ysize) == (128, 64)
    assert native.validate(f)[0] == 0
    for bad in ([], ["x.npz", "--highlight", "8", "8"]):
        with pytest.raises(SystemExit):
            run_frame.parse_args(bad)
