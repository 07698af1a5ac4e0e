"""Parity of the CUDA path (through the C ABI) with the reference and the
oracle. Tolerances: float planes on the [0,1]-normalised scale (reference
linear value / 255) within 2e-5 of the reference given the same EPF
decisions; bit-identical to the FP32 oracle (same operation order);
8-bit output within 1 LSB."""

import os

import numpy as np
import pytest

from oracle import decisions, oraclepy, refpy
from pik_b200 import layout, native, synthetic
from tests import golden_cases

pytestmark = pytest.mark.gpu

STAGES = ("dc", "dequant_ac", "idct", "smoothed", "epf", "ar", "pre_opsin")


def run_gpu(frame, *, guide=None, sigma=None, keep=True):
    ctx = native.Context(0, keep_stages=keep)
    try:
        ctx.begin(frame)
        ctx.set_ac()
        if guide is not None or sigma is not None:
            ctx.set_decisions(guide, sigma)
        lin, rgb = ctx.reconstruct(linear=True, srgb8=True)
        out = {"linear": lin, "srgb8": rgb}
        if keep:
            for k in STAGES:
                if k in ("smoothed", "epf", "ar") and not frame.have_ar:
                    continue
                out[k] = ctx.stage(k)
        if frame.have_ar:
            out["guide"], out["sigma"] = ctx.decisions()
        return out
    finally:
        ctx.close()


def assert_bitexact_vs_oracle(frame, gpu):
    o = oraclepy.run(frame, precision=32, export_decisions=bool(frame.have_ar))
    for k in STAGES + ("linear", "srgb8"):
        if k in gpu:
            np.testing.assert_array_equal(gpu[k], o[k], err_msg=k)
    if frame.have_ar:
        np.testing.assert_array_equal(gpu["guide"], o["guide"])
        np.testing.assert_array_equal(gpu["sigma"], o["sigma"])


def test_c1_dct8_epf_off():
    frame, ref = golden_cases.load("c1_256_dct8")
    gpu = run_gpu(frame)
    np.testing.assert_array_equal(gpu["dc"], ref["dc"])
    assert np.abs(gpu["idct"] - ref["idct"]).max() <= 2e-6
    assert np.abs(gpu["linear"] - ref["linear"]).max() / 255 <= 2e-5
    lsb = np.abs(gpu["srgb8"].transpose(2, 0, 1).astype(np.int32) -
                 golden_cases.srgb8_exact(ref["linear"]))
    assert lsb.max() <= 1
    assert_bitexact_vs_oracle(frame, gpu)


def test_c2_mixed_epf_on():
    frame, ref = golden_cases.load("c2_256_d1")
    gpu = run_gpu(frame)
    np.testing.assert_array_equal(gpu["dc"], ref["dc"])
    assert np.abs(gpu["idct"] - ref["idct"]).max() <= 2e-6
    assert np.abs(gpu["smoothed"] - ref["smoothed"]).max() <= 2e-6
    d = np.abs(gpu["linear"] - ref["linear"]) / 255
    assert np.quantile(d, 0.999) <= 2e-5 and (d > 2e-5).mean() <= 1e-3
    assert_bitexact_vs_oracle(frame, gpu)
    # Same discrete EPF decisions as the reference: arithmetic within 2e-5.
    g, s = decisions.frame_decisions(ref["smoothed"], frame.raw_quant_field,
                                     frame.ac_strategy,
                                     frame.ar_sigma_lut_ids)
    gpu2 = run_gpu(frame, guide=g, sigma=s, keep=False)
    assert np.abs(gpu2["linear"] - ref["linear"]).max() / 255 <= 2e-5
    lsb = np.abs(gpu2["srgb8"].transpose(2, 0, 1).astype(np.int32) -
                 golden_cases.srgb8_exact(ref["linear"]))
    assert lsb.max() <= 1


@pytest.mark.parametrize("name", list(layout.ACS_TYPES))
def test_every_transform_type_bitexact(name):
    """All nine AcStrategy types, including those the encoder never emits
    (LINES, DCT_NOHF, DCT4X4_NOHF), against the FP32 oracle."""
    shares = ({name: 1.0} if name not in ("DCT16X16", "DCT32X32")
              else {name: 0.9, "DCT": 0.1})
    frame = synthetic.make_frame(136, 104, seed=11, shares=shares,
                                 qf_median=9.0)
    assert_bitexact_vs_oracle(frame, run_gpu(frame))


@pytest.mark.parametrize("shares", [
    {"DCT2X2": 0.4, "IDENTITY": 0.3, "LINES": 0.3},
    {"DCT4X4": 0.5, "DCT4X4_NOHF": 0.5},
])
def test_many_small_blocks_bitexact(shares):
    """4225 small-transform blocks: more than the one-CTA-per-block forms of
    the DCT2X2 / IDENTITY / LINES inverse and clamp take (16 blocks per SM),
    so the one-thread-per-block-and-channel forms run; the frames above run
    the others."""
    frame = synthetic.make_frame(520, 520, seed=13, shares=shares,
                                 qf_median=9.0)
    assert_bitexact_vs_oracle(frame, run_gpu(frame))


@pytest.mark.parametrize("size", [(8, 8), (1, 1), (13, 7), (520, 9),
                                  (1030, 530), (64, 520)])
def test_sizes_and_group_borders(size):
    """Partial blocks, single-block images and frames crossing 512-pixel
    group boundaries (ragged groups)."""
    w, h = size
    frame = synthetic.make_frame(w, h, seed=w * 7 + h, qf_median=10.0)
    assert native.validate(frame)[0] == 0
    assert_bitexact_vs_oracle(frame, run_gpu(frame))


@pytest.mark.parametrize("variant", ["no_lf", "no_hf", "no_pred",
                                     "gaborish_off", "epf_off", "sharpened",
                                     "gaborish_1000", "lut1"])
def test_header_variants(variant):
    frame = synthetic.make_frame(200, 136, seed=3, qf_median=9.0)
    if variant in ("no_lf", "no_pred"):
        frame.predict_lf = 0
    if variant in ("no_hf", "no_pred"):
        frame.predict_hf = 0
    if variant == "gaborish_off":
        frame.gaborish = 0
    if variant == "gaborish_1000":
        frame.gaborish = 4
    if variant == "epf_off":
        frame.have_ar = 0
    if variant == "sharpened":
        frame.epf_use_sharpened = 1
    if variant == "lut1":
        frame.ar_sigma_lut_ids = np.ones_like(frame.ar_sigma_lut_ids)
    assert_bitexact_vs_oracle(frame, run_gpu(frame))


def test_group_upload_matches_frame_upload():
    frame = synthetic.make_frame(1100, 600, seed=4)
    by, bx = frame.blocks
    whole = run_gpu(frame, keep=False)["linear"]
    ctx = native.Context(0)
    try:
        ctx.begin(frame)
        gx = -(-frame.xsize // 512)
        for gi in range(frame.num_groups):
            x0, y0 = (gi % gx) * 64, (gi // gx) * 64
            ctx.set_group_ac(gi, frame.quantized_ac[:, y0:y0 + 64,
                                                    x0 * 64:(x0 + 64) * 64])
        lin, _ = ctx.reconstruct(linear=True)
    finally:
        ctx.close()
    np.testing.assert_array_equal(lin, whole)


def test_group_uploads_from_concurrent_threads():
    """Groups uploaded from several host threads at once, as pik's group
    threads decode them (pik/pik_frame.cc:1108-1135), give the same frame
    as one whole-frame upload. ctypes releases the GIL during each call, so
    the uploads overlap."""
    from concurrent.futures import ThreadPoolExecutor
    frame = synthetic.make_frame(2100, 1100, seed=6)
    whole = run_gpu(frame, keep=False)["linear"]
    gx = -(-frame.xsize // 512)
    parts = []
    for gi in range(frame.num_groups):
        x0, y0 = (gi % gx) * 64, (gi // gx) * 64
        parts.append(np.ascontiguousarray(
            frame.quantized_ac[:, y0:y0 + 64, x0 * 64:(x0 + 64) * 64]))
    ctx = native.Context(0)
    try:
        ctx.begin(frame)
        with ThreadPoolExecutor(max_workers=8) as pool:
            list(pool.map(lambda gi: ctx.set_group_ac(gi, parts[gi]),
                          range(frame.num_groups)))
        lin, _ = ctx.reconstruct(linear=True)
    finally:
        ctx.close()
    np.testing.assert_array_equal(lin, whole)


def test_errors_leave_context_usable():
    frame = synthetic.make_frame(64, 64, seed=1)
    ctx = native.Context(0)
    try:
        with pytest.raises(native.PikGpuError) as e:
            ctx.reconstruct()  # no frame yet
        assert e.value.code == -4
        bad = synthetic.make_frame(64, 64, seed=1)
        bad.raw_quant_field[0, 0] = 0
        with pytest.raises(native.PikGpuError) as e:
            ctx.begin(bad)
        assert e.value.code == -1
        ctx.begin(frame)
        with pytest.raises(native.PikGpuError):
            ctx.reconstruct()  # AC not supplied
        ctx.set_ac()
        lin, _ = ctx.reconstruct()
        assert np.isfinite(lin).all()
    finally:
        ctx.close()


@pytest.mark.skipif(not refpy.available("scalar"),
                    reason="reference build (oracle/_ref) not present")
def test_4k_real_frame_against_reference_and_fp64():
    """The config-2 workload itself (3840x2160, reference-encoded at
    distance 1) at full size. With the reference's own EPF decisions the GPU
    is within 2e-5 of the FP64 oracle everywhere; its few differences from
    the reference beyond 2e-5 are pixels where the reference's FP32 result
    is itself that far from FP64."""
    frame = layout.Frame.load(os.path.join(golden_cases.GOLDEN,
                                           "c2_4k_d1_frame.npz"))
    bs = open(os.path.join(golden_cases.GOLDEN, "c2_4k_d1.pik"), "rb").read()
    fz = refpy.Frozen(bs, flavour="scalar")
    st, _ = fz.run_stages(threads=os.cpu_count() or 1,
                          want=("smoothed", "linear"))
    gpu = run_gpu(frame, keep=False)
    d = np.abs(gpu["linear"] - st["linear"]) / 255
    assert np.quantile(d, 0.999) <= 2e-5 and (d > 2e-5).mean() <= 1e-3
    g, s = decisions.frame_decisions(st["smoothed"], frame.raw_quant_field,
                                     frame.ac_strategy,
                                     frame.ar_sigma_lut_ids)
    dg, ds = decisions.dc_decisions(frame)
    gpu2 = run_gpu(frame, guide=g, sigma=s, keep=False)
    o64 = oraclepy.run(frame, precision=64, want=("linear",), guide=g,
                       sigma=s, dc_guide=dg, dc_sigma=ds)["linear"]
    err_gpu = np.abs(gpu2["linear"] - o64) / 255
    err_ref = np.abs(st["linear"] - o64) / 255
    assert err_gpu.max() <= 2e-5
    diff = np.abs(gpu2["linear"] - st["linear"]) / 255
    assert np.quantile(diff, 0.99999) <= 2e-5
    # Where the two differ by more than 2e-5, most of the difference is the
    # reference's own rounding error (its distance from FP64).
    far = diff > 2e-5
    assert np.all(err_ref[far] >= 0.75 * diff[far])
    lsb = np.abs(gpu2["srgb8"].transpose(2, 0, 1).astype(np.int32) -
                 golden_cases.srgb8_exact(o64))
    assert lsb.max() <= 1


@pytest.mark.parametrize("sigma", [0, 16, 100, 672])
def test_fixed_sigma_epf_bitexact(sigma):
    """EpfParams::enable_adaptive = false (Filter, pik/epf_target.cc:
    1342-1386): every block filtered with one sigma, or copied when it is 0;
    every stage bit-identical to the FP32 oracle."""
    frame = synthetic.make_frame(264, 200, seed=sigma + 1, qf_median=9.0)
    frame.epf_enable_adaptive = 0
    frame.epf_sigma = sigma
    gpu = run_gpu(frame)
    assert np.all(gpu["sigma"] == sigma)
    assert_bitexact_vs_oracle(frame, gpu)
    if sigma == 0:
        np.testing.assert_array_equal(gpu["epf"], gpu["idct"])
