"""The output-format step on the device (pikgpu_encode_pnm): the PPM / PFM
file dpik writes (WriteOutput, pik/dpik.cc:196-223), against the
reference's own writer (EncodeImagePNM, pik/codec_pnm.cc:179-196,260-294,
compiled from its sources into oracle/_ref) run on the same linear planes.

The container, the byte order, the row order and the casts and rounding
of ExternalImage are the reference's own code; the sRGB transfer on the
reference side goes through the shim's colour management, the
reference's skip-lcms route. Both evaluate TF_SRGB with an exact square
root and division, so every byte must match (8 and 16 bits per sample in
sRGB and linear light, and 32-bit PFM). The 16-bit sRGB samples are also
checked against the reference's own TF_SRGB in its shipped AVX2 flavour
(oracle/srgb_probe.cc): within 1 LSB."""

import numpy as np
import pytest

from oracle import refpy, srgbprobe
from pik_b200 import native, synthetic
from tests import golden_cases

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not refpy.available("scalar"),
                       reason="reference build (oracle/_ref) not present"),
]


def _reconstruct(frame):
    ctx = native.Context(0)
    ctx.begin(frame)
    ctx.set_ac()
    lin, rgb = ctx.reconstruct(linear=True, srgb8=True)
    return ctx, lin, rgb


@pytest.mark.parametrize("bits", [8, 16, 32])
@pytest.mark.parametrize("srgb", [True, False])
def test_pnm_matches_reference_writer(bits, srgb):
    frame, _ = golden_cases.load("c2_256_d1")
    ctx, lin, rgb = _reconstruct(frame)
    try:
        got = ctx.encode_pnm(bits, srgb)
    finally:
        ctx.close()
    want = refpy.encode_pnm(lin, bits, srgb)
    assert got[:16] == want[:16]
    assert got == want
    if bits == 8 and srgb:
        # The body of the 8-bit sRGB file is the reconstruction's sRGB-8.
        assert got[-rgb.size:] == rgb.tobytes()


def test_pnm_ragged_frame_and_probe():
    frame = synthetic.make_frame(203, 77, seed=4)
    ctx, lin, _ = _reconstruct(frame)
    try:
        got = ctx.encode_pnm(16, True)
    finally:
        ctx.close()
    assert got == refpy.encode_pnm(lin, 16, True)
    hdr = b"P6\n203 77\n65535\n"
    assert got.startswith(hdr)
    body = np.frombuffer(got[len(hdr):], ">u2").reshape(77, 203, 3)
    probe = srgbprobe.encode(lin, 16, flavour="avx2")
    assert np.abs(body.astype(np.int64) - probe.astype(np.int64)).max() <= 1


def test_pnm_errors():
    ctx = native.Context(0)
    try:
        with pytest.raises(native.PikGpuError) as e:
            ctx.encode_pnm(8, True)
        assert e.value.code == -4  # nothing reconstructed yet
        frame = synthetic.make_frame(64, 48, seed=2)
        ctx.begin(frame)
        ctx.set_ac()
        ctx.reconstruct(linear=True)
        with pytest.raises(native.PikGpuError) as e:
            ctx.encode_pnm(12, True)
        assert e.value.code == -1
    finally:
        ctx.close()
