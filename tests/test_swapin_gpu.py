"""The reference decoder with the GPU swapped in, end to end.

oracle/dpik_gpu is the reference's own PikToPixels (pik/pik.cc:92-131,
compiled from its unmodified sources into oracle/_ref/libpikref_scalar.so)
with four of the library's functions bound to libpikgpu by symbol
interposition: AdaptiveDCReconstruction (keeps the dequantised DC),
DecodeFromBitstream<true> (per group, from the ThreadPool: the reference's
entropy decoding, then pikgpu_frame_begin once and
pikgpu_frame_set_group_ac), ReconOpsinImage (skipped) and
FinalizeFrameDecoding (pikgpu_reconstruct). It decodes the 4K bitstream
and must match, bit for bit, the GPU-only path: the same ABI fed with the
frozen decoder state of the same bitstream (tests/golden/c2_4k_d1_frame.npz)
in one call of pikgpu_frame_set_ac."""

import os
import re
import subprocess

import numpy as np
import pytest

from pik_b200 import layout, native
from tests import golden_cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DPIK = os.path.join(ROOT, "oracle", "_ref", "dpik_gpu")
PIK = os.path.join(golden_cases.GOLDEN, "c2_4k_d1.pik")

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not os.path.exists(DPIK),
                       reason="oracle/_ref/dpik_gpu not built"),
]


@pytest.mark.parametrize("form", ["fp32", "split_bf16"])
def test_swapin_decodes_4k_bitstream(form, tmp_path):
    out = tmp_path / "out.f32"
    r = subprocess.run([DPIK, PIK, str(out), form, "8"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    # Every hook ran: the DC smoothing once, one decode and one skipped
    # ReconOpsinImage per 512x512 group (8 x 5 at 3840x2160), one finalize.
    m = re.search(r"AdaptiveDCReconstruction (\d+), DecodeFromBitstream "
                  r"(\d+), ReconOpsinImage (\d+), FinalizeFrameDecoding "
                  r"(\d+)", r.stdout)
    assert m, r.stdout
    assert tuple(int(v) for v in m.groups()) == (1, 40, 40, 1)
    raw = out.read_bytes()
    w, h = np.frombuffer(raw[:8], np.int32)
    assert (w, h) == (3840, 2160)
    swapped = np.frombuffer(raw[8:], np.float32).reshape(3, h, w)

    frame = layout.Frame.load(os.path.join(golden_cases.GOLDEN,
                                           "c2_4k_d1_frame.npz"))
    ctx = native.Context(0, form=form)
    try:
        ctx.begin(frame)
        ctx.set_ac()
        lin, _ = ctx.reconstruct(linear=True)
    finally:
        ctx.close()
    np.testing.assert_array_equal(swapped, lin)
