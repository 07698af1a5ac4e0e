"""oracle/dpik_gpu without a GPU: the reference decoder runs with the
swap-in hooks bound (every hook called: the DC smoothing once, the decode
and the skipped ReconOpsinImage per 512x512 group, FinalizeFrameDecoding
once); the frame parameters it builds from the live decoder state pass the
ABI's host-side validation (pikgpu_validate); and the quantised DC it
recovers from DequantDC's output and the un-scattered coefficients its
DecodeAC hook collects per group equal the frozen decoder state of the same
bitstream (tests/golden/c2_4k_d1_frame.npz)."""

import os
import re
import subprocess

import numpy as np
import pytest

from pik_b200 import layout
from tests import golden_cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DPIK = os.path.join(ROOT, "oracle", "_ref", "dpik_gpu")

pytestmark = pytest.mark.skipif(not os.path.exists(DPIK),
                                reason="oracle/_ref/dpik_gpu not built")


def test_swapin_hooks_and_frame_state(tmp_path):
    out = tmp_path / "state.bin"
    r = subprocess.run([DPIK, os.path.join(golden_cases.GOLDEN,
                                           "c2_4k_d1.pik"),
                        str(out), "validate", "4"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    m = re.search(r"AdaptiveDCReconstruction (\d+), DecodeFromBitstream "
                  r"(\d+), ReconOpsinImage (\d+), FinalizeFrameDecoding "
                  r"(\d+)", r.stdout)
    assert m and tuple(int(v) for v in m.groups()) == (1, 40, 40, 1)
    assert "validated" in r.stdout
    raw = out.read_bytes()
    bx, by = (int(v) for v in np.frombuffer(raw[:8], np.int32))
    n_dc = 3 * by * bx
    qdc = np.frombuffer(raw[8:8 + 2 * n_dc], np.int16).reshape(3, by, bx)
    qac = np.frombuffer(raw[8 + 2 * n_dc:], np.int16).reshape(3, by, bx * 64)
    frame = layout.Frame.load(os.path.join(golden_cases.GOLDEN,
                                           "c2_4k_d1_frame.npz"))
    np.testing.assert_array_equal(qdc, frame.quantized_dc.reshape(qdc.shape))
    np.testing.assert_array_equal(qac, frame.quantized_ac.reshape(qac.shape))
