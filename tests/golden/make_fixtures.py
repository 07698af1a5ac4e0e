"""Generates the golden fixtures of this directory from the reference
decoder/encoder compiled from google/pik's own sources (oracle/_ref/, built
by oracle/Makefile from the reference checkout).

    python tests/golden/make_fixtures.py

Fixtures (all seeded, reproducible):
  c1_256_dct8.npz   config-1 shape: 256x256 generator image (6 sinusoids,
                    3 rectangles, noise 4), all-DCT8, EPF off, gaborish on,
                    through the reference's compressed_image_test encoder
                    route (uniform quant 4.0); the frozen frame and the
                    reference (scalar build) stages dc, idct, linear.
  c2_256_d1.npz     config-2 shape at 256x256 (12 sinusoids, 20 rectangles,
                    noise 3) encoded by the reference encoder at distance 1.0
                    (mixed AcStrategy, adaptive quant field, CfL, EPF on);
                    frozen frame + reference stages dc, idct, smoothed,
                    linear.
  c2_4k_d1.pik      the config-2 workload itself: 3840x2160 generator image
                    (seed 0) encoded by the reference encoder at distance 1.0.
  c2_4k_d1_frame.npz  that bitstream decoded to the reconstruction boundary
                    by the reference's own decoding functions (bench input).
  c4_1k_d15_frame.npz  the adjoint workload's frame: a 1024x1024
                    generator image (synthetic.ADJOINT_SOURCE) encoded by the reference
                    encoder at distance 1.5 and decoded to the
                    reconstruction boundary.
  probes.npz        single-function outputs of the reference: every
                    AcStrategy transform on seeded random blocks, the LLF/LF
                    helpers, EPF weights, the opsin inverse matrix and
                    gaborish on a small random image.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import refpy  # noqa: E402
from pik_b200 import synthetic  # noqa: E402


def frame_dict(frame) -> dict:
    import dataclasses
    return {"frame_" + k: (v if isinstance(v, np.ndarray) else np.asarray(v))
            for k, v in dataclasses.asdict(frame).items() if v is not None}


def save(name: str, **arrays) -> None:
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print(f"{name}: {os.path.getsize(path) / 1e6:.2f} MB")


def c1() -> None:
    img = synthetic.make_image(256, 256, seed=0, sinusoids=6, rectangles=3,
                               noise_sigma=4)
    fz = refpy.encode_dct8(synthetic.srgb8_to_linear255(img), 4.0)
    st, _ = fz.run_stages(want=("dc", "idct", "linear"))
    save("c1_256_dct8.npz", **frame_dict(fz.frame()),
         ref_dc=st["dc"], ref_idct=st["idct"], ref_linear=st["linear"])


def c2_small() -> None:
    img = synthetic.make_image(256, 256, seed=0, sinusoids=12, rectangles=20,
                               noise_sigma=3)
    bs = refpy.encode(synthetic.srgb8_to_linear255(img), 1.0, threads=8)
    fz = refpy.Frozen(bs, flavour="scalar")
    st, _ = fz.run_stages(want=("dc", "idct", "smoothed", "linear"))
    save("c2_256_d1.npz", **frame_dict(fz.frame()),
         ref_dc=st["dc"], ref_idct=st["idct"], ref_smoothed=st["smoothed"],
         ref_linear=st["linear"], bitstream=np.frombuffer(bs, np.uint8))


def c2_4k() -> None:
    img = synthetic.make_image(3840, 2160, seed=0, sinusoids=12,
                               rectangles=20, noise_sigma=3)
    bs = refpy.encode(synthetic.srgb8_to_linear255(img), 1.0, threads=8)
    with open(os.path.join(HERE, "c2_4k_d1.pik"), "wb") as f:
        f.write(bs)
    fz = refpy.Frozen(bs, flavour="scalar")
    fz.frame().save(os.path.join(HERE, "c2_4k_d1_frame.npz"))
    print("c2_4k_d1: bitstream", len(bs), "bytes")


# The adjoint workload's source image (synthetic.ADJOINT_SOURCE): the bench
# regenerates it and takes its XYB (pik_b200.xyb) as the loss target.
C4_DISTANCE = 1.5


def c4() -> None:
    src = dict(synthetic.ADJOINT_SOURCE)
    img = synthetic.make_image(src.pop("xsize"), src.pop("ysize"), **src)
    bs = refpy.encode(synthetic.srgb8_to_linear255(img), C4_DISTANCE,
                      threads=8)
    fz = refpy.Frozen(bs, flavour="scalar")
    fz.frame().save(os.path.join(HERE, "c4_1k_d15_frame.npz"))
    print("c4_1k_d15: bitstream", len(bs), "bytes")


def probes() -> None:
    L = refpy.lib("scalar")
    rng = np.random.default_rng(7)
    out = {}
    for t in range(9):
        cov = {4: 2, 5: 4}.get(t, 1)
        n = 8 * cov
        coef = rng.normal(size=(4, cov, 64 * cov)).astype(np.float32)
        pix = rng.normal(size=(4, n, n)).astype(np.float32)
        inv = np.zeros((4, n, n), np.float32)
        fwd = np.zeros((4, cov, 64 * cov), np.float32)
        for i in range(4):
            L.pikref_transform(t, 1, coef[i].ctypes.data, 64 * cov,
                               inv[i].ctypes.data, n)
            L.pikref_transform(t, 0, pix[i].ctypes.data, n,
                               fwd[i].ctypes.data, 64 * cov)
        out[f"tr{t}_coef"], out[f"tr{t}_inv"] = coef, inv
        out[f"tr{t}_pix"], out[f"tr{t}_fwd"] = pix, fwd
    for t in range(9):
        for which in range(4):
            src = rng.normal(size=(8, 32)).astype(np.float32)
            dst = np.zeros((8, 32), np.float32)
            L.pikref_lf_helper(t, which, src.ctypes.data, 32,
                               dst.ctypes.data, 32)
            out[f"lf{t}_{which}_in"], out[f"lf{t}_{which}_out"] = src, dst
    sigmas = np.arange(16, 673, dtype=np.int32)
    sads = np.array([0, 1, 2, 3, 4, 5, 7, 10, 16, 25, 40, 63, 100, 160, 250,
                     400, 507, 508, 1000, 3060], np.int32)
    w = np.zeros((len(sigmas), len(sads)), np.float32)
    for i, s in enumerate(sigmas):
        for j, d in enumerate(sads):
            w[i, j] = L.pikref_epf_weight(int(s), int(d))
    out["epf_sigma"], out["epf_sad"], out["epf_weight"] = sigmas, sads, w
    m = np.zeros(9, np.float32)
    L.pikref_opsin_inverse_matrix(m.ctypes.data)
    out["opsin_inverse"] = m
    img = rng.uniform(0, 1, size=(3, 13, 19)).astype(np.float32)
    out["gab_in"] = img
    for s in range(1, 5):
        g = np.zeros_like(img)
        L.pikref_gaborish(s, img.ctypes.data, 19, 13, g.ctypes.data)
        out[f"gab_{s}"] = g
    save("probes.npz", **out)


if __name__ == "__main__":
    which = sys.argv[1:] or ["c1", "c2_small", "c2_4k", "c4", "probes"]
    for w in which:
        globals()[w]()
