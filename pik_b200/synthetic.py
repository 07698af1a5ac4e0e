"""Seeded synthetic workloads for the reconstruction path.

Three generators:

* ``make_image`` -- the test-image generator the benchmark configurations are
  defined with: a sum of random 2-D sinusoids (period 4..64 px, random
  orientation, phase and amplitude), random flat axis-aligned rectangles and
  Gaussian noise, clipped to the 8-bit (or 16-bit) range. Images from it are
  encoded by the reference encoder in the parity tests.

* ``make_frame`` -- a synthetic *decoded frame*: the integer coefficients and
  side information a pik bitstream carries for the reconstruction path
  (AcStrategy layout with all nine transform types, raw quant field, EPF LUT
  ids, colour-correlation maps, quantized DC and AC), drawn from seeded
  distributions shaped like the reference encoder's output at
  butteraugli distance ~1. It lets the benchmark build 4K/8K inputs on the
  GPU host without running an encoder. Its global scale and quant_dc equal
  the reference encoder's on the generator images at distance 1, and its
  quant-field and DC distributions are close to them (quant field median
  18 against 15, Y DC mean 240 against 253). Its AC is sparser (3.6% of
  the Y coefficients non-zero against 11%), and its transform mix is
  broader (see _DEFAULT_SHARES).

* ``make_highlight_frame`` -- ``make_frame`` at a lower distance (finer
  quant field, larger AC) with a share of the area in highlights.
"""

from __future__ import annotations

import numpy as np

from . import layout

__all__ = ["make_image", "make_frame", "make_highlight_frame",
           "srgb8_to_linear255"]


def make_image(xsize: int, ysize: int, *, seed: int = 0, sinusoids: int = 6,
               rectangles: int = 3, noise_sigma: float = 4.0,
               maxval: float = 255.0) -> np.ndarray:
    """Returns a (3, ysize, xsize) float32 image in [0, maxval]."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:ysize, 0:xsize].astype(np.float32)
    img = np.full((3, ysize, xsize), 0.5 * maxval, dtype=np.float32)
    for _ in range(sinusoids):
        period = rng.uniform(4.0, 64.0)
        theta = rng.uniform(0.0, np.pi)
        phase = rng.uniform(0.0, 2.0 * np.pi)
        amp = rng.uniform(0.02, 0.12) * maxval * rng.uniform(0.3, 1.0, size=3)
        arg = (2.0 * np.pi / period) * (np.cos(theta) * xx +
                                        np.sin(theta) * yy) + phase
        wave = np.sin(arg).astype(np.float32)
        img += amp[:, None, None].astype(np.float32) * wave[None]
    for _ in range(rectangles):
        w = int(rng.integers(max(2, xsize // 16), max(3, xsize // 3)))
        h = int(rng.integers(max(2, ysize // 16), max(3, ysize // 3)))
        x0 = int(rng.integers(0, max(1, xsize - w)))
        y0 = int(rng.integers(0, max(1, ysize - h)))
        colour = rng.uniform(0.0, maxval, size=3).astype(np.float32)
        img[:, y0:y0 + h, x0:x0 + w] = colour[:, None, None]
    img += rng.normal(0.0, noise_sigma, size=img.shape).astype(np.float32)
    return np.clip(img, 0.0, maxval).astype(np.float32)


def srgb8_to_linear255(img: np.ndarray) -> np.ndarray:
    """sRGB-encoded [0,255] -> linear on the reference's 0..255 scale
    (IEC 61966-2-1 transfer function)."""
    v = np.asarray(img, dtype=np.float64) / 255.0
    lin = np.where(v <= 0.04045, v / 12.92, ((v + 0.055) / 1.055) ** 2.4)
    return (lin * 255.0).astype(np.float32)


# Shares of 8x8 cells covered by each transform type: a broad mix that
# gives every type, including those the reference encoder rarely or never
# picks, a real share of the frame. On the generator images at distance 1
# the reference encoder picks about 90% DCT16X16 and 9% DCT8; at distance
# 0.5, 72% DCT16X16 and 22% DCT32X32; at distance 3, 89% DCT32X32.
# Multi-block transforms are placed first, aligned to their size.
_DEFAULT_SHARES = {
    "DCT32X32": 0.18, "DCT16X16": 0.22, "DCT": 0.36, "DCT4X4": 0.08,
    "DCT2X2": 0.04, "IDENTITY": 0.03, "LINES": 0.02, "DCT_NOHF": 0.04,
    "DCT4X4_NOHF": 0.03,
}


def make_frame(xsize: int, ysize: int, *, seed: int = 0,
               shares: dict | None = None, have_ar: bool = True,
               gaborish: int = 2, global_scale: int = 3065,
               quant_dc: int = 16, qf_median: float = 18.0,
               qf_spread: float = 0.3, ac_scale: float = 1.0,
               qf_max: int = 31) -> "layout.Frame":
    """Synthetic decoded frame of ``xsize`` x ``ysize`` pixels.

    Defaults follow the reference encoder on the generator images at
    butteraugli distance 1: global_scale 3065, quant_dc 16, raw quant field
    log-normal around 18 (5th-95th percentile ~11-25), quantized DC of
    X ~ -10 +- 20, Y ~ 240 +- 48, B ~ 0 +- 27, and sparse AC whose mean
    magnitude falls off with frequency (Y dominant, X and B ~10x smaller).
    The raw quant field is clipped to [6, qf_max].
    """
    rng = np.random.default_rng(seed)
    shares = dict(_DEFAULT_SHARES if shares is None else shares)
    bx, by = -(-xsize // 8), -(-ysize // 8)
    tx, ty = -(-xsize // 64), -(-ysize // 64)
    acs = np.full((by, bx), 0xFF, dtype=np.uint8)

    def place(size: int, code: int, share: float) -> None:
        if share <= 0:
            return
        target = int(share * by * bx / (size * size))
        ys = np.arange(0, by - size + 1, size)
        xs = np.arange(0, bx - size + 1, size)
        if len(ys) == 0 or len(xs) == 0 or target == 0:
            return
        cand = np.stack(np.meshgrid(ys, xs, indexing="ij"), -1).reshape(-1, 2)
        rng.shuffle(cand)
        sub = (np.arange(size)[:, None] * size +
               np.arange(size)[None, :]).astype(np.uint8)
        placed = 0
        for y0, x0 in cand:
            if placed >= target:
                break
            if np.all(acs[y0:y0 + size, x0:x0 + size] == 0xFF):
                acs[y0:y0 + size, x0:x0 + size] = (code << 4) | sub
                placed += 1

    place(4, layout.ACS_TYPES["DCT32X32"], shares.pop("DCT32X32", 0.0))
    place(2, layout.ACS_TYPES["DCT16X16"], shares.pop("DCT16X16", 0.0))
    single = [(layout.ACS_TYPES[k], v) for k, v in shares.items() if v > 0]
    free = acs == 0xFF
    codes = np.array([c for c, _ in single], dtype=np.uint8)
    p = np.array([v for _, v in single], dtype=np.float64)
    pick = rng.choice(codes, size=int(free.sum()), p=p / p.sum())
    acs[free] = (pick << 4).astype(np.uint8)

    def smooth(shape, scale_blocks, amp):
        sy, sx = shape
        coarse = rng.normal(0.0, 1.0, size=(sy // scale_blocks + 2,
                                            sx // scale_blocks + 2))
        f = np.kron(coarse, np.ones((scale_blocks, scale_blocks)))[:sy, :sx]
        return amp * f

    qf = qf_median * np.exp(smooth((by, bx), 8, qf_spread) +
                            rng.normal(0.0, 0.08, size=(by, bx)))
    raw_qf = np.clip(np.round(qf), 6, qf_max).astype(np.int32)
    layout.broadcast_first_block(acs, raw_qf)
    lut = np.zeros((by, bx), dtype=np.uint8)

    dc = np.zeros((3, by, bx), dtype=np.int16)
    for c, (mean, sd) in enumerate(((-10.0, 20.0), (240.0, 48.0),
                                    (0.0, 27.0))):
        f = mean + smooth((by, bx), 16, sd * 0.8) + rng.normal(
            0.0, sd * 0.3, size=(by, bx))
        dc[c] = np.clip(np.round(f), -2000, 2000).astype(np.int16)

    # AC: per coefficient of each transform, mean magnitude falling with the
    # coefficient's frequency (row + column, in 8-point units).
    k = np.arange(64)
    ac = np.zeros((3, by, bx * 64), dtype=np.int16)
    freq = np.zeros((by, bx * 64), dtype=np.float32)
    types = acs >> 4
    blk = acs & 0xF
    cov = np.where(types == 5, 4, np.where(types == 4, 2, 1))
    # Position of each stored coefficient inside its (8c x 8c) matrix.
    flat = blk[:, :, None].astype(np.int64) * 64 + k[None, None, :]
    n = (8 * cov)[:, :, None]
    row = flat // n
    col = flat % n
    freq = ((row + col) * 8.0 / n).reshape(by, bx * 64).astype(np.float32)
    for c, amp in enumerate((0.12, 2.5, 0.25)):
        mean = ac_scale * amp * np.exp(-freq / 1.6)
        mag = np.floor(rng.exponential(1.0, size=freq.shape) * mean)
        sign = np.where(rng.random(size=freq.shape) < 0.5, -1, 1)
        ac[c] = np.clip(mag * sign, -2000, 2000).astype(np.int16)
    ytox = (rng.integers(98, 129, size=(ty, tx))).astype(np.int32)
    ytob = np.full((ty, tx), 120, dtype=np.int32)
    return layout.Frame(
        xsize=xsize, ysize=ysize, gaborish=gaborish, predict_lf=1,
        predict_hf=1, have_ar=int(have_ar), epf_enable_adaptive=1,
        epf_sigma=0, epf_use_sharpened=0, global_scale=global_scale,
        quant_dc=quant_dc, ytox_dc=130, ytob_dc=120, ytox_map=ytox,
        ytob_map=ytob, ac_strategy=acs, raw_quant_field=raw_qf,
        ar_sigma_lut_ids=lut, quantized_dc=dc, quantized_ac=ac)


# Shares of 8x8 cells per transform type that the reference encoder picks
# on the generator images (12 sinusoids, 20 rectangles, noise sigma 3,
# 1024x1024) at distance 0.5.
# The adjoint workload's source image (make_image arguments): its
# reference-encoded frame (distance 1.5) is tests/golden/c4_1k_d15_frame.npz,
# and its XYB (pik_b200.xyb) is the loss target.
ADJOINT_SOURCE = dict(xsize=1024, ysize=1024, seed=4, sinusoids=12,
                      rectangles=20, noise_sigma=3)

ENCODER_SHARES_D05 = {
    "DCT16X16": 0.7231, "DCT32X32": 0.2217, "DCT": 0.0528, "DCT4X4": 0.0012,
    "DCT2X2": 0.0012,
}


def make_highlight_frame(xsize: int, ysize: int, *, seed: int = 0,
                         distance: float = 0.5, highlight_share: float = 0.01,
                         highlight_gain: float = 4.0,
                         shares: dict | None = None) -> "layout.Frame":
    """Synthetic frame of a high-quality encode with highlights.

    ``make_frame`` at ``distance``: the quant field scales with 1 / distance
    (clipped to [6, 64]) and the AC magnitudes with 1 / distance. Random
    axis-aligned rectangles cover ``highlight_share`` of the blocks; their
    light is ``highlight_gain`` x the rest, which in the cube-root XYB domain
    scales their quantized Y DC and their AC by highlight_gain^(1/3).
    ``shares`` is the transform mix (make_frame's default if None).
    """
    f = make_frame(xsize, ysize, seed=seed, qf_median=18.0 / distance,
                   ac_scale=1.0 / distance, qf_max=64, shares=shares)
    by, bx = f.blocks
    rng = np.random.default_rng(seed)
    mask = np.zeros((by, bx), bool)
    target = max(1, int(highlight_share * by * bx))
    while mask.sum() < target:
        h = min(by, int(rng.integers(2, max(3, by // 32))))
        w = min(bx, int(rng.integers(2, max(3, bx // 32))))
        y0 = int(rng.integers(0, by - h + 1))
        x0 = int(rng.integers(0, bx - w + 1))
        mask[y0:y0 + h, x0:x0 + w] = True
    gain = highlight_gain ** (1.0 / 3.0)
    f.quantized_dc[1][mask] = np.clip(
        np.round(f.quantized_dc[1][mask] * gain), -2000, 2000)
    acm = np.repeat(mask, 64, axis=1)
    for c in range(3):
        f.quantized_ac[c][acm] = np.clip(
            np.round(f.quantized_ac[c][acm] * gain), -2000, 2000)
    return f
