"""EPF discrete decisions (u8 guide and per-block sigma) computed from a
given guide-source image with the reference's float32 arithmetic
(MinMax/MakeGuide/SigmaFromQuant, pik/epf_target.cc:980-1111,1113-1226).

Used by the parity tests to run two implementations on the SAME discrete
decisions, so that their difference measures arithmetic only. Test
infrastructure.
"""

from __future__ import annotations

import numpy as np

KBORDER = 6
_LUT = np.array([1.9815775622811198, 1.9715084740908622, 1.6819963065873933,
                 1.2146133632942862, 1.0395364091521881, 0.93552327583169714,
                 0.68568655651684773, 0.51174440217871964,
                 0.36397262821018583, 0.31621830414136975,
                 0.30262954326557712, 0.246314237855494, 0.21617524864418683,
                 0.10, 0.05, 0.0])
_AR_SCALE = {5: np.float32(1.2282996852328099),
             4: np.float32(1.1423171621463439), 3: np.float32(1.2),
             8: np.float32(1.2), 2: np.float32(1.0098134203870499)}


def _mirror_pad(img: np.ndarray, b: int) -> np.ndarray:
    # Mirror with the edge repeated once (pik/image_ops.h:217-227).
    return np.pad(img, ((0, 0), (b, b), (b, b)), mode="symmetric")


def guide_and_stretch(src: np.ndarray):
    """src: (3, H, W) float32 guide source. Returns (guide (3,H+12,W+12)
    uint8, stretch float32)."""
    p = _mirror_pad(np.asarray(src, np.float32), KBORDER)
    all_min = np.float32(p.min())
    all_max = np.float32(p.max())
    rng = np.float32(all_max - all_min)
    stretch = np.float32(1.0) if all_min == all_max else np.float32(
        np.float32(255.0) / rng)
    mul = np.float32(1.0) if rng == 0 else np.float32(np.float32(255.0) / rng)
    scaled = (p - all_min).astype(np.float32) * mul
    guide = scaled.astype(np.int32).astype(np.uint32).astype(np.uint8)
    return guide, stretch


def sigma_from_quant(signal: np.ndarray, stretch: np.float32,
                     lut_id: np.ndarray) -> np.ndarray:
    f32 = np.float32
    lut = np.stack([_LUT.astype(np.float32),
                    (_LUT / 2.0).astype(np.float32)])
    signal = signal.astype(np.float32)
    out = np.empty(signal.shape, np.float32)
    lo = signal <= f32(0.022156)
    hi = signal >= f32(0.531738)
    mid = ~(lo | hi)
    out[lo] = lut[lut_id[lo], 0]
    out[hi] = lut[lut_id[hi], 15]
    pos = (signal[mid] - f32(0.022156)) * f32(29.435892)
    tr = pos.astype(np.int64)
    frac = (pos - tr.astype(np.float32)).astype(np.float32)
    lid = lut_id[mid]
    out[mid] = (frac * lut[lid, tr + 1] +
                (f32(1.0) - frac) * lut[lid, tr]).astype(np.float32)
    sig = (out * stretch + f32(0.5182760822018414)).astype(np.float32)
    return np.minimum(sig.astype(np.int32), 672)


def frame_decisions(smoothed: np.ndarray, raw_qf: np.ndarray,
                    acs: np.ndarray, lut_ids: np.ndarray):
    """Decisions of the frame EPF given its guide source (the smoothed
    padded frame)."""
    guide, stretch = guide_and_stretch(smoothed)
    scale = np.ones(acs.shape, np.float32)
    for t, s in _AR_SCALE.items():
        scale[(acs >> 4) == t] = s
    quant = (raw_qf.astype(np.float32) * scale) * np.float32(0.039324273)
    return guide, sigma_from_quant(quant, stretch, lut_ids.astype(np.int64))


def dc_decisions(frame):
    """Decisions of AdaptiveDCReconstruction's EPF
    (pik/adaptive_reconstruction.cc:300-318): guide over the dequantized DC
    padded to a multiple of 8 by edge replication, one sigma for every block
    (qf = quant_dc / 2, DCT strategy, LUT 0). The dequantized DC is formed
    like DequantDC (pik/compressed_dc.cc:181-231) in float32."""
    f32 = np.float32
    inv_gs = f32(1.0 * 65536 / frame.global_scale)
    inv_qdc = f32(inv_gs / f32(frame.quant_dc))
    m0 = frame.dequant_table[frame.dequant_offsets[:3]].astype(np.float32)
    mul = (m0 * inv_qdc).astype(np.float32)
    q = frame.quantized_dc.astype(np.float32)
    y = (q[1] * mul[1]).astype(np.float32)
    ytox = f32(f32(frame.ytox_dc - 128) * f32(1.0 / 256))
    ytob = f32(f32(frame.ytob_dc) * f32(1.0 / 128))
    dc = np.stack([(ytox * y + (q[0] * mul[0]).astype(np.float32)),
                   y, (ytob * y + (q[2] * mul[2]).astype(np.float32))]
                  ).astype(np.float32)
    by, bx = dc.shape[1:]
    py, px = -(-by // 8) * 8, -(-bx // 8) * 8
    pad = np.pad(dc, ((0, 0), (0, py - by), (0, px - bx)), mode="edge")
    guide, stretch = guide_and_stretch(pad)
    nb = (py // 8, px // 8)
    quant = np.full(nb, np.float32(frame.quant_dc // 2), np.float32)
    quant = (quant * np.float32(1.0)) * np.float32(0.039324273)
    sigma = sigma_from_quant(quant, stretch, np.zeros(nb, np.int64))
    return guide, sigma
