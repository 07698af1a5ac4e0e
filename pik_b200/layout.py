"""Data surface of the reconstruction path: the frame description handed to
the C ABI (``include/pikgpu.h``), mirroring the decoder state the reference
holds when it reaches the reconstruction calls (FrameDecCache, Quantizer,
ColorCorrelationMap, AcStrategyImage; pik/compressed_image_fwd.h:104-230,
pik/quantizer.h:111-389, pik/color_correlation.h:44-89,
pik/ac_strategy.h:41-356).
"""

from __future__ import annotations

import dataclasses
import os

import numpy as np

# AcStrategy::Type (pik/ac_strategy.h:51-70).
ACS_TYPES = {
    "DCT": 0, "IDENTITY": 1, "DCT2X2": 2, "DCT4X4": 3, "DCT16X16": 4,
    "DCT32X32": 5, "LINES": 6, "DCT_NOHF": 7, "DCT4X4_NOHF": 8,
}
ACS_NAMES = {v: k for k, v in ACS_TYPES.items()}
# covered blocks per side (pik/ac_strategy.h:138-151)
ACS_COVER = {0: 1, 1: 1, 2: 1, 3: 1, 4: 2, 5: 4, 6: 1, 7: 1, 8: 1}

NUM_QUANT_KINDS = 7
GROUP_DIM = 512          # kGroupDim (pik/common.h:40)
TILE_DIM = 64            # kTileDim / kColorTileDim (pik/common.h:46)
BLOCK_DIM = 8

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


def default_dequant_table() -> tuple[np.ndarray, np.ndarray]:
    """The library (predefined) DequantMatrices table and its offsets
    [(table * 7 + kind) * 3 + c] -- what DequantMatrices(false) computes
    (pik/quant_weights.cc:607-926) and what every reference encoder writes
    (FindBestDequantMatrices, pik/quant_weights.cc:928-940)."""
    table = np.load(os.path.join(_DATA, "dequant_table.npy"))
    offsets = np.load(os.path.join(_DATA, "dequant_offsets.npy"))
    return table.astype(np.float32), offsets.astype(np.uint32)


def broadcast_first_block(acs: np.ndarray, field: np.ndarray) -> None:
    """Copies each multi-block transform's first-block value of a per-block
    field to its other blocks, in place."""
    by, bx = acs.shape
    for y in range(by):
        for x in range(bx):
            v = int(acs[y, x])
            t, blk = v >> 4, v & 0xF
            n = ACS_COVER.get(t, 1)
            if n > 1 and blk == 0:
                field[y:y + n, x:x + n] = field[y, x]


@dataclasses.dataclass
class Frame:
    """One frame's inputs to the reconstruction path (host arrays)."""
    xsize: int
    ysize: int
    gaborish: int
    predict_lf: int
    predict_hf: int
    have_ar: int
    epf_enable_adaptive: int
    epf_sigma: int
    epf_use_sharpened: int
    global_scale: int
    quant_dc: int
    ytox_dc: int
    ytob_dc: int
    ytox_map: np.ndarray          # (Ty, Tx) int32
    ytob_map: np.ndarray          # (Ty, Tx) int32
    ac_strategy: np.ndarray       # (By, Bx) uint8
    raw_quant_field: np.ndarray   # (By, Bx) int32
    ar_sigma_lut_ids: np.ndarray  # (By, Bx) uint8
    quantized_dc: np.ndarray      # (3, By, Bx) int16
    quantized_ac: np.ndarray      # (3, By, Bx*64) int16
    flags: int = 0
    dequant_table: np.ndarray | None = None
    dequant_offsets: np.ndarray | None = None
    dequant_control_field: np.ndarray | None = None  # (Ty, Tx) uint8
    dequant_map: np.ndarray | None = None            # (16, 256) uint8

    def __post_init__(self) -> None:
        if self.dequant_table is None or self.dequant_offsets is None:
            self.dequant_table, self.dequant_offsets = default_dequant_table()
        ty, tx = self.tiles
        if self.dequant_control_field is None:
            self.dequant_control_field = np.zeros((ty, tx), np.uint8)
        if self.dequant_map is None:
            self.dequant_map = np.zeros((16, 256), np.uint8)

    @property
    def blocks(self) -> tuple[int, int]:
        return -(-self.ysize // 8), -(-self.xsize // 8)

    @property
    def tiles(self) -> tuple[int, int]:
        return -(-self.ysize // 64), -(-self.xsize // 64)

    @property
    def num_groups(self) -> int:
        return (-(-self.xsize // GROUP_DIM)) * (-(-self.ysize // GROUP_DIM))

    def save(self, path: str) -> None:
        np.savez_compressed(path, **{
            k: (v if isinstance(v, np.ndarray) else np.asarray(v))
            for k, v in dataclasses.asdict(self).items()})

    @classmethod
    def load(cls, path: str) -> "Frame":
        z = np.load(path)
        kw = {}
        for f in dataclasses.fields(cls):
            if f.name not in z:
                continue
            v = z[f.name]
            kw[f.name] = v if v.ndim > 0 else int(v)
        return cls(**kw)
