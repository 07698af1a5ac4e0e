// Constant tables of the reconstruction path, computed on the host from
// their closed forms / the reference's literal constants, uploaded once per
// device into __constant__ memory. Each group cites the reference code whose
// arithmetic it reproduces (paths relative to the google/pik checkout).
#pragma once

#include <stdint.h>

namespace pikgpu {

constexpr int kMaxSigma = 672;  // pik/epf.h:70-76
constexpr int kMinSigma = 16;
constexpr int kSigmaShift = 2;

// Offsets of the N x N matrices in the packed transform arrays.
// N = 2, 4, 8, 16, 32 -> offsets 0, 4, 20, 84, 340; total 1364.
__host__ __device__ constexpr int MatOffset(int n) {
  return n == 2 ? 0 : n == 4 ? 4 : n == 8 ? 20 : n == 16 ? 84 : 340;
}
constexpr int kMatTotal = 1364;
// Small-size index into [5][8][8] scale tables.
__host__ __device__ constexpr int SizeIndex(int n) {
  return n == 2 ? 0 : n == 4 ? 1 : n == 8 ? 2 : n == 16 ? 3 : 4;
}

struct DevTables {
  // Transposed-scaled IDCT / DCT matrices (pik/dct.h:341-507):
  //   idct[u][k] = N sqrt(2/N) alpha(k) DCTScales_N[k] cos(k (u+1/2) pi/N)
  //   dct[k][x]  = N sqrt(2/N) alpha(k) IDCTScales_N[k] cos((x+1/2) k pi/N)
  float idct[kMatTotal];
  float dct[kMatTotal];
  // DCTTotalScale / DCTInvTotalScale (pik/ac_strategy.cc:256-268) for
  // x, y < 8 of each size.
  float total_scale[5][8][8];
  float inv_total_scale[5][8][8];
  // ARLowestFrequencyScale (pik/ac_strategy.h:35-38, 171-221):
  // [0] 16x16 (2x2), [1] 32x32 (4x4); indexed [y][x].
  float ar_llf16[2][2];
  float ar_llf32[4][4];
  // LINES 1-D transforms (pik/ac_strategy.cc:13-250): [n][k][x] / [n][x][k].
  float lines_fwd[9][8][8];
  float lines_inv[9][8][8];
  // UpSample4x4BlurDCT kernel (pik/ac_predictions.cc:234-254).
  float ub4[3][4];
  // HF prediction corner of a 16x16 block: hf_corner16[k][m] = sum over x of
  // dct16[k][x] * ub4[m - x / 4][x % 4] (taps 0..2), so that the 4x4 corner
  // of the 2-D DCT of the upsampled prediction is C * Pred * C^T with Pred
  // the block's 6x6 window of 2x2-cell values.
  float hf_corner16[4][6];
  // The same for a 32x32 block: its 8x8 corner from the 10x10 window.
  float hf_corner32[8][10];
  // LFPredictionBlur (pik/ac_predictions.cc:120-133) w0, w1, w2.
  float lf_blur[3];
  // Gaborish weights per strength 1..4 (pik/gaborish.cc:16-88): w0, w1, w2.
  float gaborish[5][3];
  // XybToRgb (pik/opsin_inverse.cc:38-88): inverse matrix, -bias.
  float opsin_inv[9];
  float opsin_neg_bias[3];
  // AdjustQuantBias (pik/quantizer.h:43-88).
  float one_bias[3];
  // EPF: MulTable (pik/epf_target.cc:371-413), SigmaFromQuant LUTs
  // (pik/epf_target.cc:1160-1195).
  int mul_table[kMaxSigma + 1];
  // Largest SAD whose weight (the device's EpfWeight of mul_table * 64) is
  // at least 0.05, per sigma; 507 when every clamped SAD keeps its weight.
  int epf_thr[kMaxSigma + 1];
  float sigma_lut[2][16];
  // sRGB TF_SRGB::EncodedFromDisplay polynomial (pik/color_management.cc:
  // 323-349): p[5], q[5].
  float srgb_p[5];
  float srgb_q[5];
};

// Fills `t` (host side).
void BuildTables(DevTables* t);

}  // namespace pikgpu
