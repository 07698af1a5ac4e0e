// CPU restatement of google/pik's decoder reconstruction path -- the parity
// oracle (test infrastructure; see pik_oracle.h). Every function names the
// reference code it restates (paths relative to the google/pik checkout).

#include "pik_oracle.h"

#include <string.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <vector>

namespace {

constexpr int kBlockDim = 8;
constexpr int kGroupDimInBlocks = 64;  // pik/common.h:40-43
constexpr int kTileDimInBlocks = 8;    // pik/common.h:46-50
constexpr double kPi = 3.14159265358979323846;

enum AcsType {
  kDCT = 0, kIDENTITY = 1, kDCT2X2 = 2, kDCT4X4 = 3, kDCT16X16 = 4,
  kDCT32X32 = 5, kLINES = 6, kDCT_NOHF = 7, kDCT4X4_NOHF = 8
};

// ---------------------------------------------------------------------------
// AcStrategy properties (pik/ac_strategy.h:95-151).

int Covered(int type) {
  return type == kDCT32X32 ? 4 : type == kDCT16X16 ? 2 : 1;
}
int QuantKind(int type) {
  if (type == kDCT_NOHF) return 0;
  if (type == kDCT4X4_NOHF) return 3;
  return type;  // QuantKind values equal the first seven types
}
bool PredictHF(int type) {
  return type != kDCT2X2 && type != kIDENTITY && type != kDCT_NOHF &&
         type != kDCT4X4_NOHF && type != kLINES;
}
float ARQuantScale(int type) {
  if (type == kDCT32X32) return 1.2282996852328099f;
  if (type == kDCT16X16) return 1.1423171621463439f;
  if (type == kDCT4X4 || type == kDCT4X4_NOHF) return 1.2f;
  if (type == kDCT2X2) return 1.0098134203870499f;
  return 1.0f;
}

// ---------------------------------------------------------------------------
// DCT scale tables (pik/dct.h:46-269), from their closed forms.
// iscale_N(k) = sqrt(2/N) * alpha(k) * cos(k pi / 2N); the 8-point tables
// follow Arai-Agui-Nakajima (DCTScales = 1/(N iscale), IDCTScales = iscale),
// all other sizes the flipped convention (pik/dct.h:24-31).

struct Tables {
  float ds[33][32], is[33][32], l1[33][32], l1inv[33][32];
  Tables() {
    for (int n : {2, 4, 8, 16, 32}) {
      for (int k = 0; k < n; ++k) {
        const double alpha = k == 0 ? std::sqrt(0.5) : 1.0;
        const double iscale =
            std::sqrt(2.0 / n) * alpha * std::cos(k * kPi / (2.0 * n));
        const double inv = 1.0 / (n * iscale);
        ds[n][k] = static_cast<float>(n == 8 ? inv : iscale);
        is[n][k] = static_cast<float>(n == 8 ? iscale : inv);
        // Relative L1 norm of basis k: product of cos(pi/2^(j+3)) for
        // j = 0 .. log2(n) - 2 - trailing_zeros(k); 1 for k = 0 and n/2.
        double norm = 1.0;
        if (k != 0 && k != n / 2) {
          int tz = 0;
          while (((k >> tz) & 1) == 0) ++tz;
          int log2n = 0;
          while ((1 << log2n) < n) ++log2n;
          for (int j = 0; j <= log2n - 2 - tz; ++j) {
            norm *= std::cos(kPi / double(1 << (j + 3)));
          }
        }
        l1[n][k] = static_cast<float>(norm);
        l1inv[n][k] = static_cast<float>(1.0 / norm);
      }
    }
  }
};
const Tables& T() {
  static Tables t;
  return t;
}

// DCTTotalScale / DCTInvTotalScale (pik/ac_strategy.cc:256-268), evaluated
// in float left to right like the reference's constexpr functions.
float DCTTotalScale(int n, int x, int y) {
  const Tables& t = T();
  return float(n) * t.ds[n][x] * t.ds[n][y] * t.l1inv[n][x] * t.l1inv[n][y];
}
float DCTInvTotalScale(int n, int x, int y) {
  const Tables& t = T();
  return float(n) * t.is[n][x] * t.is[n][y] * t.l1[n][x] * t.l1[n][y];
}
// ARLowestFrequencyScale (pik/ac_strategy.h:35-38).
float ARLowestFrequencyScale(int n, int bx, int by) {
  const Tables& t = T();
  return float(n) * t.is[n][bx] * t.is[n][by] * t.l1[n][bx] * t.l1[n][by];
}

// ---------------------------------------------------------------------------
// Transposed-scaled 2-D transforms (pik/dct.h:341-507) as separable matrix
// products. Coefficient block C is stored with its ROW index = horizontal
// frequency (the "transposed" convention, pik/dct.h:430-440):
//   tsIDCT:  P = A C^T A^T,  A[u][k] = N sqrt(2/N) alpha(k) DS_N[k]
//                                      cos(k (u + 1/2) pi / N)
//   tsDCT:   C = (1/N^2) B P^T B^T (the 1/N^2 is ScaleToBlock,
//            pik/block.h:103-132), B[k][x] = N sqrt(2/N) alpha(k) IS_N[k]
//                                      cos((x + 1/2) k pi / N)

struct Mats {
  double a[33][32][32];  // [n][u][k]
  double b[33][32][32];  // [n][k][x]
  Mats() {
    const Tables& t = T();
    for (int n : {2, 4, 8, 16, 32}) {
      for (int i = 0; i < n; ++i) {
        for (int k = 0; k < n; ++k) {
          const double alpha = k == 0 ? std::sqrt(0.5) : 1.0;
          const double s = n * std::sqrt(2.0 / n) * alpha;
          a[n][i][k] = s * double(t.ds[n][k]) *
                       std::cos(k * (i + 0.5) * kPi / n);
          b[n][k][i] = s * double(t.is[n][k]) *
                       std::cos((i + 0.5) * k * kPi / n);
        }
      }
    }
  }
};
const Mats& M() {
  static Mats m;
  return m;
}

// in: n x n block, element (r, c) at in[r * istride + c]; out likewise.
template <typename F>
void TsIDCT(int n, const F* in, size_t istride, F* out, size_t ostride) {
  const Mats& m = M();
  F tmp[32 * 32];
  // tmp[k][v] = sum_l C[k][l] A[v][l]
  for (int k = 0; k < n; ++k) {
    for (int v = 0; v < n; ++v) {
      F s = 0;
      for (int l = 0; l < n; ++l) s += in[k * istride + l] * F(m.a[n][v][l]);
      tmp[k * n + v] = s;
    }
  }
  // P[v][u] = sum_k A[u][k] tmp[k][v]
  for (int v = 0; v < n; ++v) {
    for (int u = 0; u < n; ++u) {
      F s = 0;
      for (int k = 0; k < n; ++k) s += F(m.a[n][u][k]) * tmp[k * n + v];
      out[v * ostride + u] = s;
    }
  }
}

template <typename F>
void TsDCT(int n, const F* in, size_t istride, F* out, size_t ostride) {
  const Mats& m = M();
  F tmp[32 * 32];
  // tmp[k][y] = sum_x B[k][x] P[y][x]
  for (int k = 0; k < n; ++k) {
    for (int y = 0; y < n; ++y) {
      F s = 0;
      for (int x = 0; x < n; ++x) s += F(m.b[n][k][x]) * in[y * istride + x];
      tmp[k * n + y] = s;
    }
  }
  const F scale = F(1) / F(n * n);
  for (int k = 0; k < n; ++k) {
    for (int l = 0; l < n; ++l) {
      F s = 0;
      for (int y = 0; y < n; ++y) s += tmp[k * n + y] * F(m.b[n][l][y]);
      out[k * ostride + l] = s * scale;
    }
  }
}

// ReinterpretingDCT / ReinterpretingIDCT (pik/ac_strategy.cc:270-311).
template <typename F>
void ReinterpretingDCT(int dctn, int n, const F* input, size_t istride,
                       F* output, size_t ostride) {
  F block[64], res[64];
  for (int y = 0; y < n; ++y) {
    for (int x = 0; x < n; ++x) block[y * n + x] = input[y * istride + x];
  }
  TsDCT<F>(n, block, n, res, n);
  for (int y = 0; y < n; ++y) {
    for (int x = 0; x < n; ++x) {
      output[y * ostride + x] = res[y * n + x] * F(DCTTotalScale(n, x, y)) *
                                F(DCTInvTotalScale(dctn, x, y));
    }
  }
}
template <typename F>
void ReinterpretingIDCT(int dctn, int lf, int n, const F* input,
                        size_t istride, F* output, size_t ostride) {
  F block[64] = {};
  for (int y = 0; y < lf; ++y) {
    for (int x = 0; x < lf; ++x) {
      block[y * n + x] = input[y * istride + x] *
                         F(DCTInvTotalScale(n, x, y)) *
                         F(DCTTotalScale(dctn, x, y));
    }
  }
  F res[64];
  TsIDCT<F>(n, block, n, res, n);
  for (int y = 0; y < n; ++y) {
    for (int x = 0; x < n; ++x) output[y * ostride + x] = res[y * n + x];
  }
}

// ---------------------------------------------------------------------------
// LINES strategy index tables (pik/ac_strategy.cc:344-390): pixel groups of
// the four 2x2 DCs and the diagonal 3/4/6/8-point transforms.
const int kLinesDc00[] = {0, 8, 9, 16, 17, 18, 25, 26, 27, 34, 35,
                          36, 43, 44, 45, 52, 53, 54, 61, 62, 63};
const int kLinesDc01[] = {24, 32, 33, 40, 41, 42, 48, 49,
                          50, 51, 56, 57, 58, 59, 60};
const int kLinesDc10[] = {3, 4, 5, 6, 7, 12, 13, 14,
                          15, 21, 22, 23, 30, 31, 39};
const int kLinesDc11[] = {1, 2, 10, 11, 19, 20, 28, 29, 37, 38, 46, 47, 55};
const int kLinesP3[4][3] = {{6, 7, 15}, {5, 14, 23}, {40, 49, 58},
                            {48, 56, 57}};
const int kLinesP4[4][4] = {{4, 13, 22, 31}, {3, 12, 30, 39},
                            {24, 33, 51, 60}, {32, 41, 50, 59}};
const int kLinesP6[4][6] = {{2, 11, 20, 29, 38, 47}, {1, 10, 19, 37, 46, 55},
                            {8, 17, 26, 44, 53, 62}, {16, 25, 34, 43, 52, 61}};
const int kLinesP8[1][8] = {{0, 9, 18, 27, 36, 45, 54, 63}};
const int kLinesC3[4][3] = {{6, 7, 15}, {5, 14, 23}, {40, 49, 58},
                            {48, 56, 57}};
const int kLinesC4[4][4] = {{4, 13, 22, 31}, {3, 12, 21, 30},
                            {24, 33, 42, 51}, {32, 41, 50, 59}};
const int kLinesC6[4][6] = {{2, 11, 20, 29, 38, 47}, {10, 19, 28, 37, 46, 55},
                            {17, 26, 35, 44, 53, 62}, {16, 25, 34, 43, 52, 61}};
const int kLinesC8[1][8] = {{18, 27, 36, 45, 54, 39, 60, 63}};

// The 1-D transforms of LINES (pik/ac_strategy.cc:13-250) are scaled
// DCT-II / DCT-III pairs of length n in {3, 4, 6, 8}:
//   forward  X[k] = s_n(k) * sum_x cos(k (x + 1/2) pi / n) x[x]
//   inverse  x[x] = sum_k t_n(k) cos(k (x + 1/2) pi / n) X[k],
// with t_n(k) s_n(k) = 1/n (k = 0) or 2/n (k > 0) so that they invert.
// s_n(k) is 1/n for k = 0 (the mean) and, for k > 0, 2/n for n = 3, 6 and
// sqrt(2)/n for n = 4, 8 (the inverses then carry 1 resp. sqrt(2)).
// Index lists address pixels and coefficients column-major:
// P1(i) = P(i / 8, i % 8) = pixels[(i % 8) * stride + i / 8]
// (pik/ac_strategy.cc:334-341).
int ColMajor(int i) { return (i & 7) * 8 + (i >> 3); }
double LinesFwdScale(int n, int k) {
  if (k == 0) return 1.0 / n;
  if (n == 3 || n == 6) return 2.0 / n;
  return 2.0 / n / std::sqrt(2.0);  // n = 4, 8
}
struct LinesMats {
  double fwd[9][8][8], inv[9][8][8];
  LinesMats() {
    for (int n : {3, 4, 6, 8}) {
      for (int k = 0; k < n; ++k) {
        const double s = LinesFwdScale(n, k);
        const double t = (k == 0 ? 1.0 / n : 2.0 / n) / s;
        for (int x = 0; x < n; ++x) {
          const double c = std::cos(k * (x + 0.5) * kPi / n);
          fwd[n][k][x] = s * c;
          inv[n][x][k] = t * c;
        }
      }
    }
  }
};
const LinesMats& LM() {
  static LinesMats m;
  return m;
}

// ---------------------------------------------------------------------------
// AcStrategy::TransformToPixels / TransformFromPixels
// (pik/ac_strategy.cc:531-848). Coefficients use the frame layout: for a
// block covering c x c cells, element i of the (8c x 8c) coefficient matrix
// is at coeff[(i / (64 c)) * cstride + i % (64 c)].

template <typename F>
struct CoefView {
  F* p;
  size_t stride;
  int chunk;
  F& operator[](int i) const { return p[(i / chunk) * stride + i % chunk]; }
};

template <typename F>
void TransformToPixels(int type, const F* coefficients, size_t cstride,
                       F* pixels, size_t pstride) {
  const int cov = Covered(type);
  CoefView<const F> c{coefficients, cstride, 64 * cov};
  switch (type) {
    case kDCT:
    case kDCT_NOHF:
    case kDCT16X16:
    case kDCT32X32: {
      const int n = 8 * cov;
      F in[32 * 32];
      for (int i = 0; i < n * n; ++i) in[i] = c[i];
      TsIDCT<F>(n, in, n, pixels, pstride);
      break;
    }
    case kDCT4X4:
    case kDCT4X4_NOHF: {
      const F b00 = c[0], b01 = c[1], b10 = c[8], b11 = c[9];
      const F dcs[4] = {b00 + b01 + b10 + b11, b00 + b01 - b10 - b11,
                        b00 - b01 + b10 - b11, b00 - b01 - b10 + b11};
      for (int y = 0; y < 2; ++y) {
        for (int x = 0; x < 2; ++x) {
          F block[16];
          block[0] = dcs[y * 2 + x];
          for (int iy = 0; iy < 4; ++iy) {
            for (int ix = 0; ix < 4; ++ix) {
              if (ix == 0 && iy == 0) continue;
              block[iy * 4 + ix] = c[(y + iy * 2) * 8 + x + ix * 2];
            }
          }
          TsIDCT<F>(4, block, 4, pixels + y * 4 * pstride + x * 4, pstride);
        }
      }
      break;
    }
    case kDCT2X2: {
      F coeffs[64];
      for (int i = 0; i < 64; ++i) coeffs[i] = c[i];
      for (int s : {2, 4, 8}) {  // IDCT2TopBlock<2>, <4>, <8>
        F temp[64];
        const int h = s / 2;
        for (int y = 0; y < h; ++y) {
          for (int x = 0; x < h; ++x) {
            const F c00 = coeffs[y * 8 + x];
            const F c01 = coeffs[y * 8 + h + x];
            const F c10 = coeffs[(y + h) * 8 + x];
            const F c11 = coeffs[(y + h) * 8 + h + x];
            temp[y * 2 * 8 + x * 2] = c00 + c01 + c10 + c11;
            temp[y * 2 * 8 + x * 2 + 1] = c00 + c01 - c10 - c11;
            temp[(y * 2 + 1) * 8 + x * 2] = c00 - c01 + c10 - c11;
            temp[(y * 2 + 1) * 8 + x * 2 + 1] = c00 - c01 - c10 + c11;
          }
        }
        for (int y = 0; y < s; ++y) {
          for (int x = 0; x < s; ++x) coeffs[y * 8 + x] = temp[y * 8 + x];
        }
      }
      for (int y = 0; y < 8; ++y) {
        for (int x = 0; x < 8; ++x) pixels[y * pstride + x] = coeffs[y * 8 + x];
      }
      break;
    }
    case kIDENTITY: {
      const F b00 = c[0], b01 = c[1], b10 = c[8], b11 = c[9];
      const F dcs[4] = {b00 + b01 + b10 + b11, b00 + b01 - b10 - b11,
                        b00 - b01 + b10 - b11, b00 - b01 - b10 + b11};
      for (int y = 0; y < 2; ++y) {
        for (int x = 0; x < 2; ++x) {
          const F block_dc = dcs[y * 2 + x];
          F residual_sum = 0;
          for (int iy = 0; iy < 4; ++iy) {
            for (int ix = 0; ix < 4; ++ix) {
              if (ix == 0 && iy == 0) continue;
              residual_sum += c[(y + iy * 2) * 8 + x + ix * 2];
            }
          }
          F* ctr = &pixels[(4 * y + 1) * pstride + 4 * x + 1];
          *ctr = block_dc - residual_sum * F(1.0f / 16);
          for (int iy = 0; iy < 4; ++iy) {
            for (int ix = 0; ix < 4; ++ix) {
              if (ix == 1 && iy == 1) continue;
              pixels[(y * 4 + iy) * pstride + x * 4 + ix] =
                  c[(y + iy * 2) * 8 + x + ix * 2] + *ctr;
            }
          }
          pixels[y * 4 * pstride + x * 4] = c[(y + 2) * 8 + x + 2] + *ctr;
        }
      }
      break;
    }
    case kLINES: {
      const LinesMats& lm = LM();
      F temp[64] = {};
      auto idcts = [&](int n, const int* ip, const int* ic) {
        F v[8];
        for (int j = 0; j < n; ++j) v[j] = c[ColMajor(ic[j])];
        for (int j = 0; j < n; ++j) {
          F s = 0;
          for (int k = 0; k < n; ++k) s += F(lm.inv[n][j][k]) * v[k];
          temp[ColMajor(ip[j])] = s;
        }
      };
      for (int i = 0; i < 4; ++i) idcts(3, kLinesP3[i], kLinesC3[i]);
      for (int i = 0; i < 4; ++i) idcts(4, kLinesP4[i], kLinesC4[i]);
      for (int i = 0; i < 4; ++i) idcts(6, kLinesP6[i], kLinesC6[i]);
      idcts(8, kLinesP8[0], kLinesC8[0]);
      // IDCT2x2 of the four DCs (C(0,0), C(0,1), C(1,0), C(1,1) with C(x,y)
      // = coefficients[y * 8 + x]).
      const F i0 = c[0], i1 = c[8], i2 = c[1], i3 = c[9];
      const F d00 = i0 + i1 + i2 + i3, d01 = i0 - i1 + i2 - i3;
      const F d10 = i0 + i1 - i2 - i3, d11 = i0 - i1 - i2 + i3;
      for (int v : kLinesDc00) temp[ColMajor(v)] += d00;
      for (int v : kLinesDc01) temp[ColMajor(v)] += d01;
      for (int v : kLinesDc10) temp[ColMajor(v)] += d10;
      for (int v : kLinesDc11) temp[ColMajor(v)] += d11;
      temp[21] = (temp[12] + temp[30]) * F(0.5f);
      temp[28] = (temp[19] + temp[37]) * F(0.5f);
      temp[35] = (temp[26] + temp[44]) * F(0.5f);
      temp[42] = (temp[33] + temp[51]) * F(0.5f);
      // P(x, y) = pixels[y * stride + x] = T(x, y) = temp[y * 8 + x].
      for (int y = 0; y < 8; ++y) {
        for (int x = 0; x < 8; ++x) pixels[y * pstride + x] = temp[y * 8 + x];
      }
      break;
    }
  }
}

template <typename F>
void TransformFromPixels(int type, const F* pixels, size_t pstride,
                         F* coefficients, size_t cstride) {
  const int cov = Covered(type);
  CoefView<F> c{coefficients, cstride, 64 * cov};
  switch (type) {
    case kDCT:
    case kDCT_NOHF:
    case kDCT16X16:
    case kDCT32X32: {
      const int n = 8 * cov;
      F out[32 * 32];
      TsDCT<F>(n, pixels, pstride, out, n);
      for (int i = 0; i < n * n; ++i) c[i] = out[i];
      break;
    }
    case kDCT4X4:
    case kDCT4X4_NOHF: {
      for (int y = 0; y < 2; ++y) {
        for (int x = 0; x < 2; ++x) {
          F block[16];
          TsDCT<F>(4, pixels + y * 4 * pstride + x * 4, pstride, block, 4);
          for (int iy = 0; iy < 4; ++iy) {
            for (int ix = 0; ix < 4; ++ix) {
              c[(y + iy * 2) * 8 + x + ix * 2] = block[iy * 4 + ix];
            }
          }
        }
      }
      const F b00 = c[0], b01 = c[1], b10 = c[8], b11 = c[9];
      c[0] = (b00 + b01 + b10 + b11) * F(0.25f);
      c[1] = (b00 + b01 - b10 - b11) * F(0.25f);
      c[8] = (b00 - b01 + b10 - b11) * F(0.25f);
      c[9] = (b00 - b01 - b10 + b11) * F(0.25f);
      break;
    }
    case kDCT2X2: {
      F cur[64];
      for (int y = 0; y < 8; ++y) {
        for (int x = 0; x < 8; ++x) cur[y * 8 + x] = pixels[y * pstride + x];
      }
      for (int s : {8, 4, 2}) {  // DCT2TopBlock<8>, <4>, <2>
        F temp[64];
        const int h = s / 2;
        for (int y = 0; y < h; ++y) {
          for (int x = 0; x < h; ++x) {
            const F c00 = cur[y * 2 * 8 + x * 2];
            const F c01 = cur[y * 2 * 8 + x * 2 + 1];
            const F c10 = cur[(y * 2 + 1) * 8 + x * 2];
            const F c11 = cur[(y * 2 + 1) * 8 + x * 2 + 1];
            temp[y * 8 + x] = (c00 + c01 + c10 + c11) * F(0.25f);
            temp[y * 8 + h + x] = (c00 + c01 - c10 - c11) * F(0.25f);
            temp[(y + h) * 8 + x] = (c00 - c01 + c10 - c11) * F(0.25f);
            temp[(y + h) * 8 + h + x] = (c00 - c01 - c10 + c11) * F(0.25f);
          }
        }
        for (int y = 0; y < s; ++y) {
          for (int x = 0; x < s; ++x) cur[y * 8 + x] = temp[y * 8 + x];
        }
      }
      for (int i = 0; i < 64; ++i) c[i] = cur[i];
      break;
    }
    case kIDENTITY: {
      for (int y = 0; y < 2; ++y) {
        for (int x = 0; x < 2; ++x) {
          F block_dc = 0;
          for (int iy = 0; iy < 4; ++iy) {
            for (int ix = 0; ix < 4; ++ix) {
              block_dc += pixels[(y * 4 + iy) * pstride + x * 4 + ix];
            }
          }
          block_dc *= F(1.0f / 16);
          const F ctr = pixels[(y * 4 + 1) * pstride + x * 4 + 1];
          for (int iy = 0; iy < 4; ++iy) {
            for (int ix = 0; ix < 4; ++ix) {
              if (ix == 1 && iy == 1) continue;
              c[(y + iy * 2) * 8 + x + ix * 2] =
                  pixels[(y * 4 + iy) * pstride + x * 4 + ix] - ctr;
            }
          }
          c[(y + 2) * 8 + x + 2] = c[y * 8 + x];
          c[y * 8 + x] = block_dc;
        }
      }
      const F b00 = c[0], b01 = c[1], b10 = c[8], b11 = c[9];
      c[0] = (b00 + b01 + b10 + b11) * F(0.25f);
      c[1] = (b00 + b01 - b10 - b11) * F(0.25f);
      c[8] = (b00 - b01 + b10 - b11) * F(0.25f);
      c[9] = (b00 - b01 - b10 + b11) * F(0.25f);
      break;
    }
    case kLINES: {
      const LinesMats& lm = LM();
      F temp[64];
      for (int y = 0; y < 8; ++y) {
        for (int x = 0; x < 8; ++x) temp[y * 8 + x] = pixels[y * pstride + x];
      }
      for (int i = 0; i < 64; ++i) c[i] = 0;
      auto dc_part = [&](const int* idx, int num) {
        F dc = 0;
        for (int i = 0; i < num; ++i) dc += temp[ColMajor(idx[i])];
        dc /= F(num);
        for (int i = 0; i < num; ++i) temp[ColMajor(idx[i])] -= dc;
        return dc;
      };
      F d00 = dc_part(kLinesDc00, 21), d01 = dc_part(kLinesDc01, 15);
      F d10 = dc_part(kLinesDc10, 15), d11 = dc_part(kLinesDc11, 13);
      const F r0 = (d00 + d01 + d10 + d11) * F(0.25f);
      const F r1 = (d00 - d01 + d10 - d11) * F(0.25f);
      const F r2 = (d00 + d01 - d10 - d11) * F(0.25f);
      const F r3 = (d00 - d01 - d10 + d11) * F(0.25f);
      c[0] = r0;
      c[8] = r1;
      c[1] = r2;
      c[9] = r3;
      auto dcts = [&](int n, const int* ip, const int* ic) {
        for (int k = 0; k < n; ++k) {
          F s = 0;
          for (int j = 0; j < n; ++j) {
            s += F(lm.fwd[n][k][j]) * temp[ColMajor(ip[j])];
          }
          c[ColMajor(ic[k])] = s;
        }
      };
      for (int i = 0; i < 4; ++i) dcts(3, kLinesP3[i], kLinesC3[i]);
      for (int i = 0; i < 4; ++i) dcts(4, kLinesP4[i], kLinesC4[i]);
      for (int i = 0; i < 4; ++i) dcts(6, kLinesP6[i], kLinesC6[i]);
      dcts(8, kLinesP8[0], kLinesC8[0]);
      break;
    }
  }
}

// LLF / LF helpers (pik/ac_strategy.cc:850-1056).
template <typename F>
void LowestFrequenciesFromDC(int type, const F* dc, size_t dc_stride, F* llf,
                             size_t llf_stride) {
  if (type == kDCT16X16) {
    F tmp[4];
    ReinterpretingDCT<F>(16, 2, dc, dc_stride, tmp, 2);
    for (int y = 0; y < 2; ++y) {
      for (int x = 0; x < 2; ++x) llf[y * llf_stride + x] = tmp[y * 2 + x];
    }
  } else if (type == kDCT32X32) {
    F tmp[16];
    ReinterpretingDCT<F>(32, 4, dc, dc_stride, tmp, 4);
    for (int y = 0; y < 4; ++y) {
      for (int x = 0; x < 4; ++x) llf[y * llf_stride + x] = tmp[y * 4 + x];
    }
  } else {
    llf[0] = dc[0];
  }
}

template <typename F>
void DC2x2FromLowestFrequencies(int type, const F* llf, size_t llf_stride,
                                F* dc2x2, size_t dc2x2_stride) {
  switch (type) {
    case kDCT:
    case kDCT_NOHF:
    case kLINES:
      ReinterpretingIDCT<F>(8, 1, 2, llf, 0, dc2x2, dc2x2_stride);
      break;
    case kDCT16X16: {
      F dest[16] = {};
      dest[0] = llf[0];
      dest[1] = llf[1];
      dest[4] = llf[llf_stride];
      dest[5] = llf[llf_stride + 1];
      ReinterpretingIDCT<F>(16, 2, 4, dest, 4, dc2x2, dc2x2_stride);
      break;
    }
    case kDCT32X32: {
      F dest[64] = {};
      for (int iy = 0; iy < 4; ++iy) {
        for (int ix = 0; ix < 4; ++ix) {
          dest[iy * 8 + ix] = llf[iy * llf_stride + ix];
        }
      }
      ReinterpretingIDCT<F>(32, 4, 8, dest, 8, dc2x2, dc2x2_stride);
      break;
    }
    default:
      dc2x2[0] = llf[0];
      dc2x2[1] = llf[0];
      dc2x2[dc2x2_stride] = llf[0];
      dc2x2[dc2x2_stride + 1] = llf[0];
      break;
  }
}

// `block` is the block's contiguous coefficient layout (rows of 8c).
template <typename F>
void DC2x2FromLowFrequencies(int type, const F* block, F* dc2x2,
                             size_t dc2x2_stride) {
  switch (type) {
    case kDCT:
    case kDCT_NOHF:
    case kLINES:
      ReinterpretingIDCT<F>(8, 2, 2, block, 8, dc2x2, dc2x2_stride);
      break;
    case kDCT16X16: {
      F dest[16] = {};
      for (int y = 0; y < 4; ++y) {
        for (int x = 0; x < 4; ++x) dest[4 * y + x] = block[16 * y + x];
      }
      ReinterpretingIDCT<F>(16, 4, 4, dest, 4, dc2x2, dc2x2_stride);
      break;
    }
    case kDCT32X32: {
      F dest[64] = {};
      for (int y = 0; y < 8; ++y) {
        for (int x = 0; x < 8; ++x) dest[8 * y + x] = block[32 * y + x];
      }
      ReinterpretingIDCT<F>(32, 8, 8, dest, 8, dc2x2, dc2x2_stride);
      break;
    }
    default: {
      const F b00 = block[0], b01 = block[1], b10 = block[8], b11 = block[9];
      dc2x2[0] = b00 + b01 + b10 + b11;
      dc2x2[1] = b00 + b01 - b10 - b11;
      dc2x2[dc2x2_stride] = b00 - b01 + b10 - b11;
      dc2x2[dc2x2_stride + 1] = b00 - b01 - b10 + b11;
      break;
    }
  }
}

template <typename F>
void LowFrequenciesFromDC2x2(int type, const F* dc2x2, size_t dc2x2_stride,
                             F* block, size_t block_stride) {
  switch (type) {
    case kDCT:
    case kDCT_NOHF:
    case kLINES:
      ReinterpretingDCT<F>(8, 2, dc2x2, dc2x2_stride, block, block_stride);
      break;
    case kDCT16X16: {
      F dest[16];
      ReinterpretingDCT<F>(16, 4, dc2x2, dc2x2_stride, dest, 4);
      for (int y = 0; y < 4; ++y) {
        for (int x = 0; x < 4; ++x) block[block_stride * y + x] = dest[y * 4 + x];
      }
      break;
    }
    case kDCT32X32: {
      F dest[64];
      ReinterpretingDCT<F>(32, 8, dc2x2, dc2x2_stride, dest, 8);
      for (int y = 0; y < 8; ++y) {
        for (int x = 0; x < 8; ++x) block[block_stride * y + x] = dest[y * 8 + x];
      }
      break;
    }
    default: {
      const F b00 = dc2x2[0], b01 = dc2x2[1];
      const F b10 = dc2x2[dc2x2_stride], b11 = dc2x2[dc2x2_stride + 1];
      block[0] = (b00 + b01 + b10 + b11) * F(0.25f);
      block[1] = (b00 + b01 - b10 - b11) * F(0.25f);
      block[block_stride] = (b00 - b01 + b10 - b11) * F(0.25f);
      block[block_stride + 1] = (b00 - b01 - b10 + b11) * F(0.25f);
      break;
    }
  }
}

// ---------------------------------------------------------------------------
// Planar images.

template <typename F>
struct Plane {
  int xs = 0, ys = 0;
  std::vector<F> v;
  Plane() {}
  Plane(int x, int y) : xs(x), ys(y), v(size_t(x) * y, F(0)) {}
  F* Row(int y) { return v.data() + size_t(y) * xs; }
  const F* Row(int y) const { return v.data() + size_t(y) * xs; }
  F& at(int x, int y) { return v[size_t(y) * xs + x]; }
  F at(int x, int y) const { return v[size_t(y) * xs + x]; }
};
template <typename F>
struct Img3 {
  Plane<F> p[3];
  Img3() {}
  Img3(int x, int y) {
    for (auto& q : p) q = Plane<F>(x, y);
  }
  int xs() const { return p[0].xs; }
  int ys() const { return p[0].ys; }
};

// Mirror (pik/image_ops.h:217-227): the edge sample is repeated once.
int Mirror(int x, int size) {
  while (x < 0 || x >= size) {
    if (x < 0) {
      x = -x - 1;
    } else {
      x = 2 * size - 1 - x;
    }
  }
  return x;
}

// Symmetric 3x3 convolution with mirrored borders, in the summation order
// of strategy::Symmetric3::WeightedSum (pik/convolve.h:611-629).
template <typename F>
void Symmetric3(const Plane<F>& in, float w0, float w1, float w2,
                Plane<F>* out) {
  const int xs = in.xs, ys = in.ys;
  *out = Plane<F>(xs, ys);
  for (int y = 0; y < ys; ++y) {
    const F* t = in.Row(Mirror(y - 1, ys));
    const F* m = in.Row(y);
    const F* b = in.Row(Mirror(y + 1, ys));
    F* o = out->Row(y);
    for (int x = 0; x < xs; ++x) {
      const int xl = Mirror(x - 1, xs), xr = Mirror(x + 1, xs);
      const F sum_tb = t[x] + b[x];
      const F mul0 = m[x] * F(w0);
      const F sum_lr = m[xl] + m[xr];
      const F x1 = sum_tb + sum_lr;
      const F mul1 = x1 * F(w1) + mul0;
      const F sum_t2 = t[xl] + t[xr];
      const F sum_b2 = b[xl] + b[xr];
      const F x2 = sum_t2 + sum_b2;
      o[x] = x2 * F(w2) + mul1;
    }
  }
}

// Gaborish weights (pik/gaborish.cc:16-88).
void GaborishWeights(int strength, float* w) {
  float wu1, wu2;
  switch (strength) {
    case 1:  // k500
      wu1 = static_cast<float>(0.056007960760453189);
      wu2 = static_cast<float>(0.045899074552453879);
      break;
    case 2: {  // k750
      const float x = 0.75;
      wu1 = static_cast<float>(x * 0.13959942428275746);
      wu2 = static_cast<float>(x * 0.074240717189152386);
      break;
    }
    case 3: {  // k875
      const float x = 0.875;
      wu1 = static_cast<float>(x * 0.11501538179658321);
      wu2 = static_cast<float>(x * 0.089979079587015454);
      break;
    }
    default:  // k1000
      wu1 = static_cast<float>(0.11501538179658321);
      wu2 = static_cast<float>(0.089979079587015454);
      break;
  }
  const float wu0 = 1.0f;
  const float mul = 1.0 / (wu0 + 4 * (wu1 + wu2));
  w[0] = wu0 * mul;
  w[1] = wu1 * mul;
  w[2] = wu2 * mul;
}

// ---------------------------------------------------------------------------
// EPF (pik/epf_target.cc:30-36, 253-428, 526-801, 1009-1278).

constexpr int kBorder = 6;
constexpr int kSigmaShift = 2;
constexpr int kMinSigma = 16;
constexpr int kMaxSigma = 672;

// WeightFast (pik/epf_target.cc:300-368): 2^x through IEEE-754 bits.
float WeightFastValue(int mul, int sad) {
  const int clamped = std::min(sad, 507);
  const int16_t prescaled = int16_t(clamped << 6);
  const int16_t unbiased = int16_t((int32_t(prescaled) * mul) >> 16);
  const int16_t biased = int16_t(unbiased + (127 << (23 - 16)));
  const uint32_t bits = uint32_t(uint16_t(biased)) << 16;
  float w;
  memcpy(&w, &bits, 4);
  return w;
}

// MulTable::Init (pik/epf_target.cc:371-413).
struct MulTable {
  int t[kMaxSigma + 1] = {};
  MulTable() {
    const int gap = 1 << kSigmaShift;
    int mul = -32768;
    for (int sigma = kMinSigma; sigma <= kMaxSigma; sigma += gap) {
      for (; mul < 0; ++mul) {
        if (WeightFastValue(mul, sigma >> kSigmaShift) > 0.5f) break;
      }
      t[sigma] = mul;
    }
    for (int sigma = kMinSigma; sigma < kMaxSigma; sigma += gap) {
      const float step = (t[sigma + gap] - t[sigma]) / float(gap);
      for (int i = 1; i < gap; ++i) t[sigma + i] = t[sigma] + i * step;
    }
  }
};
const MulTable& Mul() {
  static MulTable m;
  return m;
}

// SigmaFromQuant LUTs (pik/epf_target.cc:1160-1195).
float SigmaLut(int id, int i) {
  static const double base[16] = {
      1.9815775622811198, 1.9715084740908622, 1.6819963065873933,
      1.2146133632942862, 1.0395364091521881, 0.93552327583169714,
      0.68568655651684773, 0.51174440217871964, 0.36397262821018583,
      0.31621830414136975, 0.30262954326557712, 0.246314237855494,
      0.21617524864418683, 0.10, 0.05, 0.0};
  return static_cast<float>(id == 0 ? base[i] : base[i] / 2.0);
}

// SigmaFromQuant (pik/epf_target.cc:1072-1111).
int SigmaFromQuant(float signal, float stretch, int lut_id) {
  const float min_signal = 0.022156f;
  const float max_signal = 0.531738f;
  const float mul_signal = 29.435892f;
  float unscaled;
  if (signal <= min_signal) {
    unscaled = SigmaLut(lut_id, 0);
  } else if (signal >= max_signal) {
    unscaled = SigmaLut(lut_id, 15);
  } else {
    const float pos = (signal - min_signal) * mul_signal;
    const int64_t trunc = static_cast<int64_t>(pos);
    const float frac = pos - trunc;
    unscaled = frac * SigmaLut(lut_id, int(trunc) + 1) +
               (1.0f - frac) * SigmaLut(lut_id, int(trunc));
  }
  static const float kBias = 0.5182760822018414;
  const int sigma = unscaled * stretch + kBias;
  return std::min(sigma, kMaxSigma);
}

template <typename F>
Img3<F> PadMirror(const Img3<F>& in, int border) {
  Img3<F> out(in.xs() + 2 * border, in.ys() + 2 * border);
  for (int c = 0; c < 3; ++c) {
    for (int y = -border; y < in.ys() + border; ++y) {
      const F* src = in.p[c].Row(Mirror(y, in.ys()));
      F* dst = out.p[c].Row(y + border);
      for (int x = -border; x < in.xs() + border; ++x) {
        dst[x + border] = src[Mirror(x, in.xs())];
      }
    }
  }
  return out;
}

// AdaptiveFilter (pik/epf_target.cc:1113-1278). `in` is filtered with
// weights from `guide_src`; sigma per 8x8 block from qf/strategy/LUT.
// Decisions may be injected (guide with border, sigma per block).
// fixed_sigma >= 0: EpfParams::enable_adaptive is false, and every block
// takes that sigma (Filter, pik/epf_target.cc:1342-1386; FilterWorkers
// filters every block with it, and sigma 0 copies the image). The guide
// is formed the same way (MinMax of the guide source, MakeGuide).
template <typename F>
Img3<F> AdaptiveFilter(const Img3<F>& guide_src, const Img3<F>& in,
                       const int32_t* qf, const uint8_t* lut_ids,
                       const uint8_t* acs, const uint8_t* guide_in,
                       const int32_t* sigma_in, uint8_t* guide_out,
                       int32_t* sigma_out, int fixed_sigma = -1) {
  const int xs = in.xs(), ys = in.ys();
  const int bxs = xs / kBlockDim, bys = ys / kBlockDim;
  const Img3<F> padded_in = PadMirror(in, kBorder);
  const Img3<F> padded_guide = PadMirror(guide_src, kBorder);
  // MinMax over the padded guide (pik/epf_target.cc:980-1006).
  F mn[3], mx[3];
  for (int c = 0; c < 3; ++c) {
    mn[c] = mx[c] = padded_guide.p[c].v[0];
    for (F v : padded_guide.p[c].v) {
      mn[c] = std::min(mn[c], v);
      mx[c] = std::max(mx[c], v);
    }
  }
  const F all_max = std::max(std::max(mx[0], mx[1]), mx[2]);
  const F all_min = std::min(std::min(mn[0], mn[1]), mn[2]);
  // Stretch and guide scale are formed in float like the reference.
  const float range = float(all_max) - float(all_min);
  const float stretch = float(all_min) == float(all_max) ? 1.f : 255.0f / range;
  const F c_mul = range == 0.0f ? F(1.0f) : F(255.0f / range);
  const int gxs = xs + 2 * kBorder, gys = ys + 2 * kBorder;
  std::vector<uint8_t> guide(size_t(3) * gxs * gys);
  if (guide_in) {
    memcpy(guide.data(), guide_in, guide.size());
  } else {
    for (int c = 0; c < 3; ++c) {
      for (size_t i = 0; i < size_t(gxs) * gys; ++i) {
        const F scaled = (padded_guide.p[c].v[i] - all_min) * c_mul;
        const int32_t i32 = static_cast<int32_t>(scaled);
        guide[size_t(c) * gxs * gys + i] = static_cast<uint8_t>(uint32_t(i32));
      }
    }
  }
  if (guide_out) memcpy(guide_out, guide.data(), guide.size());

  Img3<F> out(xs, ys);
  const float quant_scale = 0.039324273f;
  for (int by = 0; by < bys; ++by) {
    for (int bx = 0; bx < bxs; ++bx) {
      const size_t bi = size_t(by) * bxs + bx;
      int sigma;
      if (sigma_in) {
        sigma = sigma_in[bi];
      } else if (fixed_sigma >= 0) {
        sigma = fixed_sigma;
      } else {
        const float ac_q = float(qf[bi]);
        const float scale = ARQuantScale(acs[bi] >> 4);
        const float quant = ac_q * scale * quant_scale;
        sigma = SigmaFromQuant(quant, stretch, lut_ids[bi]);
      }
      if (sigma_out) sigma_out[bi] = sigma;
      if (sigma < kMinSigma) {
        for (int c = 0; c < 3; ++c) {
          for (int iy = 0; iy < 8; ++iy) {
            for (int ix = 0; ix < 8; ++ix) {
              out.p[c].at(bx * 8 + ix, by * 8 + iy) =
                  in.p[c].at(bx * 8 + ix, by * 8 + iy);
            }
          }
        }
        continue;
      }
      const int mul = Mul().t[sigma];
      for (int iy = 0; iy < 8; ++iy) {
        for (int ix = 0; ix < 8; ++ix) {
          const int x = bx * 8 + ix, y = by * 8 + iy;
          // SAD over 3x4 patches for 7x8 neighbours, max over channels.
          float weights[56];
          for (int cy = -3; cy <= 3; ++cy) {
            for (int cx = -3; cx <= 4; ++cx) {
              int sad_max = 0;
              for (int c = 0; c < 3; ++c) {
                const uint8_t* g = guide.data() + size_t(c) * gxs * gys;
                int sad = 0;
                for (int py = -1; py <= 1; ++py) {
                  const uint8_t* rr = g + size_t(y + py + kBorder) * gxs;
                  const uint8_t* rw = g + size_t(y + cy + py + kBorder) * gxs;
                  for (int px = -1; px <= 2; ++px) {
                    sad += std::abs(int(rr[x + px + kBorder]) -
                                    int(rw[x + cx + px + kBorder]));
                  }
                }
                sad_max = std::max(sad_max, sad);
              }
              float w = WeightFastValue(mul, sad_max);
              if (!(w >= 0.05f)) w = 0.0f;
              weights[(cy + 3) * 8 + cx + 3] = w;
            }
          }
          for (int c = 0; c < 3; ++c) {
            F weighted_sum = 0, sum_weights = 0;
            int i = 0;
            for (int cy = -3; cy <= 3; ++cy) {
              const F* row = padded_in.p[c].Row(y + cy + kBorder);
              for (int cx = -3; cx <= 4; ++cx) {
                const F w = F(weights[i++]);
                weighted_sum += row[x + cx + kBorder] * w;
                sum_weights += w;
              }
            }
            out.p[c].at(x, y) = weighted_sum / sum_weights;
          }
        }
      }
    }
  }
  return out;
}

// ---------------------------------------------------------------------------
// The reconstruction.

struct Frame {
  const pikgpu_frame_params* p;
  const int16_t* ac;
  int xs, ys, bx, by, tx, ty;
  float inv_global_scale, inv_quant_dc;
  const float* Matrix(int table, int kind, int c) const {
    return p->dequant_table +
           p->dequant_offsets[(table * 7 + kind) * 3 + c];
  }
  int Acs(int x, int y) const { return p->ac_strategy[size_t(y) * bx + x]; }
  int Qf(int x, int y) const { return p->raw_quant_field[size_t(y) * bx + x]; }
};

template <typename F>
struct Recon {
  const Frame& f;
  // Adjoint checks only: per-cell factors on 1 / qf in the clamp intervals
  // (a quant field perturbed away from its integer values); NULL = 1.
  const double* ar_scale = nullptr;
  // Verification: the clamp's branch per coefficient, from another
  // implementation's forward pass (codes of pikgpu_get_clamp_decisions);
  // NULL = computed here.
  const uint8_t* clamp_tape = nullptr;
  explicit Recon(const Frame& fr) : f(fr) {}

  // Minimum ratio of a coefficient on the branch a clamp tape code names.
  static F TapeRatio(uint8_t code, const F ratio[3]) {
    return code == 0 ? F(1.0f) : code <= 3 ? ratio[code - 1] : F(0.0f);
  }

  // DequantDC (pik/compressed_dc.cc:181-231) with mul_dc from
  // DecodeDCGroups (pik/compressed_dc.cc:445-448).
  Img3<F> DequantDC() const {
    Img3<F> dc(f.bx, f.by);
    F mul_dc[3];
    for (int c = 0; c < 3; ++c) {
      mul_dc[c] = F(f.Matrix(0, 0, c)[0] * f.inv_quant_dc);
    }
    const F ytox = F(1.0f * float(f.p->ytox_dc - 128) * (1.0f / 256));
    const F ytob = F(1.0f * float(f.p->ytob_dc) * (1.0f / 128));
    const size_t n = size_t(f.bx) * f.by;
    const int16_t* q = f.p->quantized_dc;
    for (size_t i = 0; i < n; ++i) {
      const F y = F(q[n + i]) * mul_dc[1];
      dc.p[1].v[i] = y;
      dc.p[0].v[i] = ytox * y + F(q[i]) * mul_dc[0];
      dc.p[2].v[i] = ytob * y + F(q[2 * n + i]) * mul_dc[2];
    }
    return dc;
  }

  // AdaptiveDCReconstruction (pik/adaptive_reconstruction.cc:300-332).
  void DCRecon(Img3<F>* dc, const pikoracle_decisions* dec) const {
    const int pxs = (dc->xs() + 7) / 8 * 8, pys = (dc->ys() + 7) / 8 * 8;
    Img3<F> padded(pxs, pys);
    for (int c = 0; c < 3; ++c) {
      for (int y = 0; y < pys; ++y) {
        const int sy = std::min(y, dc->ys() - 1);
        for (int x = 0; x < pxs; ++x) {
          padded.p[c].at(x, y) = dc->p[c].at(std::min(x, dc->xs() - 1), sy);
        }
      }
    }
    const int nb = (pxs / 8) * (pys / 8);
    std::vector<int32_t> qf(nb, f.p->quant_dc / 2);
    std::vector<uint8_t> lut(nb, 0), acs(nb, 0);
    Img3<F> denoised = AdaptiveFilter<F>(
        padded, padded, qf.data(), lut.data(), acs.data(),
        dec ? dec->dc_guide : nullptr, dec ? dec->dc_sigma : nullptr,
        nullptr, nullptr);
    for (int c = 0; c < 3; ++c) {
      const F half_step =
          F(f.inv_quant_dc * f.Matrix(0, 0, c)[0] * 0.5f);
      for (int y = 0; y < dc->ys(); ++y) {
        for (int x = 0; x < dc->xs(); ++x) {
          F& v = dc->p[c].at(x, y);
          const F lo = v - half_step, hi = v + half_step;
          const F d = denoised.p[c].at(x, y);
          const F m = d < hi ? d : hi;  // std::min(denoised, dc + step)
          v = lo < m ? m : lo;          // std::max(dc - step, ...)
        }
      }
    }
  }

  // Dequant<true>::DoAC (pik/compressed_image.cc:586-707) over the frame.
  Img3<F> DequantAC() const {
    const size_t stride = size_t(f.bx) * 64;
    Img3<F> out(f.bx * 64, f.by);
    static const float kOneBias[3] = {0.05465007330715401f,
                                      0.07005449891748593f,
                                      0.049935103337343655f};
    const size_t plane = stride * f.by;
    for (int by = 0; by < f.by; ++by) {
      for (int bx = 0; bx < f.bx; ++bx) {
        const int qf = f.Qf(bx, by);
        const float scaled_dequant =
            qf == 0 ? 1E10f : f.inv_global_scale / qf;
        const int tx = bx / kTileDimInBlocks, ty = by / kTileDimInBlocks;
        const int cf = f.p->dequant_control_field[size_t(ty) * f.tx + tx];
        const int table = f.p->dequant_map[cf * 256 + (qf - 1)];
        const int acs = f.Acs(bx, by);
        const int kind = QuantKind(acs >> 4);
        const int blk = acs & 0xF;
        const float x_cc =
            1.0f * float(f.p->ytox_map[size_t(ty) * f.tx + tx] - 128) *
            (1.0f / 256);
        const float b_cc =
            1.0f * float(f.p->ytob_map[size_t(ty) * f.tx + tx]) * (1.0f / 128);
        const float* m[3];
        for (int c = 0; c < 3; ++c) m[c] = f.Matrix(table, kind, c) + blk * 64;
        for (int k = 0; k < 64; ++k) {
          const size_t pos = size_t(by) * stride + size_t(bx) * 64 + k;
          F dq[3];
          for (int c = 0; c < 3; ++c) {
            const F mulc = F(m[c][k]) * F(scaled_dequant);
            // AdjustQuantBias<c> (pik/quantizer.h:79-88), float form.
            const F q = F(f.ac[c * plane + pos]);
            const F qa = std::abs(q);
            F adj;
            if (qa >= F(1.5f)) {
              adj = q - F(0.145f) / q;
            } else if (qa >= F(0.5f)) {
              adj = std::copysign(F(1 - kOneBias[c]), q);
            } else {
              adj = q;
            }
            dq[c] = adj * mulc;
          }
          out.p[1].v[pos] = dq[1];
          out.p[0].v[pos] = F(x_cc) * dq[1] + dq[0];
          out.p[2].v[pos] = F(b_cc) * dq[1] + dq[2];
        }
      }
    }
    return out;
  }

  // ReconOpsinImage for one group (pik/compressed_image.cc:936-1106) with
  // ComputeLlf, PredictLf, UpdateLfForDecoder, AddPredictions
  // (pik/ac_predictions.cc:380-665) and InverseIntegralTransform (:869-934).
  void ReconGroup(int gx, int gy, const Img3<F>& dc_frame, Img3<F>* ac,
                  Img3<F>* idct) const {
    const int x0 = gx * kGroupDimInBlocks, y0 = gy * kGroupDimInBlocks;
    const int gxs = std::min(kGroupDimInBlocks, f.bx - x0);
    const int gys = std::min(kGroupDimInBlocks, f.by - y0);
    const bool predict_lf = f.p->predict_lf, predict_hf = f.p->predict_hf;
    auto acs_at = [&](int bx, int by) { return f.Acs(x0 + bx, y0 + by); };
    // Group DC with a one-block border (InitializeDecCache,
    // pik/compressed_dc.cc:530-556).
    const int dxs = gxs + 2, dys = gys + 2;
    Img3<F> dc(dxs, dys), llf(dxs, dys);
    for (int c = 0; c < 3; ++c) {
      for (int y = 0; y < dys; ++y) {
        for (int x = 0; x < dxs; ++x) {
          dc.p[c].at(x, y) = dc_frame.p[c].at(Mirror(x0 + x - 1, f.bx),
                                              Mirror(y0 + y - 1, f.by));
        }
      }
    }
    // ComputeLlf: border cells act as DCT8.
    for (int c = 0; c < 3; ++c) {
      for (int by = 0; by < dys; ++by) {
        for (int bx = 0; bx < dxs; ++bx) {
          const bool border =
              by == 0 || by == dys - 1 || bx == 0 || bx == dxs - 1;
          const int a = border ? 0 : acs_at(bx - 1, by - 1);
          if (a & 0xF) continue;  // not the first block
          LowestFrequenciesFromDC<F>(a >> 4, &dc.p[c].at(bx, by), dxs,
                                     &llf.p[c].at(bx, by), dxs);
        }
      }
    }
    const int w2 = dxs * 2, h2 = dys * 2;
    Img3<F> lf2x2(w2, h2), pred2x2(w2, h2);
    if (predict_lf) {
      static const float kW0 = 0.41459272584128337f;
      static const float kW1 = 0.25489157325704559f;
      static const float kW2 = 0.046449679523692139f;
      for (int c = 0; c < 3; ++c) {
        Plane<F> tmp(w2, h2);
        for (int by = 0; by < dys; ++by) {
          for (int bx = 0; bx < dxs; ++bx) {
            const bool border =
                by == 0 || by == dys - 1 || bx == 0 || bx == dxs - 1;
            const int a = border ? 0 : acs_at(bx - 1, by - 1);
            if (a & 0xF) continue;
            DC2x2FromLowestFrequencies<F>(a >> 4, &llf.p[c].at(bx, by), dxs,
                                          &tmp.at(2 * bx, 2 * by), w2);
          }
        }
        Symmetric3<F>(tmp, kW0, kW1, kW2, &lf2x2.p[c]);
        for (int by = 0; by < dys; ++by) {
          for (int bx = 0; bx < dxs; ++bx) {
            const bool border =
                by == 0 || by == dys - 1 || bx == 0 || bx == dxs - 1;
            const int a = border ? 0 : acs_at(bx - 1, by - 1);
            if (a & 0xF) continue;
            F* pos = &lf2x2.p[c].at(2 * bx, 2 * by);
            LowFrequenciesFromDC2x2<F>(a >> 4, pos, w2, pos, w2);
          }
        }
      }
    }
    // Border of pred2x2 (pik/compressed_image.cc:978-1039).
    if (predict_hf) {
      for (int c = 0; c < 3; ++c) {
        auto border_cell = [&](int x, int y) {
          if (predict_lf) {
            F block[64] = {};
            block[0] = llf.p[c].at(x, y);
            block[1] = lf2x2.p[c].at(2 * x + 1, 2 * y);
            block[8] = lf2x2.p[c].at(2 * x, 2 * y + 1);
            block[9] = lf2x2.p[c].at(2 * x + 1, 2 * y + 1);
            DC2x2FromLowFrequencies<F>(kDCT, block,
                                       &pred2x2.p[c].at(2 * x, 2 * y), w2);
          } else {
            DC2x2FromLowestFrequencies<F>(kDCT, &llf.p[c].at(x, y), dxs,
                                          &pred2x2.p[c].at(2 * x, 2 * y), w2);
          }
        };
        for (int x : {0, gxs + 1}) {
          for (int y = 0; y < gys + 2; ++y) border_cell(x, y);
        }
        for (int y : {0, gys + 1}) {
          for (int x = 0; x < gxs + 2; ++x) border_cell(x, y);
        }
      }
    }
    // UpdateLfForDecoder over the whole group (tiles are independent).
    const size_t astride = size_t(f.bx) * 64;
    for (int c = 0; c < 3; ++c) {
      for (int by = 0; by < gys; ++by) {
        for (int bx = 0; bx < gxs; ++bx) {
          const int a = acs_at(bx, by);
          if (a & 0xF) continue;
          const int type = a >> 4, cov = Covered(type);
          F* ac_pos = ac->p[c].v.data() + size_t(y0 + by) * astride +
                      size_t(x0 + bx) * 64;
          CoefView<F> blk{ac_pos, astride, 64 * cov};
          for (int y = 0; y < cov; ++y) {
            for (int x = 0; x < cov; ++x) {
              blk[cov * 8 * y + x] = llf.p[c].at(bx + 1 + x, by + 1 + y);
            }
          }
          if (predict_lf) {
            for (int y = 0; y < 2 * cov; ++y) {
              const int start = y < cov ? cov : 0;
              for (int x = start; x < 2 * cov; ++x) {
                blk[y * cov * 8 + x] +=
                    lf2x2.p[c].at(2 * (bx + 1) + x, 2 * (by + 1) + y);
              }
            }
          }
          if (predict_hf) {
            F block[32 * 32];
            const int n = 8 * cov;
            for (int i = 0; i < std::min(n * n, 8 * n); ++i) block[i] = blk[i];
            DC2x2FromLowFrequencies<F>(
                type, block, &pred2x2.p[c].at(2 * (bx + 1), 2 * (by + 1)), w2);
          }
        }
      }
    }
    // AddPredictions -> UpSample4x4BlurDCT<true> (pik/ac_predictions.cc:
    // 263-374, 652-665).
    if (predict_hf) {
      float kern[3][4];
      Ub4Kernel(kern);
      const int xsp = gxs * 2, ysp = gys * 2;
      for (int c = 0; c < 3; ++c) {
        Plane<F> blur_x(xsp * 4, ysp + 2);
        for (int y = 0; y < ysp + 2; ++y) {
          const F* row = pred2x2.p[c].Row(y + 1);
          F* out = blur_x.Row(y);
          for (int x = 0; x < xsp; ++x) {
            const F v0 = row[x + 1], v1 = row[x + 2], v2 = row[x + 3];
            for (int ix = 0; ix < 4; ++ix) {
              out[4 * x + ix] = v0 * F(kern[0][ix]) + v1 * F(kern[1][ix]) +
                                v2 * F(kern[2][ix]);
            }
          }
        }
        for (int by = 0; by < gys; ++by) {
          for (int bx = 0; bx < gxs; ++bx) {
            const int a = acs_at(bx, by);
            if (a & 0xF) continue;
            const int type = a >> 4;
            if (!PredictHF(type)) continue;
            const int cov = Covered(type), n = 8 * cov;
            F block[32 * 32];
            for (int idy = 0; idy < cov; ++idy) {
              const F* r0 = blur_x.Row(2 * (by + idy));
              const F* r1 = blur_x.Row(2 * (by + idy) + 1);
              const F* r2 = blur_x.Row(2 * (by + idy) + 2);
              const F* r3 = blur_x.Row(2 * (by + idy) + 3);
              for (int idx = 0; idx < cov; ++idx) {
                for (int ix = 0; ix < 8; ++ix) {
                  const int col = (bx + idx) * 8 + ix;
                  const F v0 = r0[col], v1 = r1[col], v2 = r2[col],
                          v3 = r3[col];
                  for (int iy = 0; iy < 4; ++iy) {
                    const F va = v0 * F(kern[0][iy]) + v1 * F(kern[1][iy]) +
                                 v2 * F(kern[2][iy]);
                    const F vb = v1 * F(kern[0][iy]) + v2 * F(kern[1][iy]) +
                                 v3 * F(kern[2][iy]);
                    block[(idy * 8 + iy) * 32 + idx * 8 + ix] = va;
                    block[(idy * 8 + iy + 4) * 32 + idx * 8 + ix] = vb;
                  }
                }
              }
            }
            F coeffs[32 * 32];
            TransformFromPixels<F>(type, block, 32, coeffs, size_t(n) * 8);
            // AddBlockExceptLFAndLLFTo<true> (pik/ac_predictions.cc:38-70).
            F* ac_pos = ac->p[c].v.data() + size_t(y0 + by) * astride +
                        size_t(x0 + bx) * 64;
            CoefView<F> blk{ac_pos, astride, 64 * cov};
            for (int y = 0; y < n; ++y) {
              for (int x = (y < 2 * cov ? 2 * cov : 0); x < n; ++x) {
                blk[y * n + x] += coeffs[y * n + x];
              }
            }
          }
        }
      }
    }
    // InverseIntegralTransform.
    for (int c = 0; c < 3; ++c) {
      for (int by = 0; by < gys; ++by) {
        for (int bx = 0; bx < gxs; ++bx) {
          const int a = acs_at(bx, by);
          if (a & 0xF) continue;
          const F* ac_pos = ac->p[c].v.data() + size_t(y0 + by) * astride +
                            size_t(x0 + bx) * 64;
          F* px = &idct->p[c].at((x0 + bx) * 8, (y0 + by) * 8);
          TransformToPixels<F>(a >> 4, ac_pos, astride, px, idct->xs());
        }
      }
    }
  }

  // ComputeUb4Kernel (pik/ac_predictions.cc:234-254) with GaussianKernel
  // (pik/gauss_blur.h:18-32) at sigma = k4x4BlurStrength.
  static void Ub4Kernel(float out[3][4]) {
    const float sigma = 2.0007879236394901f;
    const float scaler = -1.0 / (2 * sigma * sigma);
    float kernel[9];
    double sum = 0.0;
    for (int i = -4; i <= 4; ++i) {
      const float val = std::exp(scaler * i * i);
      kernel[i + 4] = val;
      sum += val;
    }
    for (int i = 0; i < 9; ++i) kernel[i] /= sum;
    for (int k = 0; k < 4; ++k) {
      out[0][k] = out[1][k] = out[2][k] = 0.0f;
      for (int j = 0; j < 4 - k; ++j) out[0][k] += kernel[j];
      for (int j = 4 - k; j < 8 - k; ++j) out[1][k] += kernel[j];
      for (int j = 8 - k; j < 9; ++j) out[2][k] += kernel[j];
    }
  }

  // AdaptiveReconstruction clamp (pik/adaptive_reconstruction.cc:72-244,
  // 334-471) applied to `filt` in place.
  void ARClamp(const Img3<F>& original, Img3<F>* filt) const {
    F dc_mul[3];
    for (int c = 0; c < 3; ++c) {
      dc_mul[c] = F(f.inv_quant_dc * f.Matrix(0, 0, c)[0]);
    }
    const int xs = original.xs();
    for (int by = 0; by < f.by; ++by) {
      for (int bx = 0; bx < f.bx; ++bx) {
        const int a = f.Acs(bx, by);
        if (a & 0xF) continue;
        const int type = a >> 4, cov = Covered(type), n = 8 * cov;
        const int qac = f.Qf(bx, by);
        const float inv_quant_ac_f = f.inv_global_scale / qac;
        const F inv_quant_ac =
            ar_scale ? F(inv_quant_ac_f) * F(ar_scale[size_t(by) * f.bx + bx])
                     : F(inv_quant_ac_f);
        const int tx = bx / kTileDimInBlocks, ty = by / kTileDimInBlocks;
        const int cf = f.p->dequant_control_field[size_t(ty) * f.tx + tx];
        const int table = f.p->dequant_map[cf * 256 + (qac - 1)];
        F blocks[3][32 * 32];
        F min_ratio[32 * 32];
        F ratios[32 * 32][3];
        for (int k = 0; k < n * n; ++k) min_ratio[k] = F(1.0f);
        for (int c = 0; c < 3; ++c) {
          const float* dm = f.Matrix(table, QuantKind(type), c);
          F diff[32 * 32];
          for (int iy = 0; iy < n; ++iy) {
            for (int ix = 0; ix < n; ++ix) {
              const int x = bx * 8 + ix, y = by * 8 + iy;
              diff[iy * n + ix] = filt->p[c].at(x, y) - original.p[c].at(x, y);
            }
          }
          TransformFromPixels<F>(type, diff, n, blocks[c], size_t(n) * 8);
          auto clamp = [&](int k, F interval) {
            const F upper = F(0.5f) * interval;
            const F lower = F(-0.5f) * interval;
            const F corr = blocks[c][k];
            const F mx = lower < corr ? corr : lower;
            const F clamped = mx < upper ? mx : upper;
            // Integer test: only +0.0 counts as zero.
            const bool is_zero = IsPositiveZero(corr);
            const F divisor = is_zero ? F(1E-7f) : corr;
            const F ratio = clamped / divisor;
            ratios[k][c] = ratio;
            min_ratio[k] = ratio < min_ratio[k] ? ratio : min_ratio[k];
          };
          for (int y = 0; y < cov; ++y) {
            for (int k = 0; k < std::min(32, n); ++k) {
              const int ofs = y * n + k;
              F interval;
              if (k < cov) {
                interval = F(ARLowestFrequencyScale(n, k, y)) *
                           (type == kDCT16X16 || type == kDCT32X32
                                ? dc_mul[c]
                                : dc_mul[c]);
                if (!(type == kDCT16X16 || type == kDCT32X32)) {
                  // llf scales {1, 0, ...}: only k = 0 for 8x8 types.
                  interval = F(1.0f) * dc_mul[c];
                }
              } else {
                interval = F(dm[ofs]) * inv_quant_ac;
              }
              clamp(ofs, interval);
            }
          }
          for (int k = cov * 8 * cov; k < n * n; ++k) {
            clamp(k, F(dm[k]) * inv_quant_ac);
          }
        }
        if (clamp_tape) {
          for (int k = 0; k < n * n; ++k) {
            const size_t o = size_t(by + k / (64 * cov)) * (size_t(f.bx) * 64) +
                             size_t(bx) * 64 + k % (64 * cov);
            min_ratio[k] = TapeRatio(clamp_tape[o], ratios[k]);
          }
        }
        for (int c = 0; c < 3; ++c) {
          for (int k = 0; k < n * n; ++k) blocks[c][k] *= min_ratio[k];
          F px[32 * 32];
          TransformToPixels<F>(type, blocks[c], size_t(n) * 8, px, n);
          for (int iy = 0; iy < n; ++iy) {
            for (int ix = 0; ix < n; ++ix) {
              const int x = bx * 8 + ix, y = by * 8 + iy;
              filt->p[c].at(x, y) = px[iy * n + ix] + original.p[c].at(x, y);
            }
          }
        }
        (void)xs;
      }
    }
  }

  static bool IsPositiveZero(F v) {
    if (v != F(0)) return false;
    return !std::signbit(v);
  }
};

// XybToRgb (pik/opsin_inverse.cc:38-88) and the inverse matrix
// (Inv3x3Matrix, pik/linalg.h:153-169, of kOpsinAbsorbanceMatrix,
// pik/opsin_params.h:20-31).
struct Opsin {
  float inv[9];
  float neg_bias[3];
  Opsin() {
    const float kScale = 255.0f;
    float m[9] = {
        static_cast<float>((0.29956550340058319) / kScale),
        static_cast<float>((0.63373087833825936) / kScale),
        static_cast<float>((0.077705617820981968) / kScale),
        static_cast<float>((0.22158691104574774) / kScale),
        static_cast<float>((0.68491388044116142) / kScale),
        static_cast<float>((0.096254234043612538) / kScale),
        static_cast<float>((0.20062661225219422) / kScale),
        static_cast<float>((0.070366199217588729) / kScale),
        static_cast<float>((0.5571760754215358) / kScale),
    };
    float t[9];
    t[0] = m[4] * m[8] - m[5] * m[7];
    t[1] = m[2] * m[7] - m[1] * m[8];
    t[2] = m[1] * m[5] - m[2] * m[4];
    t[3] = m[5] * m[6] - m[3] * m[8];
    t[4] = m[0] * m[8] - m[2] * m[6];
    t[5] = m[2] * m[3] - m[0] * m[5];
    t[6] = m[3] * m[7] - m[4] * m[6];
    t[7] = m[1] * m[6] - m[0] * m[7];
    t[8] = m[0] * m[4] - m[1] * m[3];
    const float idet = 1.0 / (m[0] * t[0] + m[1] * t[3] + m[2] * t[6]);
    for (int i = 0; i < 9; ++i) inv[i] = t[i] * idet;
    neg_bias[0] = -static_cast<float>((0.26786006338144885) / kScale);
    neg_bias[1] = -static_cast<float>((0.24494032763907073) / kScale);
    neg_bias[2] = -static_cast<float>((0.14255999980363571) / kScale);
  }
};
const Opsin& Op() {
  static Opsin o;
  return o;
}

template <typename F>
void XybToRgb(F x, F y, F b, F* r, F* g, F* bl) {
  const Opsin& o = Op();
  const F gr = F(1.0f) * (y + x);
  const F gg = F(1.0f) * (y - x);
  const F gb = b;
  const F mr = gr * gr * gr + F(o.neg_bias[0]);
  const F mg = gg * gg * gg + F(o.neg_bias[1]);
  const F mb = gb * gb * gb + F(o.neg_bias[2]);
  F lr = F(o.inv[0]) * mr, lg = F(o.inv[3]) * mr, lb = F(o.inv[6]) * mr;
  const F tr = F(o.inv[1]) * mg, tg = F(o.inv[4]) * mg, tb = F(o.inv[7]) * mg;
  lr = F(o.inv[2]) * mb + lr;
  lg = F(o.inv[5]) * mb + lg;
  lb = F(o.inv[8]) * mb + lb;
  *r = lr + tr;
  *g = lg + tg;
  *bl = lb + tb;
}

// sRGB-8 of one linear sample (0..255 scale): Image3ToTemp01 (*1/255,
// pik/external_image.cc:75-88), TF_SRGB::EncodedFromDisplay
// (pik/color_management.cc:323-349), CastClip01::FromTemp (:684-691) and
// ToExternal rounding (:192-197).
uint8_t Srgb8(float lin255) {
  static const float p[5] = {-5.135152395e-04f, 5.287254571e-03f,
                             3.903842876e-01f, 1.474205315e+00f,
                             7.352629620e-01f};
  static const float q[5] = {1.004519624e-02f, 3.036675394e-01f,
                             1.340816930e+00f, 9.258482155e-01f,
                             2.424867759e-02f};
  const float x = lin255 * (1.0f / 255);
  const float a = std::fabs(x);
  float mag;
  if (a > 0.0031308f) {
    const float s = std::sqrt(a);
    float yp = p[4], yq = q[4];
    for (int i = 3; i >= 0; --i) {
      yp = yp * s + p[i];
      yq = yq * s + q[i];
    }
    mag = yp / yq;
  } else {
    mag = a * 12.92f;
  }
  const float e = std::copysign(mag, x);
  const float clamped = std::min(std::max(0.0f, e), 1.0f);
  const float sample = clamped * 255.0f + 0.0f;
  return static_cast<uint8_t>(static_cast<int>(sample + 0.5f));
}

template <typename F>
void CopyOut(const Img3<F>& img, void* dst) {
  if (!dst) return;
  F* d = static_cast<F*>(dst);
  for (int c = 0; c < 3; ++c) {
    memcpy(d + size_t(c) * img.xs() * img.ys(), img.p[c].v.data(),
           img.p[c].v.size() * sizeof(F));
  }
}

template <typename F>
int Run(const pikgpu_frame_params* p, const int16_t* ac, void* const* stages,
        const pikoracle_decisions* dec, uint8_t* guide_out,
        int32_t* sigma_out) {
  Frame fr;
  fr.p = p;
  fr.ac = ac;
  fr.xs = p->xsize;
  fr.ys = p->ysize;
  fr.bx = (p->xsize + 7) / 8;
  fr.by = (p->ysize + 7) / 8;
  fr.tx = (p->xsize + 63) / 64;
  fr.ty = (p->ysize + 63) / 64;
  // Quantizer::RecomputeFromGlobalScale and Decode
  // (pik/quantizer.h:130-135, pik/quantizer.cc:63-71).
  fr.inv_global_scale = static_cast<float>(1.0 * 65536 / p->global_scale);
  fr.inv_quant_dc = fr.inv_global_scale / p->quant_dc;
  Recon<F> r(fr);
  r.clamp_tape = dec ? dec->clamp_tape : nullptr;

  Img3<F> dc = r.DequantDC();
  r.DCRecon(&dc, dec);
  CopyOut(dc, stages ? stages[0] : nullptr);

  Img3<F> ac_img = r.DequantAC();
  CopyOut(ac_img, stages ? stages[1] : nullptr);

  Img3<F> idct(fr.bx * 8, fr.by * 8);
  const int xg = (fr.bx + 63) / 64, yg = (fr.by + 63) / 64;
  for (int gy = 0; gy < yg; ++gy) {
    for (int gx = 0; gx < xg; ++gx) r.ReconGroup(gx, gy, dc, &ac_img, &idct);
  }
  CopyOut(idct, stages ? stages[2] : nullptr);

  float gw[3] = {0, 0, 0};
  if (p->gaborish) GaborishWeights(p->gaborish, gw);
  auto gaborish = [&](const Img3<F>& in) {
    Img3<F> out(in.xs(), in.ys());
    for (int c = 0; c < 3; ++c) {
      Symmetric3<F>(in.p[c], gw[0], gw[1], gw[2], &out.p[c]);
    }
    return out;
  };
  Img3<F> cur;
  if (p->have_adaptive_reconstruction) {
    Img3<F> smoothed = p->gaborish ? gaborish(idct) : idct;
    CopyOut(smoothed, stages ? stages[3] : nullptr);
    const Img3<F>& guide_src = p->epf_use_sharpened ? idct : smoothed;
    Img3<F> filt = AdaptiveFilter<F>(
        guide_src, idct, p->raw_quant_field, p->ar_sigma_lut_ids,
        p->ac_strategy, dec ? dec->guide : nullptr, dec ? dec->sigma : nullptr,
        guide_out, sigma_out,
        p->epf_enable_adaptive ? -1 : int(p->epf_sigma));
    CopyOut(filt, stages ? stages[4] : nullptr);
    r.ARClamp(idct, &filt);
    cur = std::move(filt);
  } else {
    if (stages && stages[3]) {
      CopyOut(p->gaborish ? gaborish(idct) : idct, stages[3]);
    }
    cur = std::move(idct);
  }
  CopyOut(cur, stages ? stages[5] : nullptr);
  if (p->gaborish) cur = gaborish(cur);
  // ShrinkTo(xsize, ysize) then OpsinToLinear.
  Img3<F> shrunk(fr.xs, fr.ys);
  for (int c = 0; c < 3; ++c) {
    for (int y = 0; y < fr.ys; ++y) {
      memcpy(shrunk.p[c].Row(y), cur.p[c].Row(y), fr.xs * sizeof(F));
    }
  }
  CopyOut(shrunk, stages ? stages[6] : nullptr);
  Img3<F> lin(fr.xs, fr.ys);
  const size_t n = size_t(fr.xs) * fr.ys;
  for (size_t i = 0; i < n; ++i) {
    XybToRgb<F>(shrunk.p[0].v[i], shrunk.p[1].v[i], shrunk.p[2].v[i],
                &lin.p[0].v[i], &lin.p[1].v[i], &lin.p[2].v[i]);
  }
  CopyOut(lin, stages ? stages[7] : nullptr);
  if (stages && stages[8]) {
    uint8_t* o = static_cast<uint8_t*>(stages[8]);
    for (size_t i = 0; i < n; ++i) {
      for (int c = 0; c < 3; ++c) o[3 * i + c] = Srgb8(float(lin.p[c].v[i]));
    }
  }
  return 0;
}

#include "pik_adjoint.inc"

}  // namespace

extern "C" {

int pikoracle_run_f32(const pikgpu_frame_params* p, const int16_t* ac,
                      void* const* stages, const pikoracle_decisions* dec,
                      uint8_t* guide_out, int32_t* sigma_out) {
  return Run<float>(p, ac, stages, dec, guide_out, sigma_out);
}

int pikoracle_adjoint_f64(const pikgpu_frame_params* p, const int16_t* ac,
                          const pikoracle_decisions* decisions_in,
                          const double* ac_dequant, const double* ar_scale,
                          const double* target, double* loss,
                          double* grad_ac, double* grad_qf) {
  if (!target) return -1;
  return Adjoint(p, ac, decisions_in, ac_dequant, ar_scale, target, loss,
                 grad_ac, grad_qf);
}

int pikoracle_run_f64(const pikgpu_frame_params* p, const int16_t* ac,
                      void* const* stages, const pikoracle_decisions* dec,
                      uint8_t* guide_out, int32_t* sigma_out) {
  return Run<double>(p, ac, stages, dec, guide_out, sigma_out);
}

int pikoracle_transform_f64(int type, int inverse, const double* in,
                            size_t in_stride, double* out,
                            size_t out_stride) {
  if (type < 0 || type > 8) return -1;
  if (inverse) {
    TransformToPixels<double>(type, in, in_stride, out, out_stride);
  } else {
    TransformFromPixels<double>(type, in, in_stride, out, out_stride);
  }
  return 0;
}

int pikoracle_transform_f32(int type, int inverse, const float* in,
                            size_t in_stride, float* out, size_t out_stride) {
  if (type < 0 || type > 8) return -1;
  if (inverse) {
    TransformToPixels<float>(type, in, in_stride, out, out_stride);
  } else {
    TransformFromPixels<float>(type, in, in_stride, out, out_stride);
  }
  return 0;
}

int pikoracle_lf_helper_f32(int type, int which, const float* in,
                            size_t in_stride, float* out, size_t out_stride) {
  switch (which) {
    case 0:
      LowestFrequenciesFromDC<float>(type, in, in_stride, out, out_stride);
      return 0;
    case 1:
      DC2x2FromLowestFrequencies<float>(type, in, in_stride, out, out_stride);
      return 0;
    case 2:
      DC2x2FromLowFrequencies<float>(type, in, out, out_stride);
      return 0;
    case 3:
      LowFrequenciesFromDC2x2<float>(type, in, in_stride, out, out_stride);
      return 0;
  }
  return -1;
}

float pikoracle_epf_weight(int sigma, int sad) {
  return WeightFastValue(Mul().t[sigma], sad);
}

void pikoracle_opsin_inverse_matrix(float* out9) {
  memcpy(out9, Op().inv, sizeof(float) * 9);
}

int pikoracle_dct_table(int n, int which, float* out) {
  if (n != 2 && n != 4 && n != 8 && n != 16 && n != 32) return -1;
  const Tables& t = T();
  const float* src = which == 0   ? t.ds[n]
                     : which == 1 ? t.is[n]
                     : which == 2 ? t.l1[n]
                                  : t.l1inv[n];
  memcpy(out, src, sizeof(float) * n);
  return 0;
}

}  // extern "C"
