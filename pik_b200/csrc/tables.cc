// Host construction of the constant tables (see tables.h).

#include "tables.h"

#include <string.h>

#include <algorithm>
#include <cmath>

namespace pikgpu {
namespace {

constexpr double kPi = 3.14159265358979323846;

// iscale_N(k) = sqrt(2/N) alpha(k) cos(k pi / 2N). The 8-point tables use
// the Arai-Agui-Nakajima convention (DCTScales = 1 / (N iscale),
// IDCTScales = iscale); all other sizes the flipped one (pik/dct.h:24-139).
double IScale(int n, int k) {
  const double alpha = k == 0 ? std::sqrt(0.5) : 1.0;
  return std::sqrt(2.0 / n) * alpha * std::cos(k * kPi / (2.0 * n));
}
float DctScale(int n, int k) {
  return static_cast<float>(n == 8 ? 1.0 / (n * IScale(n, k)) : IScale(n, k));
}
float IdctScale(int n, int k) {
  return static_cast<float>(n == 8 ? IScale(n, k) : 1.0 / (n * IScale(n, k)));
}
// Relative L1 norm of IDCT basis vector k (pik/dct.h:141-269): the product
// of cos(pi / 2^(j+3)) for j = 0 .. log2(N) - 2 - trailing_zeros(k); 1 for
// k = 0 and k = N/2.
double L1Norm(int n, int k) {
  if (k == 0 || k == n / 2) return 1.0;
  int tz = 0;
  while (((k >> tz) & 1) == 0) ++tz;
  int log2n = 0;
  while ((1 << log2n) < n) ++log2n;
  double norm = 1.0;
  for (int j = 0; j <= log2n - 2 - tz; ++j) {
    norm *= std::cos(kPi / double(1 << (j + 3)));
  }
  return norm;
}

}  // namespace

void BuildTables(DevTables* t) {
  memset(t, 0, sizeof(*t));
  for (int n : {2, 4, 8, 16, 32}) {
    float* a = t->idct + MatOffset(n);
    float* b = t->dct + MatOffset(n);
    for (int i = 0; i < n; ++i) {
      for (int k = 0; k < n; ++k) {
        const double alpha = k == 0 ? std::sqrt(0.5) : 1.0;
        const double s = n * std::sqrt(2.0 / n) * alpha;
        a[i * n + k] = static_cast<float>(s * double(DctScale(n, k)) *
                                          std::cos(k * (i + 0.5) * kPi / n));
        b[k * n + i] = static_cast<float>(s * double(IdctScale(n, k)) *
                                          std::cos((i + 0.5) * k * kPi / n));
      }
    }
    const int si = SizeIndex(n);
    for (int y = 0; y < 8 && y < n; ++y) {
      for (int x = 0; x < 8 && x < n; ++x) {
        const float l1x = static_cast<float>(L1Norm(n, x));
        const float l1y = static_cast<float>(L1Norm(n, y));
        const float l1ix = static_cast<float>(1.0 / L1Norm(n, x));
        const float l1iy = static_cast<float>(1.0 / L1Norm(n, y));
        // Float arithmetic left to right, as the constexpr originals.
        t->total_scale[si][y][x] =
            float(n) * DctScale(n, x) * DctScale(n, y) * l1ix * l1iy;
        t->inv_total_scale[si][y][x] =
            float(n) * IdctScale(n, x) * IdctScale(n, y) * l1x * l1y;
      }
    }
  }
  for (int y = 0; y < 2; ++y) {
    for (int x = 0; x < 2; ++x) t->ar_llf16[y][x] = t->inv_total_scale[3][y][x];
  }
  for (int y = 0; y < 4; ++y) {
    for (int x = 0; x < 4; ++x) t->ar_llf32[y][x] = t->inv_total_scale[4][y][x];
  }
  // LINES: scaled DCT-II/III pairs; forward scale 1/n (k = 0), 2/n (n = 3,
  // 6) or sqrt(2)/n (n = 4, 8); inverse scale makes them inverse.
  for (int n : {3, 4, 6, 8}) {
    for (int k = 0; k < n; ++k) {
      const double s = k == 0 ? 1.0 / n
                       : (n == 3 || n == 6) ? 2.0 / n
                                            : 2.0 / n / std::sqrt(2.0);
      const double inv = (k == 0 ? 1.0 / n : 2.0 / n) / s;
      for (int x = 0; x < n; ++x) {
        const double c = std::cos(k * (x + 0.5) * kPi / n);
        t->lines_fwd[n][k][x] = static_cast<float>(s * c);
        t->lines_inv[n][x][k] = static_cast<float>(inv * c);
      }
    }
  }
  // GaussianKernel(4, sigma) (pik/gauss_blur.h:18-32) folded into the 4x
  // upsampling kernel (ComputeUb4Kernel).
  {
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
      float o0 = 0, o1 = 0, o2 = 0;
      for (int j = 0; j < 4 - k; ++j) o0 += kernel[j];
      for (int j = 4 - k; j < 8 - k; ++j) o1 += kernel[j];
      for (int j = 8 - k; j < 9; ++j) o2 += kernel[j];
      t->ub4[0][k] = o0;
      t->ub4[1][k] = o1;
      t->ub4[2][k] = o2;
    }
    const float* b16 = t->dct + MatOffset(16);
    for (int k = 0; k < 4; ++k)
      for (int m = 0; m < 6; ++m) {
        double acc = 0.0;
        for (int x = 0; x < 16; ++x) {
          const int i = m - x / 4;
          if (i >= 0 && i <= 2) {
            acc += double(b16[k * 16 + x]) * double(t->ub4[i][x % 4]);
          }
        }
        t->hf_corner16[k][m] = float(acc);
      }
    const float* b32 = t->dct + MatOffset(32);
    for (int k = 0; k < 8; ++k)
      for (int m = 0; m < 10; ++m) {
        double acc = 0.0;
        for (int x = 0; x < 32; ++x) {
          const int i = m - x / 4;
          if (i >= 0 && i <= 2) {
            acc += double(b32[k * 32 + x]) * double(t->ub4[i][x % 4]);
          }
        }
        t->hf_corner32[k][m] = float(acc);
      }
  }
  t->lf_blur[0] = 0.41459272584128337f;
  t->lf_blur[1] = 0.25489157325704559f;
  t->lf_blur[2] = 0.046449679523692139f;
  for (int s = 1; s <= 4; ++s) {
    float wu1, wu2;
    if (s == 1) {
      wu1 = static_cast<float>(0.056007960760453189);
      wu2 = static_cast<float>(0.045899074552453879);
    } else if (s == 2) {
      const float x = 0.75;
      wu1 = static_cast<float>(x * 0.13959942428275746);
      wu2 = static_cast<float>(x * 0.074240717189152386);
    } else if (s == 3) {
      const float x = 0.875;
      wu1 = static_cast<float>(x * 0.11501538179658321);
      wu2 = static_cast<float>(x * 0.089979079587015454);
    } else {
      wu1 = static_cast<float>(0.11501538179658321);
      wu2 = static_cast<float>(0.089979079587015454);
    }
    const float wu0 = 1.0f;
    const float mul = 1.0 / (wu0 + 4 * (wu1 + wu2));
    t->gaborish[s][0] = wu0 * mul;
    t->gaborish[s][1] = wu1 * mul;
    t->gaborish[s][2] = wu2 * mul;
  }
  // Opsin absorbance matrix / 255 and its inverse (pik/opsin_params.h:20-44,
  // Inv3x3Matrix pik/linalg.h:153-169, in float).
  {
    const float kScale = 255.0f;
    const float m[9] = {
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
    float c[9];
    c[0] = m[4] * m[8] - m[5] * m[7];
    c[1] = m[2] * m[7] - m[1] * m[8];
    c[2] = m[1] * m[5] - m[2] * m[4];
    c[3] = m[5] * m[6] - m[3] * m[8];
    c[4] = m[0] * m[8] - m[2] * m[6];
    c[5] = m[2] * m[3] - m[0] * m[5];
    c[6] = m[3] * m[7] - m[4] * m[6];
    c[7] = m[1] * m[6] - m[0] * m[7];
    c[8] = m[0] * m[4] - m[1] * m[3];
    const float idet = 1.0 / (m[0] * c[0] + m[1] * c[3] + m[2] * c[6]);
    for (int i = 0; i < 9; ++i) t->opsin_inv[i] = c[i] * idet;
    t->opsin_neg_bias[0] = -static_cast<float>((0.26786006338144885) / kScale);
    t->opsin_neg_bias[1] = -static_cast<float>((0.24494032763907073) / kScale);
    t->opsin_neg_bias[2] = -static_cast<float>((0.14255999980363571) / kScale);
  }
  t->one_bias[0] = 0.05465007330715401f;
  t->one_bias[1] = 0.07005449891748593f;
  t->one_bias[2] = 0.049935103337343655f;
  // MulTable: for each sigma (step 4), the first multiplier whose weight at
  // SAD = sigma / 4 exceeds 0.5, searching upward from -32768 and carrying
  // the search position; then linear interpolation in between.
  {
    auto weight = [](int mul, int sad) {
      const int clamped = sad < 507 ? sad : 507;
      const int16_t prescaled = int16_t(clamped << 6);
      const int16_t unbiased = int16_t((int32_t(prescaled) * mul) >> 16);
      const int16_t biased = int16_t(unbiased + (127 << 7));
      const uint32_t bits = uint32_t(uint16_t(biased)) << 16;
      float w;
      memcpy(&w, &bits, 4);
      return w;
    };
    const int gap = 1 << kSigmaShift;
    int mul = -32768;
    for (int sigma = kMinSigma; sigma <= kMaxSigma; sigma += gap) {
      for (; mul < 0; ++mul) {
        if (weight(mul, sigma >> kSigmaShift) > 0.5f) break;
      }
      t->mul_table[sigma] = mul;
    }
    for (int sigma = kMinSigma; sigma < kMaxSigma; sigma += gap) {
      const float step = (t->mul_table[sigma + gap] - t->mul_table[sigma]) /
                         float(gap);
      for (int i = 1; i < gap; ++i) {
        t->mul_table[sigma + i] = t->mul_table[sigma] + i * step;
      }
    }
    // The weight falls as the SAD grows: scan down from the clamp.
    for (int sigma = 0; sigma < kMinSigma; ++sigma) t->epf_thr[sigma] = 507;
    for (int sigma = kMinSigma; sigma <= kMaxSigma; ++sigma) {
      const int m64 = t->mul_table[sigma] * 64;
      auto w = [&](int sad) {
        const uint32_t u =
            (uint32_t(std::min(sad, 507) * m64) & 0xFFFF0000u) + 0x3F800000u;
        float f;
        memcpy(&f, &u, 4);
        return f;
      };
      int thr = 507;
      while (thr > 0 && !(w(thr) >= 0.05f)) --thr;
      t->epf_thr[sigma] = thr;
    }
  }
  {
    static const double lut[16] = {
        1.9815775622811198, 1.9715084740908622, 1.6819963065873933,
        1.2146133632942862, 1.0395364091521881, 0.93552327583169714,
        0.68568655651684773, 0.51174440217871964, 0.36397262821018583,
        0.31621830414136975, 0.30262954326557712, 0.246314237855494,
        0.21617524864418683, 0.10, 0.05, 0.0};
    for (int i = 0; i < 16; ++i) {
      t->sigma_lut[0][i] = static_cast<float>(lut[i]);
      t->sigma_lut[1][i] = static_cast<float>(lut[i] / 2.0);
    }
  }
  {
    const float p[5] = {-5.135152395e-04f, 5.287254571e-03f,
                        3.903842876e-01f, 1.474205315e+00f, 7.352629620e-01f};
    const float q[5] = {1.004519624e-02f, 3.036675394e-01f, 1.340816930e+00f,
                        9.258482155e-01f, 2.424867759e-02f};
    memcpy(t->srgb_p, p, sizeof(p));
    memcpy(t->srgb_q, q, sizeof(q));
  }
}

}  // namespace pikgpu
