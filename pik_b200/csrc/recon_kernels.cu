// Included by pikgpu.cu (single translation unit, so the __constant__
// tables need no relocatable device code).
//
// Reconstruction kernels: DC, dequantisation, LF/HF prediction, the
// variable-size inverse transforms, gaborish, EPF, the DCT-domain clamp and
// XYB -> linear RGB / sRGB-8. Each kernel names the reference function it
// implements (paths relative to the google/pik checkout).

#include "kernels.cuh"


namespace pikgpu {

__constant__ DevTables c_t;

namespace {

__device__ __forceinline__ const float* IdctMat(int n) {
  return c_t.idct + MatOffset(n);
}
__device__ __forceinline__ const float* DctMat(int n) {
  return c_t.dct + MatOffset(n);
}

// ---------------------------------------------------------------------------
// Single-thread transforms used by the small LF kernels (n <= 8).

// tsIDCT (pik/dct.h:441-507): out = A C^T A^T (C row = horizontal freq).
// Runtime size n <= 8: compact loops (these run once per block in the LF
// kernels, where code size and registers matter more than unrolling).
__device__ void TsIdct1(int n, const float* in, int is, float* out, int os) {
  const float* a = IdctMat(n);
  float tmp[64];
  for (int k = 0; k < n; ++k) {
    for (int v = 0; v < n; ++v) {
      float s = 0.f;
      for (int l = 0; l < n; ++l) s += in[k * is + l] * a[v * n + l];
      tmp[k * n + v] = s;
    }
  }
  for (int v = 0; v < n; ++v) {
    for (int u = 0; u < n; ++u) {
      float s = 0.f;
      for (int k = 0; k < n; ++k) s += a[u * n + k] * tmp[k * n + v];
      out[v * os + u] = s;
    }
  }
}

// tsDCT with ScaleToBlock (pik/dct.h:362-428, pik/block.h:103-132).
__device__ void TsDct1(int n, const float* in, int is, float* out, int os) {
  const float* b = DctMat(n);
  float tmp[64];
  for (int k = 0; k < n; ++k) {
    for (int y = 0; y < n; ++y) {
      float s = 0.f;
      for (int x = 0; x < n; ++x) s += b[k * n + x] * in[y * is + x];
      tmp[k * n + y] = s;
    }
  }
  const float scale = 1.0f / float(n * n);
  for (int k = 0; k < n; ++k) {
    for (int l = 0; l < n; ++l) {
      float s = 0.f;
      for (int y = 0; y < n; ++y) s += tmp[k * n + y] * b[l * n + y];
      out[k * os + l] = s * scale;
    }
  }
}

// The same two transforms for N <= 4, unrolled into registers (the same
// sums in the same order).
template <int N>
__device__ __forceinline__ void TsIdctSmall(const float* in, int is,
                                            float* out, int os) {
  const float* a = IdctMat(N);
  float tmp[N * N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
#pragma unroll
    for (int v = 0; v < N; ++v) {
      float s = 0.f;
#pragma unroll
      for (int l = 0; l < N; ++l) s += in[k * is + l] * a[v * N + l];
      tmp[k * N + v] = s;
    }
  }
#pragma unroll
  for (int v = 0; v < N; ++v) {
#pragma unroll
    for (int u = 0; u < N; ++u) {
      float s = 0.f;
#pragma unroll
      for (int k = 0; k < N; ++k) s += a[u * N + k] * tmp[k * N + v];
      out[v * os + u] = s;
    }
  }
}
template <int N>
__device__ __forceinline__ void TsDctSmall(const float* in, int is, float* out,
                                           int os) {
  const float* b = DctMat(N);
  float tmp[N * N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
#pragma unroll
    for (int y = 0; y < N; ++y) {
      float s = 0.f;
#pragma unroll
      for (int x = 0; x < N; ++x) s += b[k * N + x] * in[y * is + x];
      tmp[k * N + y] = s;
    }
  }
  const float scale = 1.0f / float(N * N);
#pragma unroll
  for (int k = 0; k < N; ++k) {
#pragma unroll
    for (int l = 0; l < N; ++l) {
      float s = 0.f;
#pragma unroll
      for (int y = 0; y < N; ++y) s += tmp[k * N + y] * b[l * N + y];
      out[k * os + l] = s * scale;
    }
  }
}

// ReinterpretingDCT / ReinterpretingIDCT (pik/ac_strategy.cc:270-311).
template <int DCTN, int N>
__device__ void ReinterpDct(const float* in, int is, float* out, int os) {
  float block[N * N], res[N * N];
#pragma unroll
  for (int y = 0; y < N; ++y) {
#pragma unroll
    for (int x = 0; x < N; ++x) block[y * N + x] = in[y * is + x];
  }
  if constexpr (N <= 4) {
    TsDctSmall<N>(block, N, res, N);
  } else {
    TsDct1(N, block, N, res, N);
  }
  constexpr int sn = SizeIndex(N), sd = SizeIndex(DCTN);
#pragma unroll
  for (int y = 0; y < N; ++y) {
#pragma unroll
    for (int x = 0; x < N; ++x) {
      out[y * os + x] = res[y * N + x] * c_t.total_scale[sn][y][x] *
                        c_t.inv_total_scale[sd][y][x];
    }
  }
}
template <int DCTN, int LF, int N>
__device__ void ReinterpIdct(const float* in, int is, float* out, int os) {
  float block[N * N];
#pragma unroll
  for (int i = 0; i < N * N; ++i) block[i] = 0.f;
  constexpr int sn = SizeIndex(N), sd = SizeIndex(DCTN);
#pragma unroll
  for (int y = 0; y < LF; ++y) {
#pragma unroll
    for (int x = 0; x < LF; ++x) {
      block[y * N + x] = in[y * is + x] * c_t.inv_total_scale[sn][y][x] *
                         c_t.total_scale[sd][y][x];
    }
  }
  if constexpr (N <= 4) {
    TsIdctSmall<N>(block, N, out, os);
  } else {
    TsIdct1(N, block, N, out, os);
  }
}

// AcStrategy LLF/LF helpers (pik/ac_strategy.cc:850-1056).
__device__ void LowestFreqFromDC(int type, const float* dc, int ds, float* llf,
                                 int ls) {
  if (type == kDCT16X16) {
    float t[4];
    ReinterpDct<16, 2>(dc, ds, t, 2);
    for (int y = 0; y < 2; ++y)
      for (int x = 0; x < 2; ++x) llf[y * ls + x] = t[y * 2 + x];
  } else if (type == kDCT32X32) {
    float t[16];
    ReinterpDct<32, 4>(dc, ds, t, 4);
    for (int y = 0; y < 4; ++y)
      for (int x = 0; x < 4; ++x) llf[y * ls + x] = t[y * 4 + x];
  } else {
    llf[0] = dc[0];
  }
}

__device__ void DC2x2FromLowestFreq(int type, const float* llf, int ls,
                                    float* d, int dstr) {
  if (type == kDCT || type == kDCT_NOHF || type == kLINES) {
    ReinterpIdct<8, 1, 2>(llf, 0, d, dstr);
  } else if (type == kDCT16X16) {
    float dest[16];
    for (int i = 0; i < 16; ++i) dest[i] = 0.f;
    dest[0] = llf[0];
    dest[1] = llf[1];
    dest[4] = llf[ls];
    dest[5] = llf[ls + 1];
    ReinterpIdct<16, 2, 4>(dest, 4, d, dstr);
  } else if (type == kDCT32X32) {
    float dest[64];
    for (int i = 0; i < 64; ++i) dest[i] = 0.f;
    for (int iy = 0; iy < 4; ++iy)
      for (int ix = 0; ix < 4; ++ix) dest[iy * 8 + ix] = llf[iy * ls + ix];
    ReinterpIdct<32, 4, 8>(dest, 8, d, dstr);
  } else {
    d[0] = llf[0];
    d[1] = llf[0];
    d[dstr] = llf[0];
    d[dstr + 1] = llf[0];
  }
}

// `blk(i)` reads element i of the block's coefficient matrix.
template <class Blk>
__device__ void DC2x2FromLowFreq(int type, const Blk& blk, float* d,
                                 int dstr) {
  if (type == kDCT || type == kDCT_NOHF || type == kLINES) {
    float in[4] = {blk(0), blk(1), blk(8), blk(9)};
    ReinterpIdct<8, 2, 2>(in, 2, d, dstr);
  } else if (type == kDCT16X16) {
    float dest[16];
    for (int y = 0; y < 4; ++y)
      for (int x = 0; x < 4; ++x) dest[4 * y + x] = blk(16 * y + x);
    ReinterpIdct<16, 4, 4>(dest, 4, d, dstr);
  } else if (type == kDCT32X32) {
    float dest[64];
    for (int y = 0; y < 8; ++y)
      for (int x = 0; x < 8; ++x) dest[8 * y + x] = blk(32 * y + x);
    ReinterpIdct<32, 8, 8>(dest, 8, d, dstr);
  } else {
    const float b00 = blk(0), b01 = blk(1), b10 = blk(8), b11 = blk(9);
    d[0] = b00 + b01 + b10 + b11;
    d[1] = b00 + b01 - b10 - b11;
    d[dstr] = b00 - b01 + b10 - b11;
    d[dstr + 1] = b00 - b01 - b10 + b11;
  }
}

__device__ void LowFreqFromDC2x2(int type, float* d, int dstr) {
  if (type == kDCT || type == kDCT_NOHF || type == kLINES) {
    float out[4];
    ReinterpDct<8, 2>(d, dstr, out, 2);
    d[0] = out[0];
    d[1] = out[1];
    d[dstr] = out[2];
    d[dstr + 1] = out[3];
  } else if (type == kDCT16X16) {
    float out[16];
    ReinterpDct<16, 4>(d, dstr, out, 4);
    for (int y = 0; y < 4; ++y)
      for (int x = 0; x < 4; ++x) d[dstr * y + x] = out[y * 4 + x];
  } else if (type == kDCT32X32) {
    float out[64];
    ReinterpDct<32, 8>(d, dstr, out, 8);
    for (int y = 0; y < 8; ++y)
      for (int x = 0; x < 8; ++x) d[dstr * y + x] = out[y * 8 + x];
  } else {
    const float b00 = d[0], b01 = d[1], b10 = d[dstr], b11 = d[dstr + 1];
    d[0] = (b00 + b01 + b10 + b11) * 0.25f;
    d[1] = (b00 + b01 - b10 - b11) * 0.25f;
    d[dstr] = (b00 - b01 + b10 - b11) * 0.25f;
    d[dstr + 1] = (b00 - b01 - b10 + b11) * 0.25f;
  }
}

__device__ __forceinline__ void GroupDims(const Geo& g, int gi, int* x0,
                                          int* y0, int* gxs, int* gys) {
  const int gx = gi % g.Gx, gy = gi / g.Gx;
  *x0 = gx * 64;
  *y0 = gy * 64;
  *gxs = min(64, g.Bx - *x0);
  *gys = min(64, g.By - *y0);
}

}  // namespace

// ---------------------------------------------------------------------------
// Min/max of 3 planes (MinMax, pik/epf_target.cc:980-1006): ordered-integer
// atomics. mm[0..2] = min, mm[3..5] = max (encoded).
__device__ __forceinline__ uint32_t OrderedBits(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__host__ __device__ inline float FromOrderedBits(uint32_t u) {
  const uint32_t b = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
#ifdef __CUDA_ARCH__
  return __uint_as_float(b);
#else
  float f;
  memcpy(&f, &b, 4);
  return f;
#endif
}

// Start of a frame: the two min/max sets (the frame EPF's at mm[0..5], the
// DC EPF's at mm[8..13]) reset to empty, and `n` counters to 0.
__global__ void k_frame_init(uint32_t* mm, int* counters, int n) {
  const int t = threadIdx.x;
  if (t < 16) mm[t] = (t & 7) < 3 ? 0xFFFFFFFFu : 0u;
  if (t < n) counters[t] = 0;
}

__global__ void __launch_bounds__(256)
    k_minmax(const float* planes, size_t n, uint32_t* mm) {
  PdlLaunchDependents();  // the EPF may start on free SMs
  __shared__ uint32_t s_lo[8], s_hi[8];
  const int c = blockIdx.y;
  const float* p = planes + size_t(c) * n;
  uint32_t lo = 0xFFFFFFFFu, hi = 0u;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x) {
    const uint32_t o = OrderedBits(p[i]);
    lo = min(lo, o);
    hi = max(hi, o);
  }
  for (int off = 16; off; off >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, off));
    hi = max(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, off));
  }
  if ((threadIdx.x & 31) == 0) {
    s_lo[threadIdx.x >> 5] = lo;
    s_hi[threadIdx.x >> 5] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < 8; ++i) {
      lo = min(lo, s_lo[i]);
      hi = max(hi, s_hi[i]);
    }
    atomicMin(&mm[c], lo);
    atomicMax(&mm[3 + c], hi);
  }
}

// DC: DequantDC (pik/compressed_dc.cc:181-231) into `dc`, the 8-padded copy
// of AdaptiveDCReconstruction (PadImageToMultiple, pik/image.cc:45-77: the
// last column and row replicated) into `pad` (3 x ph x pw), and its
// min/max (MinMax, pik/epf_target.cc:980-1006; replication adds no value)
// into mm[0..5]. One thread per padded position, all three channels.
__global__ void __launch_bounds__(256)
    k_dc_prep(Geo g, DevFrame f, FrameScalars s, float* pad, int pw, int ph,
              uint32_t* mm) {
  __shared__ uint32_t s_mm[8][6];
  const int x = blockIdx.x * 32 + (threadIdx.x & 31);
  const int y = blockIdx.y * 8 + (threadIdx.x >> 5);
  uint32_t lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, hi[3] = {0, 0, 0};
  if (x < pw && y < ph) {
    const int n = g.Bx * g.By;
    const int i = min(y, g.By - 1) * g.Bx + min(x, g.Bx - 1);
    const float yv = float(f.qdc[n + i]) * s.mul_dc[1];
    const float v[3] = {s.ytox_dc * yv + float(f.qdc[i]) * s.mul_dc[0], yv,
                        s.ytob_dc * yv + float(f.qdc[2 * n + i]) * s.mul_dc[2]};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (x < g.Bx && y < g.By) f.dc[c * n + i] = v[c];
      pad[(size_t(c) * ph + y) * pw + x] = v[c];
      lo[c] = hi[c] = OrderedBits(v[c]);
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    for (int off = 16; off; off >>= 1) {
      lo[c] = min(lo[c], __shfl_xor_sync(0xFFFFFFFFu, lo[c], off));
      hi[c] = max(hi[c], __shfl_xor_sync(0xFFFFFFFFu, hi[c], off));
    }
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) s_mm[w][c] = lo[c], s_mm[w][3 + c] = hi[c];
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    const int k = threadIdx.x;
    uint32_t v = s_mm[0][k];
    for (int i = 1; i < 8; ++i) v = k < 3 ? min(v, s_mm[i][k]) : max(v, s_mm[i][k]);
    if (k < 3) atomicMin(&mm[k], v);
    else atomicMax(&mm[k], v);
  }
}

// Stretch and guide multiplier from the min/max (AdaptiveFilter and
// MakeGuide, pik/epf_target.cc:1040-1047, 1140-1151).
__device__ __forceinline__ void GuideParams(const uint32_t* mm, float* all_min,
                                            float* mul, float* stretch) {
  const float mn0 = FromOrderedBits(mm[0]), mn1 = FromOrderedBits(mm[1]),
              mn2 = FromOrderedBits(mm[2]);
  const float mx0 = FromOrderedBits(mm[3]), mx1 = FromOrderedBits(mm[4]),
              mx2 = FromOrderedBits(mm[5]);
  const float amax = fmaxf(fmaxf(mx0, mx1), mx2);
  const float amin = fminf(fminf(mn0, mn1), mn2);
  const float range = amax - amin;
  *all_min = amin;
  *mul = range == 0.0f ? 1.0f : 255.0f / range;
  *stretch = amin == amax ? 1.0f : 255.0f / range;
}

// SigmaFromQuant (pik/epf_target.cc:1072-1111) of one 8x8 block with raw
// quant field ac_q, strategy scale (ARQuantScale) and LUT `lut_id`.
__device__ __forceinline__ int SigmaFromQuant(float ac_q, float scale,
                                              int lut_id, float stretch) {
  const float quant = ac_q * scale * 0.039324273f;
  float unscaled;
  const float* l = c_t.sigma_lut[lut_id];
  if (quant <= 0.022156f) {
    unscaled = l[0];
  } else if (quant >= 0.531738f) {
    unscaled = l[15];
  } else {
    const float pos = (quant - 0.022156f) * 29.435892f;
    const int trunc = int(pos);
    const float frac = pos - float(trunc);
    unscaled = frac * l[trunc + 1] + (1.0f - frac) * l[trunc];
  }
  const int sg = int(unscaled * stretch + 0.5182760822018414f);
  return min(sg, kMaxSigma);
}

// Guide decision export (verification hook): u8 guide with the 6-pixel
// mirrored border, 3 x (h + 12) x (w + 12).
__global__ void k_export_guide(const float* src, int w, int h,
                               const uint32_t* mm, uint8_t* guide) {
  const int gx = blockIdx.x * blockDim.x + threadIdx.x - 6;
  const int gy = blockIdx.y * blockDim.y + threadIdx.y - 6;
  const int c = blockIdx.z;
  if (gx >= w + 6 || gy >= h + 6) return;
  float amin, mul, stretch;
  GuideParams(mm, &amin, &mul, &stretch);
  const float s = src[(size_t(c) * h + MirrorIdx(gy, h)) * w + MirrorIdx(gx, w)];
  guide[(size_t(c) * (h + 12) + gy + 6) * (w + 12) + gx + 6] =
      uint8_t(uint32_t(__float2int_rz((s - amin) * mul)));
}

// ---------------------------------------------------------------------------
// sRGB-8 of one linear value on the 0..255 scale: TF_SRGB's rational
// polynomial (pik/color_management.cc:323-345) and the rounding of
// ExternalImage::CopyTo (pik/external_image.cc:1205). The gaborish / opsin
// stencil kernels are in stencil_kernels.cuh.
// TF_SRGB::EncodedFromDisplay of a linear value on the 0..255 scale after
// Image3ToTemp01's x (1 / 255) (pik/external_image.cc:79-90).
__device__ __forceinline__ float SrgbEncoded(float lin255) {
  const float x = lin255 * (1.0f / 255);
  const float a = fabsf(x);
  float mag;
  if (a > 0.0031308f) {
    const float s = sqrtf(a);
    float yp = c_t.srgb_p[4], yq = c_t.srgb_q[4];
    for (int i = 3; i >= 0; --i) {
      yp = yp * s + c_t.srgb_p[i];
      yq = yq * s + c_t.srgb_q[i];
    }
    mag = yp / yq;
  } else {
    mag = a * 12.92f;
  }
  return copysignf(mag, x);
}

__device__ __forceinline__ uint8_t Srgb8(float lin255) {
  const float x = lin255 * (1.0f / 255);
  const float a = fabsf(x);
  float mag;
  if (a > 0.0031308f) {
    const float s = sqrtf(a);
    float yp = c_t.srgb_p[4], yq = c_t.srgb_q[4];
    for (int i = 3; i >= 0; --i) {
      yp = yp * s + c_t.srgb_p[i];
      yq = yq * s + c_t.srgb_q[i];
    }
    mag = yp / yq;
  } else {
    mag = a * 12.92f;
  }
  const float e = copysignf(mag, x);
  const float cl = fminf(fmaxf(0.0f, e), 1.0f);
  const float sample = cl * 255.0f + 0.0f;
  return uint8_t(int(sample + 0.5f));
}

// ---------------------------------------------------------------------------
// The output-format step of dpik's writer (EncodeImagePNM,
// pik/codec_pnm.cc:260-294, through ExternalImage, pik/external_image.cc):
// the body of a PPM (8 or 16 bits per sample, big-endian) or PFM (32-bit
// little-endian floats) file, rows top to bottom, RGB interleaved, from the
// linear planes (0..255 scale, row stride `stride` floats). Each sample is
// Image3ToTemp01's value (x (1 / 255)), transfer-encoded to sRGB if
// `srgb` (else kept linear), then:
//  8 / 16 bits: CastClip01 (clamp to [0, 1], x (2^bits - 1) + 0) and
//               ToExternal's int(sample + 0.5f) (pik/external_image.cc:
//               192-205, 666-696);
//  32 bits:     CastFloat01's x 255 (pik/external_image.cc:754-773).
// One thread per pixel.
__global__ void k_encode_pnm(const float* lin, size_t stride, int w, int h,
                             int bits, int srgb, uint8_t* out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= w) return;
  const size_t plane = stride * h;
  const size_t p = size_t(y) * w + x;
  for (int c = 0; c < 3; ++c) {
    const float v = lin[c * plane + size_t(y) * stride + x];
    const float e = srgb ? SrgbEncoded(v) : v * (1.0f / 255);
    if (bits == 32) {
      const uint32_t u = __float_as_uint(e * 255.0f);
      uint8_t* o = out + 4 * (3 * p + c);
      o[0] = uint8_t(u), o[1] = uint8_t(u >> 8);
      o[2] = uint8_t(u >> 16), o[3] = uint8_t(u >> 24);
    } else {
      const float width = bits == 8 ? 255.0f : 65535.0f;
      const float cl = fminf(fmaxf(0.0f, e), 1.0f);
      const int q = int(cl * width + 0.0f + 0.5f);
      if (bits == 8) {
        out[3 * p + c] = uint8_t(q);
      } else {
        out[2 * (3 * p + c)] = uint8_t(q >> 8);
        out[2 * (3 * p + c) + 1] = uint8_t(q);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// AC dequantisation + chroma from luma (Dequant<true>::DoAC,
// pik/compressed_image.cc:586-707). Each thread dequantises kDequantCoefs
// consecutive coefficients of one cell in all three channels (vector loads
// of the int16 input and the matrix row, 128-bit stores); a CTA covers
// 256 / (64 / kDequantCoefs) cells of one block row. The loads come first,
// the int16 coefficients, then the chain quant field -> table -> matrix
// row. Four coefficients per thread: 0.040 ms at 4K against 0.048 with
// eight (twice the threads; the kernel is bound by latency, not traffic).
constexpr int kDequantCoefs = 4;
constexpr int kDequantCells = 256 / (64 / kDequantCoefs);

__device__ __forceinline__ float AdjustQuantBias(float q, float one_bias) {
  const float qa = fabsf(q);
  if (qa >= 1.5f) return q - 0.145f / q;
  if (qa >= 0.5f) return copysignf(1.0f - one_bias, q);
  return q;
}

__global__ void __launch_bounds__(256) k_dequant_ac(Geo g, DevFrame f,
                                                    FrameScalars s) {
  constexpr int K = kDequantCoefs, TPC = 64 / K;
  static_assert(K == 4 || K == 8, "uint2 or uint4 loads of the int16 input");
  const int part = threadIdx.x % TPC;  // coefficients K part .. K part + K-1
  const int bx = blockIdx.x * kDequantCells + threadIdx.x / TPC;
  const int by = blockIdx.y;
  if (bx >= g.Bx) return;
  const size_t plane = size_t(g.ac_stride) * g.By;
  const size_t pos = size_t(by) * g.ac_stride + size_t(bx) * 64 + K * part;
  uint32_t raw[3][K / 2];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int16_t* src = f.qac + c * plane + pos;
    if constexpr (K == 8) {
      const uint4 v = *reinterpret_cast<const uint4*>(src);
      raw[c][0] = v.x, raw[c][1] = v.y, raw[c][2] = v.z, raw[c][3] = v.w;
    } else {
      const uint2 v = *reinterpret_cast<const uint2*>(src);
      raw[c][0] = v.x, raw[c][1] = v.y;
    }
  }
  const int cell = by * g.Bx + bx;
  const int qf = f.qf[cell];
  const float scaled = qf == 0 ? 1E10f : s.inv_global_scale / float(qf);
  const int tx = bx >> 3, ty = by >> 3;
  const int cf = f.dq_cf[ty * g.Tx + tx];
  const int table = f.dq_map[cf * 256 + (qf - 1)];
  const int a = f.acs[cell];
  const int kind = QuantKindOf(a >> 4);
  const int blk = a & 0xF;
  const float x_cc = 1.0f * float(f.ytox[ty * g.Tx + tx] - 128) * (1.0f / 256);
  const float b_cc = 1.0f * float(f.ytob[ty * g.Tx + tx]) * (1.0f / 128);
  float dq[3][K];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float* m = f.table + f.offsets[(table * 7 + kind) * 3 + c] +
                     blk * 64 + K * part;
    float mv[K];
    if ((reinterpret_cast<uintptr_t>(m) & 15) == 0) {
#pragma unroll
      for (int i = 0; i < K / 4; ++i) {
        const float4 v = reinterpret_cast<const float4*>(m)[i];
        mv[4 * i] = v.x, mv[4 * i + 1] = v.y, mv[4 * i + 2] = v.z,
               mv[4 * i + 3] = v.w;
      }
    } else {
#pragma unroll
      for (int k = 0; k < K; ++k) mv[k] = m[k];
    }
    const float ob = c_t.one_bias[c];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int16_t qi = int16_t(raw[c][k >> 1] >> (16 * (k & 1)));
      const float mulc = mv[k] * scaled;
      dq[c][k] = AdjustQuantBias(float(qi), ob) * mulc;
    }
  }
  float o0[K], o2[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    o0[k] = x_cc * dq[1][k] + dq[0][k];
    o2[k] = b_cc * dq[1][k] + dq[2][k];
  }
  float4* d0 = reinterpret_cast<float4*>(f.ac + pos);
  float4* d1 = reinterpret_cast<float4*>(f.ac + plane + pos);
  float4* d2 = reinterpret_cast<float4*>(f.ac + 2 * plane + pos);
#pragma unroll
  for (int i = 0; i < K / 4; ++i) {
    d1[i] = make_float4(dq[1][4 * i], dq[1][4 * i + 1], dq[1][4 * i + 2],
                        dq[1][4 * i + 3]);
    d0[i] = make_float4(o0[4 * i], o0[4 * i + 1], o0[4 * i + 2],
                        o0[4 * i + 3]);
    d2[i] = make_float4(o2[4 * i], o2[4 * i + 1], o2[4 * i + 2],
                        o2[4 * i + 3]);
  }
}

// ---------------------------------------------------------------------------
// LF prediction (ComputeLlf, PredictLf, pik/ac_predictions.cc:380-470) and
// UpdateLfForDecoder (pik/ac_predictions.cc:560-635,
// pik/compressed_image.cc:978-1084), per 512x512 group as the reference
// computes them. Group-local cell (X, Y) in [0, gxs+2) x [0, gys+2): the
// group's cells shifted by one, with a border ring that acts as DCT8; DC
// from the frame with mirroring (InitializeDecCache,
// pik/compressed_dc.cc:530-556). The 2x2 image of the group is
// 2 (gxs + 2) x 2 (gys + 2), mirrored at its edges by the blur.
//
// A CTA (k_lf_tile) takes one channel of a tile of kLfTile x kLfTile cells
// of a group and keeps the images it needs in shared memory: the LLF and
// 2x2 images of every block that reaches the tile's blurred range (one
// cell beyond the tile, and the ring where the tile touches it), so its
// first cell may lie up to 3 cells before that range (DCT32X32).
struct LfGroup {
  int gi, c, x0, y0, gxs, gys;
  __device__ int Acs(const Geo& g, const DevFrame& f, int bx, int by) const {
    const bool border = bx == 0 || by == 0 || bx == gxs + 1 || by == gys + 1;
    return border ? 0 : f.acs[(y0 + by - 1) * g.Bx + x0 + bx - 1];
  }
};

constexpr int kLfTile = 16;           // cells per tile side
constexpr int kLfWin = kLfTile + 12;  // shared-memory window, cells
constexpr int kLfWin2 = 2 * kLfWin;   // the 2x2 images' window, pixels
constexpr int kLfThreads = 128;
// Shared memory of k_lf_tile: the LLF image, the 2x2 image before and after
// LFPredictionBlur, over the window, and the list of the window's first
// cells (by block size: 8x8-class blocks, then 16x16, then 32x32).
constexpr int kLfList1 = kLfWin * kLfWin;
constexpr int kLfList2 = (kLfWin / 2 + 1) * (kLfWin / 2 + 1);
constexpr int kLfList4 = (kLfWin / 4 + 1) * (kLfWin / 4 + 1);
constexpr size_t kLfSmemBytes =
    4 * (size_t(kLfWin) * kLfWin + 2 * size_t(kLfWin2) * kLfWin2 + kLfList1 +
         kLfList2 + kLfList4);

// The window of a tile: cell (X, Y) of the group is at (X - ex, Y - ey).
struct LfWin {
  int ex, ey;
  float* llf;  // kLfWin x kLfWin
  float* tmp;  // kLfWin2 x kLfWin2
  float* lf;   // kLfWin2 x kLfWin2
  __device__ float* Llf(int X, int Y) const {
    return llf + (Y - ey) * kLfWin + (X - ex);
  }
  __device__ float* Tmp(int X2, int Y2) const {
    return tmp + (Y2 - 2 * ey) * kLfWin2 + (X2 - 2 * ex);
  }
  __device__ float* Lf(int X2, int Y2) const {
    return lf + (Y2 - 2 * ey) * kLfWin2 + (X2 - 2 * ex);
  }
};

__device__ void LlfCell(const Geo& g, const DevFrame& f, const LfGroup& q,
                        const LfWin& w, int a, int bx, int by) {
  const int type = a >> 4, cov = Covered(type);
  float dc[16];
  for (int iy = 0; iy < cov; ++iy)
    for (int ix = 0; ix < cov; ++ix)
      dc[iy * 4 + ix] =
          f.dc[(size_t(q.c) * g.By + MirrorIdx(q.y0 + by - 1 + iy, g.By)) *
                   g.Bx +
               MirrorIdx(q.x0 + bx - 1 + ix, g.Bx)];
  LowestFreqFromDC(type, dc, 4, w.Llf(bx, by), kLfWin);
}

// LFPredictionBlur over the group's 2x2 image (ConvolveT<Symmetric3>,
// mirrored at the image's edges) for the run of up to 8 pixels x0 ..
// x0 + n - 1 of row y: the 3 x (n + 2) inputs are loaded once, and each
// output keeps Symmetric3's operation order.
__device__ void LfBlurRun(const LfGroup& q, const LfWin& w, int x0, int y,
                          int n) {
  const int w2 = 2 * (q.gxs + 2), h2 = 2 * (q.gys + 2);
  const int yr[3] = {MirrorIdx(y - 1, h2), y, MirrorIdx(y + 1, h2)};
  float v[3][10];
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    if (i < n + 2) {
      const int x = MirrorIdx(x0 - 1 + i, w2);
#pragma unroll
      for (int j = 0; j < 3; ++j) v[j][i] = *w.Tmp(x, yr[j]);
    }
  }
  const float w0 = c_t.lf_blur[0], w1 = c_t.lf_blur[1], w2_ = c_t.lf_blur[2];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    if (i < n) {
      const float sum_tb = v[0][i + 1] + v[2][i + 1];
      const float mul0 = v[1][i + 1] * w0;
      const float sum_lr = v[1][i] + v[1][i + 2];
      const float x1 = sum_tb + sum_lr;
      const float mul1 = x1 * w1 + mul0;
      const float sum_t2 = v[0][i] + v[0][i + 2];
      const float sum_b2 = v[2][i] + v[2][i + 2];
      const float x2 = sum_t2 + sum_b2;
      *w.Lf(x0 + i, y) = x2 * w2_ + mul1;
    }
  }
}

// Ring cell (x, y) of pred2x2 (pik/compressed_image.cc:978-1039).
__device__ void PredBorderCell(const DevFrame& f, const LfGroup& q,
                               const LfWin& w, int x, int y,
                               int predict_lf) {
  float* pred = f.pred2x2_g + q.gi * kG2GroupFloats + q.c * kG2 * kG2;
  if (predict_lf) {
    float blk[10];
    blk[0] = *w.Llf(x, y);
    blk[1] = *w.Lf(2 * x + 1, 2 * y);
    blk[8] = *w.Lf(2 * x, 2 * y + 1);
    blk[9] = *w.Lf(2 * x + 1, 2 * y + 1);
    DC2x2FromLowFreq(kDCT, [&](int k) { return blk[k]; },
                     pred + 2 * y * kG2 + 2 * x, kG2);
  } else {
    DC2x2FromLowestFreq(kDCT, w.Llf(x, y), kLfWin,
                        pred + 2 * y * kG2 + 2 * x, kG2);
  }
}

// UpdateLfForDecoder for the first block at group cell (X, Y), in place on
// the dequantised AC: the LLF from DC into the block's corner, the LF
// prediction added to the LF coefficients, and the block's pred2x2 cells
// from the updated corner.
__device__ void LfUpdateBlock(const Geo& g, const DevFrame& f,
                              const LfGroup& q, const LfWin& w, int type,
                              int X, int Y, int predict_lf, int predict_hf) {
  const int bx = q.x0 + X - 1, by = q.y0 + Y - 1, c = q.c;
  const int cov = Covered(type);
  float* base = f.ac + size_t(c) * g.ac_stride * g.By +
                size_t(by) * g.ac_stride + size_t(bx) * 64;
  const int chunk = 64 * cov;
  auto at = [&](int i) -> float& {
    return base[(i / chunk) * size_t(g.ac_stride) + i % chunk];
  };
  for (int y = 0; y < cov; ++y)
    for (int x = 0; x < cov; ++x) at(cov * 8 * y + x) = *w.Llf(X + x, Y + y);
  if (predict_lf) {
    for (int y = 0; y < 2 * cov; ++y) {
      const int start = y < cov ? cov : 0;
      for (int x = start; x < 2 * cov; ++x) {
        at(y * cov * 8 + x) += *w.Lf(2 * X + x, 2 * Y + y);
      }
    }
  }
  if (predict_hf) {
    float* pred = f.pred2x2_g + q.gi * kG2GroupFloats + c * kG2 * kG2;
    DC2x2FromLowFreq(type, [&](int i) { return at(i); },
                     pred + 2 * Y * kG2 + 2 * X, kG2);
  }
}

// One channel of one tile: blockIdx.x = tile, blockIdx.y = group,
// blockIdx.z = channel. Phases (a barrier between them): LLF and the 2x2
// image of every block whose first cell is in [lo - 4, hi + 1) (the blur
// reads cells lo - 1 .. hi), then the blur and LowFrequenciesFromDC2x2 over
// [lo, hi) -- the tile plus the ring cells beside it -- then the ring's
// pred2x2 and the update of the tile's blocks.
__global__ void __launch_bounds__(kLfThreads, 4)
    k_lf_tile(Geo g, DevFrame f, int predict_lf, int predict_hf) {
  extern __shared__ float lf_smem[];
  LfGroup q;
  q.gi = blockIdx.y;
  q.c = blockIdx.z;
  GroupDims(g, q.gi, &q.x0, &q.y0, &q.gxs, &q.gys);
  const int ntx = (q.gxs + kLfTile - 1) / kLfTile;
  const int tx = blockIdx.x % ntx, ty = blockIdx.x / ntx;
  if (ty * kLfTile >= q.gys) return;
  // The tile's cells [X0, X1) x [Y0, Y1); the LF range adds the ring.
  const int X0 = 1 + tx * kLfTile, X1 = min(X0 + kLfTile, q.gxs + 1);
  const int Y0 = 1 + ty * kLfTile, Y1 = min(Y0 + kLfTile, q.gys + 1);
  const int lx = X0 == 1 ? 0 : X0, hx = X1 == q.gxs + 1 ? q.gxs + 2 : X1;
  const int ly = Y0 == 1 ? 0 : Y0, hy = Y1 == q.gys + 1 ? q.gys + 2 : Y1;
  LfWin w;
  w.ex = lx - 4;
  w.ey = ly - 4;
  w.llf = lf_smem;
  w.tmp = w.llf + kLfWin * kLfWin;
  w.lf = w.tmp + kLfWin2 * kLfWin2;
  // The first cells of the blocks reaching cells lx - 1 .. hx (clipped to
  // the group's ring), listed as X | Y << 10 | strategy byte << 20, so that
  // the per-block phases below give every lane a block (a cell-per-lane
  // loop leaves the lanes of the other cells of multi-block transforms
  // idle). One list per block size, read as one after the other, so that a
  // warp's lanes mostly take the same transform sizes (the 32x32 blocks'
  // LF transforms are far longer than the others').
  __shared__ int s_n[3];
  int* lists[3];
  lists[0] = reinterpret_cast<int*>(w.lf + kLfWin2 * kLfWin2);
  lists[1] = lists[0] + kLfList1;
  lists[2] = lists[1] + kLfList2;
  if (threadIdx.x < 3) s_n[threadIdx.x] = 0;
  __syncthreads();
  const int sx = max(lx - 4, 0), sy = max(ly - 4, 0);
  const int nx = min(hx + 1, q.gxs + 2) - sx, ny = min(hy + 1, q.gys + 2) - sy;
  for (int i = threadIdx.x; i < nx * ny; i += kLfThreads) {
    const int X = sx + i % nx, Y = sy + i / nx;
    const int a = q.Acs(g, f, X, Y);
    if (a & 0xF) continue;
    const int cov = Covered(a >> 4), k = cov == 1 ? 0 : cov == 2 ? 1 : 2;
    lists[k][atomicAdd(&s_n[k], 1)] = X | (Y << 10) | (a << 20);
  }
  __syncthreads();
  const int n0 = s_n[0], n01 = n0 + s_n[1], nfirst = n01 + s_n[2];
  auto first_at = [&](int i) {
    return i < n0 ? lists[0][i] : i < n01 ? lists[1][i - n0]
                                          : lists[2][i - n01];
  };
  for (int i = threadIdx.x; i < nfirst; i += kLfThreads) {
    const int e = first_at(i);
    const int X = e & 1023, Y = (e >> 10) & 1023, a = e >> 20;
    LlfCell(g, f, q, w, a, X, Y);
    if (predict_lf) {
      DC2x2FromLowestFreq(a >> 4, w.Llf(X, Y), kLfWin, w.Tmp(2 * X, 2 * Y),
                          kLfWin2);
    }
  }
  __syncthreads();
  if (predict_lf) {
    // Runs of 8 pixels of the blurred range's rows.
    const int w2 = 2 * (hx - lx), runs = (w2 + 7) / 8;
    const int n2 = runs * 2 * (hy - ly);
    for (int i = threadIdx.x; i < n2; i += kLfThreads) {
      const int r = i % runs, y = 2 * ly + i / runs;
      LfBlurRun(q, w, 2 * lx + 8 * r, y, min(8, w2 - 8 * r));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nfirst; i += kLfThreads) {
      const int e = first_at(i);
      const int X = e & 1023, Y = (e >> 10) & 1023, a = e >> 20;
      if (X < lx || X >= hx || Y < ly || Y >= hy) continue;
      LowFreqFromDC2x2(a >> 4, w.Lf(2 * X, 2 * Y), kLfWin2);
    }
    __syncthreads();
  }
  if (predict_hf) {
    // Ring cells beside the tile: left/right columns, then top/bottom rows.
    const int rows = hy - ly, cols = hx - lx;
    for (int i = threadIdx.x; i < 2 * rows + 2 * cols; i += kLfThreads) {
      int X, Y;
      if (i < 2 * rows) {
        X = (i & 1) ? q.gxs + 1 : 0;
        Y = ly + (i >> 1);
        if ((X == 0 && lx != 0) || (X != 0 && hx != q.gxs + 2)) continue;
      } else {
        const int j = i - 2 * rows;
        Y = (j & 1) ? q.gys + 1 : 0;
        X = lx + (j >> 1);
        if ((Y == 0 && ly != 0) || (Y != 0 && hy != q.gys + 2)) continue;
        // Corner cells belong to the columns' pass.
        if (X == 0 || X == q.gxs + 1) continue;
      }
      PredBorderCell(f, q, w, X, Y, predict_lf);
    }
  }
  for (int i = threadIdx.x; i < nfirst; i += kLfThreads) {
    const int e = first_at(i);
    const int X = e & 1023, Y = (e >> 10) & 1023, a = e >> 20;
    if (X < X0 || X >= X1 || Y < Y0 || Y >= Y1) continue;
    LfUpdateBlock(g, f, q, w, a >> 4, X, Y, predict_lf, predict_hf);
  }
}

// ---------------------------------------------------------------------------
// Cooperative batched transforms in shared memory. `nb` blocks of n x n,
// contiguous in smem; T threads; every thread calls __syncthreads.
__device__ void CoopTsIdct(int n, int nb, const float* a, const float* in,
                           float* tmp, float* out) {
  const int nn = n * n;
  for (int i = threadIdx.x; i < nb * nn; i += blockDim.x) {
    const int b = i / nn, r = i % nn, k = r / n, v = r % n;
    const float* src = in + b * nn + k * n;
    float s = 0.f;
    for (int l = 0; l < n; ++l) s += src[l] * a[v * n + l];
    tmp[b * nn + k * n + v] = s;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nb * nn; i += blockDim.x) {
    const int b = i / nn, r = i % nn, v = r / n, u = r % n;
    const float* t = tmp + b * nn;
    float s = 0.f;
    for (int k = 0; k < n; ++k) s += a[u * n + k] * t[k * n + v];
    out[b * nn + v * n + u] = s;
  }
  __syncthreads();
}

__device__ void CoopTsDct(int n, int nb, const float* bm, const float* in,
                          float* tmp, float* out) {
  const int nn = n * n;
  for (int i = threadIdx.x; i < nb * nn; i += blockDim.x) {
    const int b = i / nn, r = i % nn, k = r / n, y = r % n;
    const float* src = in + b * nn + y * n;
    float s = 0.f;
    for (int x = 0; x < n; ++x) s += bm[k * n + x] * src[x];
    tmp[b * nn + k * n + y] = s;
  }
  __syncthreads();
  const float scale = 1.0f / float(nn);
  for (int i = threadIdx.x; i < nb * nn; i += blockDim.x) {
    const int b = i / nn, r = i % nn, k = r / n, l = r % n;
    const float* t = tmp + b * nn + k * n;
    float s = 0.f;
    for (int y = 0; y < n; ++y) s += t[y] * bm[l * n + y];
    out[b * nn + k * n + l] = s * scale;
  }
  __syncthreads();
}

// The same two transforms with the matrix given transposed (aT[l n + v] =
// A[v][l], bT[x n + k] = B[k][x]) and the first DCT pass mapped with k
// fastest: consecutive threads then read consecutive shared-memory words of
// the matrix (the plain forms read it with a stride of n words, an n-way
// bank conflict at n = 32). Every output is the same sum of the same
// products in the same order, so the results are bit-identical.
__device__ void CoopTsIdctT(int n, int nb, const float* aT, const float* in,
                            float* tmp, float* out) {
  const int nn = n * n;
  for (int i = threadIdx.x; i < nb * nn; i += blockDim.x) {
    const int b = i / nn, r = i % nn, k = r / n, v = r % n;
    const float* src = in + b * nn + k * n;
    float s = 0.f;
    for (int l = 0; l < n; ++l) s += src[l] * aT[l * n + v];
    tmp[b * nn + k * n + v] = s;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nb * nn; i += blockDim.x) {
    const int b = i / nn, r = i % nn, v = r / n, u = r % n;
    const float* t = tmp + b * nn;
    float s = 0.f;
    for (int k = 0; k < n; ++k) s += aT[k * n + u] * t[k * n + v];
    out[b * nn + v * n + u] = s;
  }
  __syncthreads();
}

__device__ void CoopTsDctT(int n, int nb, const float* bT, const float* in,
                           float* tmp, float* out) {
  const int nn = n * n;
  for (int i = threadIdx.x; i < nb * nn; i += blockDim.x) {
    const int b = i / nn, r = i % nn, y = r / n, k = r % n;
    const float* src = in + b * nn + y * n;
    float s = 0.f;
    for (int x = 0; x < n; ++x) s += bT[x * n + k] * src[x];
    tmp[b * nn + k * n + y] = s;
  }
  __syncthreads();
  const float scale = 1.0f / float(nn);
  for (int i = threadIdx.x; i < nb * nn; i += blockDim.x) {
    const int b = i / nn, r = i % nn, k = r / n, l = r % n;
    const float* t = tmp + b * nn + k * n;
    float s = 0.f;
    for (int y = 0; y < n; ++y) s += t[y] * bT[y * n + l];
    out[b * nn + k * n + l] = s * scale;
  }
  __syncthreads();
}

// Upsampled-blurred HF prediction pixel (UpSample4x4BlurDCT,
// pik/ac_predictions.cc:263-374) at group-local pixel (X, Y).
__device__ __forceinline__ float Upsample(const float* pred, int X, int Y) {
  const int r = Y >> 2, q = X >> 2, ix = X & 3, iy = Y & 3;
  float bx[3];
  for (int j = 0; j < 3; ++j) {
    const float* row = pred + (r + j + 1) * kG2;
    const float v0 = row[q + 1], v1 = row[q + 2], v2 = row[q + 3];
    bx[j] = v0 * c_t.ub4[0][ix] + v1 * c_t.ub4[1][ix] + v2 * c_t.ub4[2][ix];
  }
  return bx[0] * c_t.ub4[0][iy] + bx[1] * c_t.ub4[1][iy] +
         bx[2] * c_t.ub4[2][iy];
}

// Upsample for the N pixels X0 .. X0 + N - 1 of row Y (X0 a multiple of 4):
// the same arithmetic as Upsample, with the 3 x (N / 4 + 2) source values
// loaded once.
template <int N>
__device__ __forceinline__ void UpsampleRow(const float* pred, int X0, int Y,
                                            float* out) {
  const int r = Y >> 2, q0 = X0 >> 2, iy = Y & 3;
  constexpr int W = N / 4 + 2;
  float src[3][W];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const float* row = pred + (r + j + 1) * kG2 + q0 + 1;
#pragma unroll
    for (int i = 0; i < W; ++i) src[j][i] = row[i];
  }
#pragma unroll
  for (int x = 0; x < N; ++x) {
    const int q = x >> 2, ix = x & 3;
    float bx[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      bx[j] = src[j][q] * c_t.ub4[0][ix] + src[j][q + 1] * c_t.ub4[1][ix] +
              src[j][q + 2] * c_t.ub4[2][ix];
    }
    out[x] = bx[0] * c_t.ub4[0][iy] + bx[1] * c_t.ub4[1][iy] +
             bx[2] * c_t.ub4[2][iy];
  }
}

// Square DCT blocks (DCT8, DCT_NOHF, DCT16, DCT32): HF prediction (if the
// type predicts HF) + AddBlockExceptLFAndLLFTo + InverseIntegralTransform
// (pik/compressed_image.cc:869-934). One CTA handles `nb` blocks of n x n.
template <int N>
__global__ void __launch_bounds__(256)
    k_square_idct(Geo g, DevFrame f, const uint32_t* list, int count,
                  int predict_hf) {
  PdlLaunchDependents();
  PdlTail pdl_tail;
  constexpr int NN = N * N;
  constexpr int NB = NN >= 256 ? 1 : 256 / NN;
  __shared__ float s_a[NN], s_b[NN];
  __shared__ float s_c[NB * NN], s_t[NB * NN], s_p[NB * NN];
  for (int i = threadIdx.x; i < NN; i += blockDim.x) {  // transposed
    s_a[i] = c_t.idct[MatOffset(N) + (i % N) * N + i / N];
    s_b[i] = c_t.dct[MatOffset(N) + (i % N) * N + i / N];
  }
  const int first = blockIdx.x * NB;
  const int nb = min(NB, count - first);
  constexpr int cov = N / 8, chunk = 64 * cov;
  const size_t plane_ac = size_t(g.ac_stride) * g.By;
  const size_t plane_px = size_t(g.PW) * g.PH;
  __syncthreads();
  for (int c = 0; c < 3; ++c) {
    // Load coefficients and, if predicting HF, the upsampled pixels.
    for (int i = threadIdx.x; i < nb * NN; i += blockDim.x) {
      const int b = i / NN, e = i % NN;
      const uint32_t pk = list[first + b];
      const int bx = pk & 0xFFFF, by = pk >> 16;
      const float* base = f.ac + c * plane_ac + size_t(by) * g.ac_stride +
                          size_t(bx) * 64;
      s_c[i] = base[(e / chunk) * size_t(g.ac_stride) + e % chunk];
      // DCT_NOHF shares this kernel with DCT but takes no HF prediction.
      if (predict_hf && !PredictHFOf(f.acs[by * g.Bx + bx] >> 4)) {
        s_p[i] = 0.f;
      } else if (predict_hf) {
        const int gi = (by >> 6) * g.Gx + (bx >> 6);
        const float* pred = f.pred2x2_g + gi * kG2GroupFloats + c * kG2 * kG2;
        const int X = (bx & 63) * 8 + e % N, Y = (by & 63) * 8 + e / N;
        s_p[i] = Upsample(pred, X, Y);
      }
    }
    __syncthreads();
    if (predict_hf) {
      CoopTsDctT(N, nb, s_b, s_p, s_t, s_p);
      for (int i = threadIdx.x; i < nb * NN; i += blockDim.x) {
        const int e = i % NN, y = e / N, x = e % N;
        if (y < 2 * cov && x < 2 * cov) continue;
        const uint32_t pk = list[first + i / NN];
        if (!PredictHFOf(f.acs[(pk >> 16) * g.Bx + (pk & 0xFFFF)] >> 4)) {
          continue;
        }
        s_c[i] += s_p[i];
      }
      __syncthreads();
    }
    CoopTsIdctT(N, nb, s_a, s_c, s_t, s_p);
    for (int i = threadIdx.x; i < nb * NN; i += blockDim.x) {
      const int b = i / NN, e = i % NN;
      const uint32_t pk = list[first + b];
      const int bx = pk & 0xFFFF, by = pk >> 16;
      f.idct[c * plane_px + size_t(by * 8 + e / N) * g.PW + bx * 8 + e % N] =
          s_p[i];
    }
    __syncthreads();
  }
}

// DCT4X4 (and _NOHF): four 4x4 transforms with interleaved coefficients
// (AcStrategy::TransformFromPixels/ToPixels, pik/ac_strategy.cc:604-629,
// 762-790), with the HF prediction (UpSample4x4BlurDCT,
// pik/ac_predictions.cc:263-374). A unit of 8 lanes takes one block and
// channel; lane j = 4 sy + k holds row sy + 2 k of the block's 64
// coefficients, which is row k of the coefficient matrices of sub-blocks
// (sy, 0) and (sy, 1) (columns sx + 2 l), and in the pixel domain pixel
// row 4 sy + k. The 4x4 transforms' second passes need the other rows of a
// sub-block: they go through a small shared-memory transpose per unit.
// Every sum has the operation order of TsIdct / TsDct (CoopTsIdct,
// CoopTsDct), so the result is bit-identical to the CTA-wide form.
constexpr int kDct4Threads = 128;
__global__ void __launch_bounds__(kDct4Threads)
    k_dct4_idct(Geo g, DevFrame f, const uint32_t* list, int count,
                int predict_hf) {
  PdlLaunchDependents();
  PdlTail pdl_tail;
  constexpr int kUnits = kDct4Threads / 8;
  __shared__ float s_t[kUnits][2][2][4][5];  // per unit: [sy][sx][row][col]
  const int unit = threadIdx.x >> 3, j = threadIdx.x & 7;
  const int sy = j >> 2, k = j & 3;
  const int item = blockIdx.x * kUnits + unit;
  const bool active = item < 3 * count;
  const int b = active ? item / 3 : 0, c = active ? item % 3 : 0;
  const uint32_t mask = 0xFFu << (threadIdx.x & 24);  // the unit's lanes
  const uint32_t pk = list[b];
  const int bx = pk & 0xFFFF, by = pk >> 16;
  const float* A = IdctMat(4);
  const float* B = DctMat(4);
  float (*t)[4][5] = s_t[unit][sy];
  // Coefficient row sy + 2 k: C_{sy,sx}[k][l] = cr[sx + 2 l].
  const float* crow = f.ac + c * size_t(g.ac_stride) * g.By +
                      size_t(by) * g.ac_stride + bx * 64 + (sy + 2 * k) * 8;
  float cr[8];
  {
    const float4 v0 = *reinterpret_cast<const float4*>(crow);
    const float4 v1 = *reinterpret_cast<const float4*>(crow + 4);
    cr[0] = v0.x, cr[1] = v0.y, cr[2] = v0.z, cr[3] = v0.w;
    cr[4] = v1.x, cr[5] = v1.y, cr[6] = v1.z, cr[7] = v1.w;
  }
  if (predict_hf && PredictHFOf(f.acs[by * g.Bx + bx] >> 4)) {
    // Prediction pixel row y = k of sub-blocks (sy, 0..1).
    const int gi = (by >> 6) * g.Gx + (bx >> 6);
    const float* pred = f.pred2x2_g + gi * kG2GroupFloats + c * kG2 * kG2;
    float P[8];
    UpsampleRow<8>(pred, (bx & 63) * 8, (by & 63) * 8 + 4 * sy + k, P);
    // TsDct pass 1: tmp[kk][y = k] = sum_x B[kk][x] P[y][x], to the tile.
#pragma unroll
    for (int sx = 0; sx < 2; ++sx) {
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        float sum = 0.f;
#pragma unroll
        for (int x = 0; x < 4; ++x) sum += B[kk * 4 + x] * P[4 * sx + x];
        t[sx][kk][k] = sum;
      }
    }
    __syncwarp(mask);
    // Pass 2: out[kk = k][l] = (sum_y tmp[k][y] B[l][y]) / 16, added to
    // coefficient (k, l) except the sub-blocks' DCs (positions 0, 1, 8, 9).
#pragma unroll
    for (int sx = 0; sx < 2; ++sx) {
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        float sum = 0.f;
#pragma unroll
        for (int y = 0; y < 4; ++y) sum += t[sx][k][y] * B[l * 4 + y];
        const float q = sum * (1.0f / 16.0f);
        if (k != 0 || l != 0) cr[sx + 2 * l] += q;
      }
    }
    __syncwarp(mask);
  }
  // The sub-blocks' DCs: the 2x2 Hadamard of positions 0, 1, 8, 9 (rows 0
  // and 1, held by lanes 0 and 4 of the unit).
  {
    const int base = threadIdx.x & 24;
    const float b00 = __shfl_sync(mask, cr[0], base);
    const float b01 = __shfl_sync(mask, cr[1], base);
    const float b10 = __shfl_sync(mask, cr[0], base + 4);
    const float b11 = __shfl_sync(mask, cr[1], base + 4);
    if (k == 0) {
      const float d[4] = {b00 + b01 + b10 + b11, b00 + b01 - b10 - b11,
                          b00 - b01 + b10 - b11, b00 - b01 - b10 + b11};
      cr[0] = d[sy * 2];
      cr[1] = d[sy * 2 + 1];
    }
  }
  // TsIdct pass 1: tmp[k][v] = sum_l C[k][l] A[v][l], to the tile.
#pragma unroll
  for (int sx = 0; sx < 2; ++sx) {
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      float sum = 0.f;
#pragma unroll
      for (int l = 0; l < 4; ++l) sum += cr[sx + 2 * l] * A[v * 4 + l];
      t[sx][k][v] = sum;
    }
  }
  __syncwarp(mask);
  // Pass 2: pixel row v = k: out[v][u] = sum_k A[u][k] tmp[k][v].
  float px[8];
#pragma unroll
  for (int sx = 0; sx < 2; ++sx) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      float sum = 0.f;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) sum += A[u * 4 + kk] * t[sx][kk][k];
      px[4 * sx + u] = sum;
    }
  }
  if (active) {
    float* out = f.idct + c * size_t(g.PW) * g.PH +
                 size_t(by * 8 + 4 * sy + k) * g.PW + bx * 8;
    *reinterpret_cast<float4*>(out) = make_float4(px[0], px[1], px[2], px[3]);
    *reinterpret_cast<float4*>(out + 4) =
        make_float4(px[4], px[5], px[6], px[7]);
  }
}

// DCT2X2, IDENTITY and LINES: inverse transforms only (no HF prediction),
// one thread per block and channel.
__device__ void SmallInverse(int type, const float* cb, float* px, int ps) {
  if (type == kDCT2X2) {
    float co[64];
    for (int i = 0; i < 64; ++i) co[i] = cb[i];
    for (int s = 2; s <= 8; s *= 2) {  // IDCT2TopBlock<2>, <4>, <8>
      float tmp[64];
      const int h = s / 2;
      for (int y = 0; y < h; ++y) {
        for (int x = 0; x < h; ++x) {
          const float c00 = co[y * 8 + x], c01 = co[y * 8 + h + x];
          const float c10 = co[(y + h) * 8 + x], c11 = co[(y + h) * 8 + h + x];
          tmp[y * 2 * 8 + x * 2] = c00 + c01 + c10 + c11;
          tmp[y * 2 * 8 + x * 2 + 1] = c00 + c01 - c10 - c11;
          tmp[(y * 2 + 1) * 8 + x * 2] = c00 - c01 + c10 - c11;
          tmp[(y * 2 + 1) * 8 + x * 2 + 1] = c00 - c01 - c10 + c11;
        }
      }
      for (int y = 0; y < s; ++y)
        for (int x = 0; x < s; ++x) co[y * 8 + x] = tmp[y * 8 + x];
    }
    for (int y = 0; y < 8; ++y)
      for (int x = 0; x < 8; ++x) px[y * ps + x] = co[y * 8 + x];
  } else if (type == kIDENTITY) {
    const float b00 = cb[0], b01 = cb[1], b10 = cb[8], b11 = cb[9];
    const float dcs[4] = {b00 + b01 + b10 + b11, b00 + b01 - b10 - b11,
                          b00 - b01 + b10 - b11, b00 - b01 - b10 + b11};
    for (int y = 0; y < 2; ++y) {
      for (int x = 0; x < 2; ++x) {
        float residual_sum = 0.f;
        for (int iy = 0; iy < 4; ++iy)
          for (int ix = 0; ix < 4; ++ix)
            if (ix != 0 || iy != 0)
              residual_sum += cb[(y + iy * 2) * 8 + x + ix * 2];
        const float ctr = dcs[y * 2 + x] - residual_sum * (1.0f / 16);
        for (int iy = 0; iy < 4; ++iy)
          for (int ix = 0; ix < 4; ++ix)
            if (ix != 1 || iy != 1)
              px[(y * 4 + iy) * ps + x * 4 + ix] =
                  cb[(y + iy * 2) * 8 + x + ix * 2] + ctr;
        px[(y * 4 + 1) * ps + x * 4 + 1] = ctr;
        px[y * 4 * ps + x * 4] = cb[(y + 2) * 8 + x + 2] + ctr;
      }
    }
  } else {  // LINES (pik/ac_strategy.cc:680-724)
    const int8_t kP3[4][3] = {{6, 7, 15}, {5, 14, 23}, {40, 49, 58},
                              {48, 56, 57}};
    const int8_t kP4[4][4] = {{4, 13, 22, 31}, {3, 12, 30, 39},
                              {24, 33, 51, 60}, {32, 41, 50, 59}};
    const int8_t kP6[4][6] = {{2, 11, 20, 29, 38, 47},
                              {1, 10, 19, 37, 46, 55},
                              {8, 17, 26, 44, 53, 62},
                              {16, 25, 34, 43, 52, 61}};
    const int8_t kP8[8] = {0, 9, 18, 27, 36, 45, 54, 63};
    const int8_t kC4[4][4] = {{4, 13, 22, 31}, {3, 12, 21, 30},
                              {24, 33, 42, 51}, {32, 41, 50, 59}};
    const int8_t kC6[4][6] = {{2, 11, 20, 29, 38, 47},
                              {10, 19, 28, 37, 46, 55},
                              {17, 26, 35, 44, 53, 62},
                              {16, 25, 34, 43, 52, 61}};
    const int8_t kC8[8] = {18, 27, 36, 45, 54, 39, 60, 63};
    const int8_t kDc00[21] = {0,  8,  9,  16, 17, 18, 25, 26, 27, 34, 35,
                              36, 43, 44, 45, 52, 53, 54, 61, 62, 63};
    const int8_t kDc01[15] = {24, 32, 33, 40, 41, 42, 48, 49,
                              50, 51, 56, 57, 58, 59, 60};
    const int8_t kDc10[15] = {3,  4,  5,  6,  7,  12, 13, 14,
                              15, 21, 22, 23, 30, 31, 39};
    const int8_t kDc11[13] = {1, 2, 10, 11, 19, 20, 28, 29, 37, 38, 46, 47, 55};
    auto cm = [](int i) { return (i & 7) * 8 + (i >> 3); };
    float temp[64];
    for (int i = 0; i < 64; ++i) temp[i] = 0.f;
    auto idcts = [&](int n, const int8_t* ip, const int8_t* ic) {
      float v[8];
      for (int j = 0; j < n; ++j) v[j] = cb[cm(ic[j])];
      for (int j = 0; j < n; ++j) {
        float s = 0.f;
        for (int k = 0; k < n; ++k) s += c_t.lines_inv[n][j][k] * v[k];
        temp[cm(ip[j])] = s;
      }
    };
    for (int i = 0; i < 4; ++i) idcts(3, kP3[i], kP3[i]);
    for (int i = 0; i < 4; ++i) idcts(4, kP4[i], kC4[i]);
    for (int i = 0; i < 4; ++i) idcts(6, kP6[i], kC6[i]);
    idcts(8, kP8, kC8);
    const float i0 = cb[0], i1 = cb[8], i2 = cb[1], i3 = cb[9];
    const float d00 = i0 + i1 + i2 + i3, d01 = i0 - i1 + i2 - i3;
    const float d10 = i0 + i1 - i2 - i3, d11 = i0 - i1 - i2 + i3;
    for (int v : kDc00) temp[cm(v)] += d00;
    for (int v : kDc01) temp[cm(v)] += d01;
    for (int v : kDc10) temp[cm(v)] += d10;
    for (int v : kDc11) temp[cm(v)] += d11;
    temp[21] = (temp[12] + temp[30]) * 0.5f;
    temp[28] = (temp[19] + temp[37]) * 0.5f;
    temp[35] = (temp[26] + temp[44]) * 0.5f;
    temp[42] = (temp[33] + temp[51]) * 0.5f;
    for (int y = 0; y < 8; ++y)
      for (int x = 0; x < 8; ++x) px[y * ps + x] = temp[y * 8 + x];
  }
}

// The LINES transform's index lists (pik/ac_strategy.cc:680-724) per
// element, for its coefficient-parallel forms: the line groups (3, 4, 6 and
// 8 points) with their pixel and coefficient positions, and the four DC
// regions. Positions are those of the row-major 8x8 arrays (the transposed
// index of the lists). Every pixel position lies in at most one line group
// (all but 21, 28, 35, 42) and in exactly one DC region; every coefficient
// position in one line group, except the DCs 0, 1, 8, 9.
struct LinesMap {
  int8_t n[13];       // points of each line group
  int8_t ip[13][8];   // its pixel positions
  int8_t ic[13][8];   // its coefficient positions
  int8_t grp[64];     // pixel position -> line group, -1: none
  int8_t j[64];       // ... and its index in the group
  int8_t cgrp[64];    // coefficient position -> line group, -1: a DC
  int8_t ck[64];      // ... and its index in the group
  int8_t dc_of[64];   // pixel position -> DC region
  int8_t dc_num[4];   // pixels per DC region
  int8_t dc_pos[4][21];  // their positions, in the reference's order
};
constexpr LinesMap MakeLinesMap() {
  constexpr int8_t kIp[13][8] = {
      {6, 7, 15},         {5, 14, 23},         {40, 49, 58},
      {48, 56, 57},       {4, 13, 22, 31},     {3, 12, 30, 39},
      {24, 33, 51, 60},   {32, 41, 50, 59},    {2, 11, 20, 29, 38, 47},
      {1, 10, 19, 37, 46, 55},                 {8, 17, 26, 44, 53, 62},
      {16, 25, 34, 43, 52, 61},                {0, 9, 18, 27, 36, 45, 54, 63}};
  constexpr int8_t kIc[13][8] = {
      {6, 7, 15},         {5, 14, 23},         {40, 49, 58},
      {48, 56, 57},       {4, 13, 22, 31},     {3, 12, 21, 30},
      {24, 33, 42, 51},   {32, 41, 50, 59},    {2, 11, 20, 29, 38, 47},
      {10, 19, 28, 37, 46, 55},                {17, 26, 35, 44, 53, 62},
      {16, 25, 34, 43, 52, 61},                {18, 27, 36, 45, 54, 39, 60, 63}};
  constexpr int8_t kN[13] = {3, 3, 3, 3, 4, 4, 4, 4, 6, 6, 6, 6, 8};
  constexpr int8_t kDc[4][21] = {
      {0, 8, 9, 16, 17, 18, 25, 26, 27, 34, 35, 36, 43, 44, 45, 52, 53, 54,
       61, 62, 63},
      {24, 32, 33, 40, 41, 42, 48, 49, 50, 51, 56, 57, 58, 59, 60},
      {3, 4, 5, 6, 7, 12, 13, 14, 15, 21, 22, 23, 30, 31, 39},
      {1, 2, 10, 11, 19, 20, 28, 29, 37, 38, 46, 47, 55}};
  constexpr int8_t kDcN[4] = {21, 15, 15, 13};
  LinesMap m{};
  for (int i = 0; i < 64; ++i) m.grp[i] = m.cgrp[i] = -1;
  for (int gi = 0; gi < 13; ++gi) {
    m.n[gi] = kN[gi];
    for (int k = 0; k < kN[gi]; ++k) {
      const int p = (kIp[gi][k] & 7) * 8 + (kIp[gi][k] >> 3);
      const int q = (kIc[gi][k] & 7) * 8 + (kIc[gi][k] >> 3);
      m.ip[gi][k] = int8_t(p);
      m.ic[gi][k] = int8_t(q);
      m.grp[p] = int8_t(gi), m.j[p] = int8_t(k);
      m.cgrp[q] = int8_t(gi), m.ck[q] = int8_t(k);
    }
  }
  for (int r = 0; r < 4; ++r) {
    m.dc_num[r] = kDcN[r];
    for (int i = 0; i < kDcN[r]; ++i) {
      const int p = (kDc[r][i] & 7) * 8 + (kDc[r][i] >> 3);
      m.dc_pos[r][i] = int8_t(p);
      m.dc_of[p] = int8_t(r);
    }
  }
  return m;
}
__constant__ LinesMap c_lines = MakeLinesMap();

// Coefficient-parallel forms of the small transforms for a CTA of 192
// threads that holds one block: thread (c, e) = (tid / 64, tid % 64) owns
// element e (row-major) of channel c. Each step reads shared memory, meets
// a barrier and writes, so every thread's arithmetic is the serial form's
// (SmallInverse, SmallForward) for that element, in the same order. The
// type is uniform in the CTA, so every thread meets every barrier.
constexpr int kSmallCtaThreads = 192;

// In: coefficients in `co`; out: pixels in `px`. `co` is overwritten.
__device__ void SmallInversePar(int type, int c, int e, float (*co)[64],
                                float (*px)[64], float (*aux)[4]) {
  const int Y = e >> 3, X = e & 7;
  if (type == kDCT2X2) {
    for (int s = 2; s <= 8; s *= 2) {  // IDCT2TopBlock<2>, <4>, <8>
      const int h = s / 2;
      const bool act = Y < s && X < s;
      float v = 0.f;
      if (act) {
        const int y = Y >> 1, x = X >> 1;
        const float c00 = co[c][y * 8 + x], c01 = co[c][y * 8 + h + x];
        const float c10 = co[c][(y + h) * 8 + x];
        const float c11 = co[c][(y + h) * 8 + h + x];
        v = (Y & 1) == 0 ? ((X & 1) == 0 ? c00 + c01 + c10 + c11
                                         : c00 + c01 - c10 - c11)
                         : ((X & 1) == 0 ? c00 - c01 + c10 - c11
                                         : c00 - c01 - c10 + c11);
      }
      __syncthreads();
      if (act) co[c][e] = v;
      __syncthreads();
    }
    px[c][e] = co[c][e];
  } else if (type == kIDENTITY) {
    if (e < 4) {  // the centre of sub-block (y, x) = (e / 2, e % 2)
      const int y = e >> 1, x = e & 1;
      const float* cb = co[c];
      const float b00 = cb[0], b01 = cb[1], b10 = cb[8], b11 = cb[9];
      const float dc = e == 0   ? b00 + b01 + b10 + b11
                       : e == 1 ? b00 + b01 - b10 - b11
                       : e == 2 ? b00 - b01 + b10 - b11
                                : b00 - b01 - b10 + b11;
      float residual_sum = 0.f;
      for (int iy = 0; iy < 4; ++iy)
        for (int ix = 0; ix < 4; ++ix)
          if (ix != 0 || iy != 0)
            residual_sum += cb[(y + iy * 2) * 8 + x + ix * 2];
      aux[c][e] = dc - residual_sum * (1.0f / 16);
    }
    __syncthreads();
    const int y = Y >> 2, iy = Y & 3, x = X >> 2, ix = X & 3;
    const float ctr = aux[c][y * 2 + x];
    float v;
    if (iy == 1 && ix == 1) {
      v = ctr;
    } else if (iy == 0 && ix == 0) {
      v = co[c][(y + 2) * 8 + x + 2] + ctr;
    } else {
      v = co[c][(y + iy * 2) * 8 + x + ix * 2] + ctr;
    }
    px[c][e] = v;
  } else {  // LINES
    const float* cb = co[c];
    float v = 0.f;
    const int gi = c_lines.grp[e];
    if (gi >= 0) {  // the line IDCT's output at this pixel
      const int n = c_lines.n[gi], jj = c_lines.j[e];
      float sum = 0.f;
      for (int k = 0; k < n; ++k) {
        sum += c_t.lines_inv[n][jj][k] * cb[c_lines.ic[gi][k]];
      }
      v = sum;
    }
    const float i0 = cb[0], i1 = cb[8], i2 = cb[1], i3 = cb[9];
    const int r = c_lines.dc_of[e];
    const float d = r == 0   ? i0 + i1 + i2 + i3
                    : r == 1 ? i0 - i1 + i2 - i3
                    : r == 2 ? i0 + i1 - i2 - i3
                             : i0 - i1 - i2 + i3;
    px[c][e] = v + d;
    __syncthreads();
    // The four pixels no line covers: the mean of their vertical neighbours.
    if (e == 21 || e == 28 || e == 35 || e == 42) {
      px[c][e] = (px[c][e - 9] + px[c][e + 9]) * 0.5f;
    }
  }
  __syncthreads();
}

// In: pixels in `px`; out: coefficients in `co`.
__device__ void SmallForwardPar(int type, int c, int e, float (*px)[64],
                                float (*co)[64], float (*aux)[4]) {
  const int Y = e >> 3, X = e & 7;
  if (type == kDCT2X2) {
    co[c][e] = px[c][e];
    __syncthreads();
    for (int s = 8; s >= 2; s /= 2) {  // DCT2TopBlock<8>, <4>, <2>
      const int h = s / 2;
      const bool act = Y < s && X < s;
      float v = 0.f;
      if (act) {
        const int qy = Y >= h, qx = X >= h;
        const int y = Y - qy * h, x = X - qx * h;
        const float c00 = co[c][y * 2 * 8 + x * 2];
        const float c01 = co[c][y * 2 * 8 + x * 2 + 1];
        const float c10 = co[c][(y * 2 + 1) * 8 + x * 2];
        const float c11 = co[c][(y * 2 + 1) * 8 + x * 2 + 1];
        v = qy == 0 ? (qx == 0 ? (c00 + c01 + c10 + c11) * 0.25f
                               : (c00 + c01 - c10 - c11) * 0.25f)
                    : (qx == 0 ? (c00 - c01 + c10 - c11) * 0.25f
                               : (c00 - c01 - c10 + c11) * 0.25f);
      }
      __syncthreads();
      if (act) co[c][e] = v;
      __syncthreads();
    }
  } else if (type == kIDENTITY) {
    // Coefficient e = (y + 2 iy, x + 2 ix) of sub-block (y, x).
    const int y = Y & 1, iy = Y >> 1, x = X & 1, ix = X >> 1;
    const float* p = px[c];
    if (iy == 0 && ix == 0) {  // the sub-block's DC
      float block_dc = 0.f;
      for (int jy = 0; jy < 4; ++jy)
        for (int jx = 0; jx < 4; ++jx)
          block_dc += p[(y * 4 + jy) * 8 + x * 4 + jx];
      block_dc *= 1.0f / 16;
      aux[c][y * 2 + x] = block_dc;
    } else {
      const float ctr = p[(y * 4 + 1) * 8 + x * 4 + 1];
      co[c][e] = iy == 1 && ix == 1 ? p[(y * 4) * 8 + x * 4] - ctr
                                    : p[(y * 4 + iy) * 8 + x * 4 + ix] - ctr;
    }
    __syncthreads();
    if (iy == 0 && ix == 0) {  // the 2x2 Hadamard of the DCs, x 0.25
      const float b00 = aux[c][0], b01 = aux[c][1];
      const float b10 = aux[c][2], b11 = aux[c][3];
      co[c][e] = y == 0 ? (x == 0 ? (b00 + b01 + b10 + b11) * 0.25f
                                  : (b00 + b01 - b10 - b11) * 0.25f)
                        : (x == 0 ? (b00 - b01 + b10 - b11) * 0.25f
                                  : (b00 - b01 - b10 + b11) * 0.25f);
    }
  } else {  // LINES
    if (e < 4) {  // the mean of DC region e
      float dc = 0.f;
      for (int i = 0; i < c_lines.dc_num[e]; ++i) {
        dc += px[c][c_lines.dc_pos[e][i]];
      }
      dc /= float(c_lines.dc_num[e]);
      aux[c][e] = dc;
    }
    __syncthreads();
    px[c][e] -= aux[c][c_lines.dc_of[e]];
    __syncthreads();
    const int gi = c_lines.cgrp[e];
    float v;
    if (gi >= 0) {  // the line DCT's output at this coefficient
      const int n = c_lines.n[gi], kk = c_lines.ck[e];
      float sum = 0.f;
      for (int j = 0; j < n; ++j) {
        sum += c_t.lines_fwd[n][kk][j] * px[c][c_lines.ip[gi][j]];
      }
      v = sum;
    } else {  // positions 0, 1, 8, 9: the 2x2 Hadamard of the DC means
      const float d00 = aux[c][0], d01 = aux[c][1];
      const float d10 = aux[c][2], d11 = aux[c][3];
      v = e == 0   ? (d00 + d01 + d10 + d11) * 0.25f
          : e == 8 ? (d00 - d01 + d10 - d11) * 0.25f
          : e == 1 ? (d00 + d01 - d10 - d11) * 0.25f
                   : (d00 - d01 - d10 + d11) * 0.25f;
    }
    co[c][e] = v;
  }
  __syncthreads();
}

// DCT2X2, IDENTITY and LINES: inverse only (no HF prediction). Two forms:
// one CTA of 192 threads per block (k_small_idct_cta: short latency, for
// the few such blocks of most frames) and one thread per block and channel
// (k_small_idct: throughput, for frames with many).
__global__ void __launch_bounds__(kSmallCtaThreads)
    k_small_idct_cta(Geo g, DevFrame f, const uint32_t* list, int count) {
  PdlLaunchDependents();
  PdlTail pdl_tail;
  __shared__ float s_co[3][64], s_px[3][64];
  __shared__ float s_aux[3][4];
  const int c = threadIdx.x >> 6, e = threadIdx.x & 63;
  const uint32_t pk = list[blockIdx.x];
  const int bx = pk & 0xFFFF, by = pk >> 16;
  const int type = f.acs[by * g.Bx + bx] >> 4;
  s_co[c][e] = f.ac[c * size_t(g.ac_stride) * g.By +
                    size_t(by) * g.ac_stride + bx * 64 + e];
  __syncthreads();
  SmallInversePar(type, c, e, s_co, s_px, s_aux);
  f.idct[c * size_t(g.PW) * g.PH + size_t(by * 8 + (e >> 3)) * g.PW + bx * 8 +
         (e & 7)] = s_px[c][e];
}

// One thread per block and channel computes the serial inverse from shared
// memory; the warp stages its 32 items' coefficients and pixels with
// coalesced 16-byte accesses (the block list of this class is ordered by
// transform type, so a warp rarely holds more than one type).
constexpr int kSmallIdctThreads = 64;
__global__ void __launch_bounds__(kSmallIdctThreads)
    k_small_idct(Geo g, DevFrame f, const uint32_t* list, int count) {
  PdlLaunchDependents();
  PdlTail pdl_tail;
  __shared__ float s_in[kSmallIdctThreads][65];
  __shared__ float s_out[kSmallIdctThreads][65];
  const int lane = threadIdx.x & 31, w0 = threadIdx.x & ~31;
  const int base = blockIdx.x * kSmallIdctThreads + w0;  // the warp's items
  const int items = 3 * count;
  const size_t plane_ac = size_t(g.ac_stride) * g.By;
  const size_t plane_px = size_t(g.PW) * g.PH;
#pragma unroll 4
  for (int r = 0; r < 16; ++r) {  // two items of 16 float4 per step
    const int it = 2 * r + (lane >> 4), e = (lane & 15) * 4;
    const int item = base + it;
    if (item < items) {
      const int b = item / 3, c = item % 3;
      const uint32_t pk = list[b];
      const int bx = pk & 0xFFFF, by = pk >> 16;
      const float4 v = *reinterpret_cast<const float4*>(
          f.ac + c * plane_ac + size_t(by) * g.ac_stride + bx * 64 + e);
      float* d = s_in[w0 + it] + e;
      d[0] = v.x, d[1] = v.y, d[2] = v.z, d[3] = v.w;
    }
  }
  __syncwarp();
  if (base + lane < items) {
    const uint32_t pk = list[(base + lane) / 3];
    const int bx = pk & 0xFFFF, by = pk >> 16;
    SmallInverse(f.acs[by * g.Bx + bx] >> 4, s_in[w0 + lane],
                 s_out[w0 + lane], 8);
  }
  __syncwarp();
#pragma unroll 4
  for (int r = 0; r < 16; ++r) {  // two items of 8 rows x 2 float4 per step
    const int it = 2 * r + (lane >> 4), y = (lane >> 1) & 7, h = lane & 1;
    const int item = base + it;
    if (item < items) {
      const int b = item / 3, c = item % 3;
      const uint32_t pk = list[b];
      const int bx = pk & 0xFFFF, by = pk >> 16;
      const float* o = s_out[w0 + it] + y * 8 + 4 * h;
      *reinterpret_cast<float4*>(f.idct + c * plane_px +
                                 size_t(by * 8 + y) * g.PW + bx * 8 + 4 * h) =
          make_float4(o[0], o[1], o[2], o[3]);
    }
  }
}

// ---------------------------------------------------------------------------
// AdaptiveReconstruction's DCT-domain clamp (pik/adaptive_reconstruction.cc:
// 72-244, 334-471): per first block, DCT of (filtered - original) per
// channel, the clamp ratio of each coefficient to half a quantisation step
// (LLF: to the DC step), the minimum over the three channels, then the
// scaled correction is transformed back and added to the original.

struct ArBlockInfo {
  const float* dm[3];  // dequant matrix per channel
  float inv_quant_ac;
};

// Clamp tape entry of one coefficient: 0 = no channel's ratio below 1 (the
// correction is kept), 1..3 = channel code - 1 set the minimum ratio by
// clamping, 4 = the minimum was the 0 of a +0.0 correction (SymmetricClamp
// divides +0.0 by 1e-7). The adjoint follows these branches instead of
// recomputing them, so rounding cannot send it down another one.
__device__ __forceinline__ uint8_t ClampTapeCode(int arg, float co_arg) {
  if (arg < 0) return 0;
  return __float_as_uint(co_arg) == 0u ? 4 : uint8_t(arg + 1);
}

// Minimum ratio on the branch a clamp tape code names.
__device__ __forceinline__ float TapeRatio(int code, float r0, float r1,
                                           float r2) {
  return code == 0   ? 1.0f
         : code == 1 ? r0
         : code == 2 ? r1
         : code == 3 ? r2
                     : 0.0f;
}

// Offset in the frame coefficient layout of element e (row-major in the
// n x n block, n = 8 cov) of the block whose first cell is (bx, by).
__device__ __forceinline__ size_t CoefOffset(const Geo& g, int bx, int by,
                                             int cov, int e) {
  const int chunk = 64 * cov;
  return size_t(by + e / chunk) * g.ac_stride + size_t(bx) * 64 + e % chunk;
}

// inv_global_scale / qf of a block, times the optional per-cell clamp scale
// (pikgpu_frame_set_clamp_scale): the factor of every non-LLF clamp
// interval.
__device__ __forceinline__ float ClampInvQuantAc(const Geo& g,
                                                 const DevFrame& f,
                                                 float inv_global_scale,
                                                 int bx, int by, int qac) {
  const float iq = inv_global_scale / float(qac);
  return f.clamp_scale ? iq * f.clamp_scale[by * g.Bx + bx] : iq;
}

__device__ __forceinline__ ArBlockInfo ArInfo(const Geo& g, const DevFrame& f,
                                              const FrameScalars& s, int bx,
                                              int by, int type) {
  ArBlockInfo r;
  const int qac = f.qf[by * g.Bx + bx];
  r.inv_quant_ac = ClampInvQuantAc(g, f, s.inv_global_scale, bx, by, qac);
  const int cf = f.dq_cf[(by >> 3) * g.Tx + (bx >> 3)];
  const int table = f.dq_map[cf * 256 + (qac - 1)];
  const int kind = QuantKindOf(type);
  for (int c = 0; c < 3; ++c) {
    r.dm[c] = f.table + f.offsets[(table * 7 + kind) * 3 + c];
  }
  return r;
}

// SymmetricClamp's ratio for one coefficient (only +0.0 counts as zero).
__device__ __forceinline__ float ClampRatio(float corr, float interval) {
  const float upper = 0.5f * interval;
  const float lower = -0.5f * interval;
  const float mx = lower < corr ? corr : lower;
  const float clamped = mx < upper ? mx : upper;
  const float divisor = __float_as_uint(corr) == 0u ? 1E-7f : corr;
  return clamped / divisor;
}

__device__ __forceinline__ float LlfScale(int type, int x, int y) {
  if (type == kDCT16X16) return c_t.ar_llf16[y][x];
  if (type == kDCT32X32) return c_t.ar_llf32[y][x];
  return 1.0f;
}

// One CTA of 256 threads per DCT32 block (the rows form's one warp per
// block leaves most SMs idle at a few hundred blocks). `count` is read from
// device memory (the compacted list of k_active_blocks); the grid covers the
// class's whole list.
template <int N>
__global__ void __launch_bounds__(256)
    k_square_ar(Geo g, DevFrame f, FrameScalars s, const uint32_t* list,
                const int* count_ptr) {
  PdlLaunchDependents();
  PdlTail pdl_tail;
  constexpr int NN = N * N;
  constexpr int NB = NN >= 256 ? 1 : 256 / NN;
  constexpr int cov = N / 8;
  const int count = *count_ptr;
  if (int(blockIdx.x) * NB >= count) return;  // whole CTA
  __shared__ float s_a[NN], s_b[NN];
  __shared__ float s_blk[3][NB * NN];
  __shared__ float s_r[NB * NN], s_t[NB * NN], s_p[NB * NN];
  for (int i = threadIdx.x; i < NN; i += blockDim.x) {  // transposed
    s_a[i] = c_t.idct[MatOffset(N) + (i % N) * N + i / N];
    s_b[i] = c_t.dct[MatOffset(N) + (i % N) * N + i / N];
  }
  const int first = blockIdx.x * NB;
  const int nb = min(NB, count - first);
  const size_t plane = size_t(g.PW) * g.PH;
  __syncthreads();
  for (int c = 0; c < 3; ++c) {
    for (int i = threadIdx.x; i < nb * NN; i += blockDim.x) {
      const int b = i / NN, e = i % NN;
      const uint32_t pk = list[first + b];
      const int bx = pk & 0xFFFF, by = pk >> 16;
      const size_t o = c * plane + size_t(by * 8 + e / N) * g.PW + bx * 8 + e % N;
      s_p[i] = f.filt[o] - f.idct[o];
    }
    __syncthreads();
    CoopTsDctT(N, nb, s_b, s_p, s_t, s_blk[c]);
  }
  for (int i = threadIdx.x; i < nb * NN; i += blockDim.x) {
    const int b = i / NN, e = i % NN, y = e / N, x = e % N;
    const uint32_t pk = list[first + b];
    const int bx = pk & 0xFFFF, by = pk >> 16;
    const int type = f.acs[by * g.Bx + bx] >> 4;
    const ArBlockInfo info = ArInfo(g, f, s, bx, by, type);
    float mr = 1.0f, rt[3];
    int arg = -1;
    for (int c = 0; c < 3; ++c) {
      const float interval =
          (y < cov && x < cov)
              ? LlfScale(type, x, y) * s.mul_dc[c]
              : info.dm[c][e] * info.inv_quant_ac;
      rt[c] = ClampRatio(s_blk[c][i], interval);
      if (rt[c] < mr) mr = rt[c], arg = c;
    }
    if (f.clamp_tape || f.clamp_tape_in) {
      const size_t to = CoefOffset(g, bx, by, cov, e);
      uint8_t code = arg < 0 ? 0 : mr == 0.0f ? 4 : uint8_t(arg + 1);
      if (f.clamp_tape_in) {
        code = f.clamp_tape_in[to];
        mr = TapeRatio(code, rt[0], rt[1], rt[2]);
      }
      if (f.clamp_tape) f.clamp_tape[to] = code;
    }
    s_r[i] = mr;
  }
  __syncthreads();
  for (int c = 0; c < 3; ++c) {
    for (int i = threadIdx.x; i < nb * NN; i += blockDim.x) {
      s_blk[c][i] = s_blk[c][i] * s_r[i];
    }
    __syncthreads();
    CoopTsIdctT(N, nb, s_a, s_blk[c], s_t, s_p);
    for (int i = threadIdx.x; i < nb * NN; i += blockDim.x) {
      const int b = i / NN, e = i % NN;
      const uint32_t pk = list[first + b];
      const int bx = pk & 0xFFFF, by = pk >> 16;
      const size_t o = c * plane + size_t(by * 8 + e / N) * g.PW + bx * 8 + e % N;
      f.filt[o] = s_p[i] + f.idct[o];
    }
    __syncthreads();
  }
}

// Clamp for DCT4X4 blocks: one warp per block, lanes 8 c + j (c < 3) on
// channel c. Lane j = 4 sy + k of a channel holds pixel row 4 sy + k of the
// correction (filtered - original) and, after the forward 4x4 transforms,
// coefficient row sy + 2 k; the minimum ratio over the channels is read
// from the lanes j, j + 8, j + 16 of the other channels. The second pass
// of each 4x4 transform reads the other rows of its sub-block through a
// shared-memory transpose. Every sum has the operation order of TsDct /
// TsIdct (CoopTsDct, CoopTsIdct). Lanes 24..31 repeat channel 2 and store
// nothing.
constexpr int kDct4ArThreads = 128;
__global__ void __launch_bounds__(kDct4ArThreads)
    k_dct4_ar(Geo g, DevFrame f, FrameScalars s, const uint32_t* list,
              const int* count_ptr) {
  PdlLaunchDependents();
  PdlTail pdl_tail;
  constexpr int kWarps = kDct4ArThreads / 32;
  const int count = *count_ptr;
  if (int(blockIdx.x) * kWarps >= count) return;  // whole CTA
  __shared__ float s_t[kWarps][4][2][2][4][5];  // [warp][c][sy][sx][row][col]
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = min(lane >> 3, 2), j = lane & 7;
  const bool owner = lane < 24;
  const int sy = j >> 2, k = j & 3;
  const int b = blockIdx.x * kWarps + w;
  const bool active = b < count;
  const int base = c * 8;  // lane of the channel's coefficient row 0
  const uint32_t pk = list[active ? b : 0];
  const int bx = pk & 0xFFFF, by = pk >> 16;
  const float* A = IdctMat(4);
  const float* B = DctMat(4);
  float (*t)[4][5] = s_t[w][lane >> 3][sy];
  const size_t plane = size_t(g.PW) * g.PH;
  const size_t row = c * plane + size_t(by * 8 + 4 * sy + k) * g.PW + bx * 8;
  // The clamp intervals of the lane's 8 coefficients, loaded first (a chain
  // of dependent loads whose latency the forward transform then hides).
  float interval[8];
  {
    const int type = f.acs[by * g.Bx + bx] >> 4;
    const ArBlockInfo info = ArInfo(g, f, s, bx, by, type);
    const float* dm = c == 0 ? info.dm[0] : c == 1 ? info.dm[1] : info.dm[2];
#pragma unroll
    for (int col = 0; col < 8; ++col) {
      const int e = (sy + 2 * k) * 8 + col;
      interval[col] = e == 0 ? 1.0f * s.mul_dc[c] : dm[e] * info.inv_quant_ac;
    }
  }
  float co[8], iv[8], d[8];
  {
    const float4 f0 = *reinterpret_cast<const float4*>(f.filt + row);
    const float4 f1 = *reinterpret_cast<const float4*>(f.filt + row + 4);
    const float4 i0 = *reinterpret_cast<const float4*>(f.idct + row);
    const float4 i1 = *reinterpret_cast<const float4*>(f.idct + row + 4);
    iv[0] = i0.x, iv[1] = i0.y, iv[2] = i0.z, iv[3] = i0.w;
    iv[4] = i1.x, iv[5] = i1.y, iv[6] = i1.z, iv[7] = i1.w;
    d[0] = f0.x - i0.x, d[1] = f0.y - i0.y, d[2] = f0.z - i0.z;
    d[3] = f0.w - i0.w, d[4] = f1.x - i1.x, d[5] = f1.y - i1.y;
    d[6] = f1.z - i1.z, d[7] = f1.w - i1.w;
  }
  // TsDct pass 1 (pixel row y = k): tmp[kk][k] = sum_x B[kk][x] d[x].
#pragma unroll
  for (int sx = 0; sx < 2; ++sx)
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      float sum = 0.f;
#pragma unroll
      for (int x = 0; x < 4; ++x) sum += B[kk * 4 + x] * d[4 * sx + x];
      t[sx][kk][k] = sum;
    }
  __syncwarp();
  // Pass 2: coefficient (k, l) of sub-block (sy, sx), at column sx + 2 l of
  // coefficient row sy + 2 k.
#pragma unroll
  for (int sx = 0; sx < 2; ++sx)
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      float sum = 0.f;
#pragma unroll
      for (int y = 0; y < 4; ++y) sum += t[sx][k][y] * B[l * 4 + y];
      co[sx + 2 * l] = sum * (1.0f / 16.0f);
    }
  __syncwarp();
  // The 2x2 Hadamard of the sub-block DCs (positions 0, 1, 8, 9) x 0.25.
  {
    const float b00 = __shfl_sync(~0u, co[0], base);
    const float b01 = __shfl_sync(~0u, co[1], base);
    const float b10 = __shfl_sync(~0u, co[0], base + 4);
    const float b11 = __shfl_sync(~0u, co[1], base + 4);
    if (k == 0) {
      if (sy == 0) {
        co[0] = (b00 + b01 + b10 + b11) * 0.25f;
        co[1] = (b00 + b01 - b10 - b11) * 0.25f;
      } else {
        co[0] = (b00 - b01 + b10 - b11) * 0.25f;
        co[1] = (b00 - b01 - b10 + b11) * 0.25f;
      }
    }
  }
  // Clamp ratios, their minimum over X, Y, B, and the scaled corrections.
#pragma unroll
  for (int col = 0; col < 8; ++col) {
    const float r = ClampRatio(co[col], interval[col]);
    float rt[3], cv[3];
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) {
      rt[cc] = __shfl_sync(~0u, r, cc * 8 + j);
      cv[cc] = __shfl_sync(~0u, co[col], cc * 8 + j);
    }
    float mr = 1.0f;
    int arg = -1;
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) {
      if (rt[cc] < mr) mr = rt[cc], arg = cc;
    }
    const int e = (sy + 2 * k) * 8 + col;
    const size_t to = CoefOffset(g, bx, by, 1, e);
    const float ca = arg == 0 ? cv[0] : arg == 1 ? cv[1] : cv[2];
    uint8_t code = ClampTapeCode(arg, arg < 0 ? 0.f : ca);
    if (f.clamp_tape_in) {
      code = f.clamp_tape_in[to];
      mr = TapeRatio(code, rt[0], rt[1], rt[2]);
    }
    if (active && lane < 8 && f.clamp_tape) f.clamp_tape[to] = code;
    co[col] = co[col] * mr;
  }
  // Inverse: sub-block DCs from the Hadamard of 0, 1, 8, 9, then TsIdct;
  // the result is added to the original.
  {
    const float b00 = __shfl_sync(~0u, co[0], base);
    const float b01 = __shfl_sync(~0u, co[1], base);
    const float b10 = __shfl_sync(~0u, co[0], base + 4);
    const float b11 = __shfl_sync(~0u, co[1], base + 4);
    if (k == 0) {
      co[0] = sy == 0 ? b00 + b01 + b10 + b11 : b00 - b01 + b10 - b11;
      co[1] = sy == 0 ? b00 + b01 - b10 - b11 : b00 - b01 - b10 + b11;
    }
  }
#pragma unroll
  for (int sx = 0; sx < 2; ++sx)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      float sum = 0.f;
#pragma unroll
      for (int l = 0; l < 4; ++l) sum += co[sx + 2 * l] * A[v * 4 + l];
      t[sx][k][v] = sum;
    }
  __syncwarp();
  float px[8];
#pragma unroll
  for (int sx = 0; sx < 2; ++sx)
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      float sum = 0.f;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) sum += A[u * 4 + kk] * t[sx][kk][k];
      px[4 * sx + u] = sum + iv[4 * sx + u];
    }
  if (active && owner) {
    *reinterpret_cast<float4*>(f.filt + row) =
        make_float4(px[0], px[1], px[2], px[3]);
    *reinterpret_cast<float4*>(f.filt + row + 4) =
        make_float4(px[4], px[5], px[6], px[7]);
  }
}

// Forward transforms of DCT2X2, IDENTITY and LINES (pik/ac_strategy.cc:
// 531-603, 630-663), single thread.
__device__ void SmallForward(int type, const float* px, int ps, float* co) {
  if (type == kDCT2X2) {
    float cur[64];
    for (int y = 0; y < 8; ++y)
      for (int x = 0; x < 8; ++x) cur[y * 8 + x] = px[y * ps + x];
    for (int s = 8; s >= 2; s /= 2) {  // DCT2TopBlock<8>, <4>, <2>
      float tmp[64];
      const int h = s / 2;
      for (int y = 0; y < h; ++y) {
        for (int x = 0; x < h; ++x) {
          const float c00 = cur[y * 2 * 8 + x * 2];
          const float c01 = cur[y * 2 * 8 + x * 2 + 1];
          const float c10 = cur[(y * 2 + 1) * 8 + x * 2];
          const float c11 = cur[(y * 2 + 1) * 8 + x * 2 + 1];
          tmp[y * 8 + x] = (c00 + c01 + c10 + c11) * 0.25f;
          tmp[y * 8 + h + x] = (c00 + c01 - c10 - c11) * 0.25f;
          tmp[(y + h) * 8 + x] = (c00 - c01 + c10 - c11) * 0.25f;
          tmp[(y + h) * 8 + h + x] = (c00 - c01 - c10 + c11) * 0.25f;
        }
      }
      for (int y = 0; y < s; ++y)
        for (int x = 0; x < s; ++x) cur[y * 8 + x] = tmp[y * 8 + x];
    }
    for (int i = 0; i < 64; ++i) co[i] = cur[i];
  } else if (type == kIDENTITY) {
    for (int y = 0; y < 2; ++y) {
      for (int x = 0; x < 2; ++x) {
        float block_dc = 0.f;
        for (int iy = 0; iy < 4; ++iy)
          for (int ix = 0; ix < 4; ++ix)
            block_dc += px[(y * 4 + iy) * ps + x * 4 + ix];
        block_dc *= 1.0f / 16;
        const float ctr = px[(y * 4 + 1) * ps + x * 4 + 1];
        for (int iy = 0; iy < 4; ++iy)
          for (int ix = 0; ix < 4; ++ix)
            if (ix != 1 || iy != 1)
              co[(y + iy * 2) * 8 + x + ix * 2] =
                  px[(y * 4 + iy) * ps + x * 4 + ix] - ctr;
        co[(y + 2) * 8 + x + 2] = co[y * 8 + x];
        co[y * 8 + x] = block_dc;
      }
    }
    const float b00 = co[0], b01 = co[1], b10 = co[8], b11 = co[9];
    co[0] = (b00 + b01 + b10 + b11) * 0.25f;
    co[1] = (b00 + b01 - b10 - b11) * 0.25f;
    co[8] = (b00 - b01 + b10 - b11) * 0.25f;
    co[9] = (b00 - b01 - b10 + b11) * 0.25f;
  } else {  // LINES
    const int8_t kP3[4][3] = {{6, 7, 15}, {5, 14, 23}, {40, 49, 58},
                              {48, 56, 57}};
    const int8_t kP4[4][4] = {{4, 13, 22, 31}, {3, 12, 30, 39},
                              {24, 33, 51, 60}, {32, 41, 50, 59}};
    const int8_t kP6[4][6] = {{2, 11, 20, 29, 38, 47},
                              {1, 10, 19, 37, 46, 55},
                              {8, 17, 26, 44, 53, 62},
                              {16, 25, 34, 43, 52, 61}};
    const int8_t kP8[8] = {0, 9, 18, 27, 36, 45, 54, 63};
    const int8_t kC4[4][4] = {{4, 13, 22, 31}, {3, 12, 21, 30},
                              {24, 33, 42, 51}, {32, 41, 50, 59}};
    const int8_t kC6[4][6] = {{2, 11, 20, 29, 38, 47},
                              {10, 19, 28, 37, 46, 55},
                              {17, 26, 35, 44, 53, 62},
                              {16, 25, 34, 43, 52, 61}};
    const int8_t kC8[8] = {18, 27, 36, 45, 54, 39, 60, 63};
    const int8_t kDc00[21] = {0,  8,  9,  16, 17, 18, 25, 26, 27, 34, 35,
                              36, 43, 44, 45, 52, 53, 54, 61, 62, 63};
    const int8_t kDc01[15] = {24, 32, 33, 40, 41, 42, 48, 49,
                              50, 51, 56, 57, 58, 59, 60};
    const int8_t kDc10[15] = {3,  4,  5,  6,  7,  12, 13, 14,
                              15, 21, 22, 23, 30, 31, 39};
    const int8_t kDc11[13] = {1, 2, 10, 11, 19, 20, 28, 29, 37, 38, 46, 47, 55};
    auto cm = [](int i) { return (i & 7) * 8 + (i >> 3); };
    float temp[64];
    for (int y = 0; y < 8; ++y)
      for (int x = 0; x < 8; ++x) temp[y * 8 + x] = px[y * ps + x];
    for (int i = 0; i < 64; ++i) co[i] = 0.f;
    auto dc_part = [&](const int8_t* idx, int num) {
      float dc = 0.f;
      for (int i = 0; i < num; ++i) dc += temp[cm(idx[i])];
      dc /= float(num);
      for (int i = 0; i < num; ++i) temp[cm(idx[i])] -= dc;
      return dc;
    };
    const float d00 = dc_part(kDc00, 21), d01 = dc_part(kDc01, 15);
    const float d10 = dc_part(kDc10, 15), d11 = dc_part(kDc11, 13);
    co[0] = (d00 + d01 + d10 + d11) * 0.25f;
    co[8] = (d00 - d01 + d10 - d11) * 0.25f;
    co[1] = (d00 + d01 - d10 - d11) * 0.25f;
    co[9] = (d00 - d01 - d10 + d11) * 0.25f;
    auto dcts = [&](int n, const int8_t* ip, const int8_t* ic) {
      for (int k = 0; k < n; ++k) {
        float sum = 0.f;
        for (int j = 0; j < n; ++j) sum += c_t.lines_fwd[n][k][j] * temp[cm(ip[j])];
        co[cm(ic[k])] = sum;
      }
    };
    for (int i = 0; i < 4; ++i) dcts(3, kP3[i], kP3[i]);
    for (int i = 0; i < 4; ++i) dcts(4, kP4[i], kC4[i]);
    for (int i = 0; i < 4; ++i) dcts(6, kP6[i], kC6[i]);
    dcts(8, kP8, kC8);
  }
}

// Clamp for DCT2X2, IDENTITY and LINES blocks, in two forms like the
// inverse. k_small_ar_cta: one CTA of 192 threads per block, thread (c, e)
// on element e of channel c, with the transforms in their
// coefficient-parallel forms; the minimum ratio over X, Y, B (in that
// order, as the reference) is read across the channels' threads.
__global__ void __launch_bounds__(kSmallCtaThreads)
    k_small_ar_cta(Geo g, DevFrame f, FrameScalars s, const uint32_t* list,
                   const int* count_ptr) {
  PdlLaunchDependents();
  PdlTail pdl_tail;
  if (int(blockIdx.x) >= *count_ptr) return;  // whole CTA
  __shared__ float s_px[3][64], s_co[3][64], s_r[3][64];
  __shared__ float s_aux[3][4];
  const int c = threadIdx.x >> 6, e = threadIdx.x & 63;
  const uint32_t pk = list[blockIdx.x];
  const int bx = pk & 0xFFFF, by = pk >> 16;
  const int type = f.acs[by * g.Bx + bx] >> 4;
  const ArBlockInfo info = ArInfo(g, f, s, bx, by, type);
  const float* dm = c == 0 ? info.dm[0] : c == 1 ? info.dm[1] : info.dm[2];
  const float interval =
      e == 0 ? 1.0f * s.mul_dc[c] : dm[e] * info.inv_quant_ac;
  const size_t o = c * size_t(g.PW) * g.PH +
                   size_t(by * 8 + (e >> 3)) * g.PW + bx * 8 + (e & 7);
  const float iv = f.idct[o];
  s_px[c][e] = f.filt[o] - iv;
  __syncthreads();
  SmallForwardPar(type, c, e, s_px, s_co, s_aux);
  const float co = s_co[c][e];
  s_r[c][e] = ClampRatio(co, interval);
  __syncthreads();
  float mr = 1.0f;
  int arg = -1;
  for (int cc = 0; cc < 3; ++cc) {
    const float r = s_r[cc][e];
    if (r < mr) mr = r, arg = cc;
  }
  if (f.clamp_tape || f.clamp_tape_in) {
    const size_t to = CoefOffset(g, bx, by, 1, e);
    // The +0.0 case is the only one with a ratio of exactly 0.
    uint8_t code = arg < 0 ? 0 : mr == 0.0f ? 4 : uint8_t(arg + 1);
    if (f.clamp_tape_in) {
      code = f.clamp_tape_in[to];
      mr = TapeRatio(code, s_r[0][e], s_r[1][e], s_r[2][e]);
    }
    if (f.clamp_tape && c == 0) f.clamp_tape[to] = code;
  }
  s_co[c][e] = co * mr;
  __syncthreads();
  SmallInversePar(type, c, e, s_co, s_px, s_aux);
  f.filt[o] = s_px[c][e] + iv;
}

// k_small_ar: one thread per (block, channel); the warp of channel c of 32
// blocks computes its serial forward transform and clamp ratios, and the
// minimum over X, Y, B is taken through shared memory. (A form that stages
// the blocks through shared memory with coalesced loads measured slower:
// 0.083 against 0.056 ms of clamp on a 4096x4096 frame of small transforms.)
constexpr int kSmallArBlocks = 32;

__global__ void __launch_bounds__(3 * kSmallArBlocks)
    k_small_ar(Geo g, DevFrame f, FrameScalars s, const uint32_t* list,
               const int* count_ptr) {
  PdlLaunchDependents();
  PdlTail pdl_tail;
  __shared__ float s_ratio[3][kSmallArBlocks][65];
  const int count = *count_ptr;
  if (int(blockIdx.x) * kSmallArBlocks >= count) return;  // whole CTA
  const int c = threadIdx.x / kSmallArBlocks;
  const int lb = threadIdx.x % kSmallArBlocks;
  const int i = blockIdx.x * kSmallArBlocks + lb;
  const bool active = i < count;
  const size_t plane = size_t(g.PW) * g.PH;
  int type = 0;
  size_t o0 = 0;
  float blk[64];
  if (active) {
    const uint32_t pk = list[i];
    const int bx = pk & 0xFFFF, by = pk >> 16;
    type = f.acs[by * g.Bx + bx] >> 4;
    const ArBlockInfo info = ArInfo(g, f, s, bx, by, type);
    o0 = c * plane + size_t(by * 8) * g.PW + bx * 8;
    float diff[64];
    for (int y = 0; y < 8; ++y)
      for (int x = 0; x < 8; ++x) {
        const size_t o = o0 + size_t(y) * g.PW + x;
        diff[y * 8 + x] = f.filt[o] - f.idct[o];
      }
    SmallForward(type, diff, 8, blk);
    for (int k = 0; k < 64; ++k) {
      const float interval = k == 0 ? 1.0f * s.mul_dc[c]
                                    : info.dm[c][k] * info.inv_quant_ac;
      s_ratio[c][lb][k] = ClampRatio(blk[k], interval);
    }
  }
  __syncthreads();
  if (!active) return;
  for (int k = 0; k < 64; ++k) {
    float mr = 1.0f;
    int arg = -1;
    for (int cc = 0; cc < 3; ++cc) {
      const float r = s_ratio[cc][lb][k];
      if (r < mr) mr = r, arg = cc;
    }
    if (f.clamp_tape || f.clamp_tape_in) {
      const uint32_t pk = list[i];
      const size_t to = CoefOffset(g, pk & 0xFFFF, pk >> 16, 1, k);
      // The +0.0 case is the only one with a ratio of exactly 0.
      uint8_t code = arg < 0 ? 0 : mr == 0.0f ? 4 : uint8_t(arg + 1);
      if (f.clamp_tape_in) {
        code = f.clamp_tape_in[to];
        mr = TapeRatio(code, s_ratio[0][lb][k], s_ratio[1][lb][k],
                       s_ratio[2][lb][k]);
      }
      if (f.clamp_tape && c == 0) f.clamp_tape[to] = code;
    }
    blk[k] = blk[k] * mr;
  }
  float px[64];
  SmallInverse(type, blk, px, 8);
  for (int y = 0; y < 8; ++y)
    for (int x = 0; x < 8; ++x) {
      const size_t o = o0 + size_t(y) * g.PW + x;
      f.filt[o] = px[y * 8 + x] + f.idct[o];
    }
}


}  // namespace pikgpu

#include "square_kernels.cuh"
#include "tc_kernels.cuh"
#include "stencil_kernels.cuh"
#include "epf_kernel.cuh"

namespace pikgpu {

// Explicit instantiations.
template __global__ void k_square_idct_rows<8>(Geo, DevFrame, const uint32_t*,
                                               int, int);
template __global__ void k_square_idct_rows<16>(Geo, DevFrame,
                                                const uint32_t*, int, int);
template __global__ void k_square_idct_rows<32>(Geo, DevFrame,
                                                const uint32_t*, int, int);
template __global__ void k_square_idct_tc1<16, 2>(Geo, DevFrame,
                                                  const uint32_t*, int, int,
                                                  int*, int*);
template __global__ void k_square_idct_tc1<16, 3>(Geo, DevFrame,
                                                  const uint32_t*, int, int,
                                                  int*, int*);
template __global__ void k_square_ar_tc<16, 2>(Geo, DevFrame, FrameScalars,
                                               const uint32_t*, const int*,
                                               int*, int*);
template __global__ void k_square_ar_tc<16, 3>(Geo, DevFrame, FrameScalars,
                                               const uint32_t*, const int*,
                                               int*, int*);
template __global__ void k_square_idct_tc1<32, 3>(Geo, DevFrame,
                                                  const uint32_t*, int, int,
                                                  int*, int*);
template __global__ void k_square_ar_tc<32, 3>(Geo, DevFrame, FrameScalars,
                                               const uint32_t*, const int*,
                                               int*, int*);
template __global__ void k_square_ar_rows<8>(Geo, DevFrame, FrameScalars,
                                             const uint32_t*, const int*);
template __global__ void k_square_ar_rows<16>(Geo, DevFrame, FrameScalars,
                                              const uint32_t*, const int*);
template __global__ void k_square_ar_rows<32>(Geo, DevFrame, FrameScalars,
                                              const uint32_t*, const int*);

}  // namespace pikgpu
