// Row-strip forms of the two full-frame 3x3 stencil passes:
//  * k_gaborish_strips: ConvolveGaborish (pik/gaborish.cc:137-159) of one
//    plane into `out` (skipped when `out` is null: the EPF recomputes the
//    smoothed values it needs), plus the plane's min/max (MinMax,
//    pik/epf_target.cc:980-1006) for the EPF guide (skipped when `mm` is
//    null);
//  * k_final_strips: gaborish #2 (or a copy), ShrinkTo(xsize, ysize), XybToRgb
//    (pik/opsin_inverse.cc:38-123) and optional sRGB-8
//    (pik/color_management.cc:323-345, pik/external_image.cc:1205).
//
// Each thread owns a 4-pixel-wide column strip of kStripRows rows: one
// 128-bit load per input row, the left/right neighbours from the adjacent
// lanes by shuffle (explicit loads only at warp and image edges) and a
// 3-row sliding window in registers, so every input value is loaded once
// per warp. A warp covers 128 pixels of a row band; the 8 warps of a CTA
// stack vertically (128 x 64 pixels per CTA). The arithmetic of each output
// is Sym3's, in the same order, so results are bit-identical to it.
// Requires the padded plane width to be a multiple of 4 (it is 8 Bx).
// Included by recon_kernels.cu.
#pragma once

namespace pikgpu {

constexpr int kStripRows = 8;
constexpr int kStripThreads = 256;
constexpr int kStripW = 128;                              // pixels per warp
constexpr int kStripH = kStripRows * (kStripThreads / 32);  // rows per CTA

// Row `y` (already mirrored) of a plane as 6 values: columns x0-1 .. x0+4.
__device__ __forceinline__ void LoadRow6(const float* plane, int w, int y,
                                         int x0, int lane, float v[6]) {
  const float* row = plane + size_t(y) * w;
  float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
  if (x0 < w) q = *reinterpret_cast<const float4*>(row + x0);
  float left = __shfl_up_sync(0xFFFFFFFFu, q.w, 1);
  float right = __shfl_down_sync(0xFFFFFFFFu, q.x, 1);
  if (x0 < w) {
    if (lane == 0 || x0 == 0) left = row[MirrorIdx(x0 - 1, w)];
    if (lane == 31 || x0 + 4 >= w) right = row[MirrorIdx(x0 + 4, w)];
  }
  v[0] = left;
  v[1] = q.x;
  v[2] = q.y;
  v[3] = q.z;
  v[4] = q.w;
  v[5] = right;
}

// Sym3 of output column i (0..3) from the three rows, same order as Sym3.
__device__ __forceinline__ float Sym3Rows(const float* t, const float* m,
                                          const float* b, int i, float w0,
                                          float w1, float w2) {
  const float sum_tb = t[i + 1] + b[i + 1];
  const float mul0 = m[i + 1] * w0;
  const float sum_lr = m[i] + m[i + 2];
  const float x1 = sum_tb + sum_lr;
  const float mul1 = x1 * w1 + mul0;
  const float sum_t2 = t[i] + t[i + 2];
  const float sum_b2 = b[i] + b[i + 2];
  const float x2 = sum_t2 + sum_b2;
  return x2 * w2 + mul1;
}

__global__ void __launch_bounds__(kStripThreads)
    k_gaborish_strips(const float* in, int w, int h, int strength, float* out,
                      uint32_t* mm) {
  __shared__ uint32_t s_lo[kStripThreads / 32], s_hi[kStripThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = blockIdx.z;
  const size_t plane = size_t(w) * h;
  const float* p = in + c * plane;
  float* o = out ? out + c * plane : nullptr;
  const int x0 = blockIdx.x * kStripW + 4 * lane;
  const int y0 = blockIdx.y * kStripH + warp * kStripRows;
  const float* wt = c_t.gaborish[strength];
  const float w0 = wt[0], w1 = wt[1], w2 = wt[2];
  uint32_t lo = 0xFFFFFFFFu, hi = 0u;
  if (y0 < h) {
    float t[6], m[6], b[6];
    LoadRow6(p, w, MirrorIdx(y0 - 1, h), x0, lane, t);
    LoadRow6(p, w, y0, x0, lane, m);
    const int y1 = min(y0 + kStripRows, h);
    for (int y = y0; y < y1; ++y) {
      LoadRow6(p, w, MirrorIdx(y + 1, h), x0, lane, b);
      if (x0 < w) {
        float r[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          r[i] = Sym3Rows(t, m, b, i, w0, w1, w2);
          const uint32_t ob = OrderedBits(r[i]);
          lo = min(lo, ob);
          hi = max(hi, ob);
        }
        if (out) {
          *reinterpret_cast<float4*>(o + size_t(y) * w + x0) =
              make_float4(r[0], r[1], r[2], r[3]);
        }
      }
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        t[i] = m[i];
        m[i] = b[i];
      }
    }
  }
  for (int off = 16; off; off >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, off));
    hi = max(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, off));
  }
  if (lane == 0) {
    s_lo[warp] = lo;
    s_hi[warp] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0 && mm) {
    for (int i = 1; i < kStripThreads / 32; ++i) {
      lo = min(lo, s_lo[i]);
      hi = max(hi, s_hi[i]);
    }
    if (lo <= hi) {
      atomicMin(&mm[c], lo);
      atomicMax(&mm[3 + c], hi);
    }
  }
}

// Opsin inverse of one pixel (XybToRgb), same operation order as before.
__device__ __forceinline__ void XybToRgb(float x, float y, float b, float* r,
                                         float* g, float* bl) {
  const float* m = c_t.opsin_inv;
  const float gr = 1.0f * (y + x);
  const float gg = 1.0f * (y - x);
  const float gb = b;
  const float mr = gr * gr * gr + c_t.opsin_neg_bias[0];
  const float mg = gg * gg * gg + c_t.opsin_neg_bias[1];
  const float mb = gb * gb * gb + c_t.opsin_neg_bias[2];
  float lr = m[0] * mr, lg = m[3] * mr, lb = m[6] * mr;
  const float tr = m[1] * mg, tg = m[4] * mg, tb = m[7] * mg;
  lr = m[2] * mb + lr;
  lg = m[5] * mb + lg;
  lb = m[8] * mb + lb;
  *r = lr + tr;
  *g = lg + tg;
  *bl = lb + tb;
}

// `vec_lin`: the linear outputs may be written as float4 (width, stride and
// base all multiples of 4 floats / 16 bytes).
__global__ void __launch_bounds__(kStripThreads)
    k_final_strips(const float* in, int pw, int ph, int w, int h,
                   int strength, float* pre, float* lin, size_t lin_stride,
                   int vec_lin, uint8_t* rgb8, size_t rgb8_stride) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t plane = size_t(pw) * ph;
  const int x0 = blockIdx.x * kStripW + 4 * lane;
  const int y0 = blockIdx.y * kStripH + warp * kStripRows;
  if (y0 >= h) return;  // whole warp: y0 is warp-uniform
  const float* wt = c_t.gaborish[strength];
  const float w0 = wt[0], w1 = wt[1], w2 = wt[2];
  float t[3][6], m[3][6], b[3][6];
  if (strength) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      LoadRow6(in + c * plane, pw, MirrorIdx(y0 - 1, ph), x0, lane, t[c]);
      LoadRow6(in + c * plane, pw, y0, x0, lane, m[c]);
    }
  }
  const int y1 = min(y0 + kStripRows, h);
  for (int y = y0; y < y1; ++y) {
    float v[3][4];
    if (strength) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        LoadRow6(in + c * plane, pw, MirrorIdx(y + 1, ph), x0, lane, b[c]);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          v[c][i] = Sym3Rows(t[c], m[c], b[c], i, w0, w1, w2);
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          t[c][i] = m[c][i];
          m[c][i] = b[c][i];
        }
      }
    } else if (x0 < pw) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float4 q = *reinterpret_cast<const float4*>(
            in + c * plane + size_t(y) * pw + x0);
        v[c][0] = q.x, v[c][1] = q.y, v[c][2] = q.z, v[c][3] = q.w;
      }
    }
    if (x0 >= w) continue;
    const int n = min(4, w - x0);
    if (pre) {
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if (i < n) pre[(size_t(c) * h + y) * w + x0 + i] = v[c][i];
    }
    float r[4], g[4], bl[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      XybToRgb(v[0][i], v[1][i], v[2][i], &r[i], &g[i], &bl[i]);
    }
    if (lin) {
      float* o0 = lin + size_t(y) * lin_stride + x0;
      float* o1 = o0 + lin_stride * h;
      float* o2 = o1 + lin_stride * h;
      if (vec_lin) {
        *reinterpret_cast<float4*>(o0) = make_float4(r[0], r[1], r[2], r[3]);
        *reinterpret_cast<float4*>(o1) = make_float4(g[0], g[1], g[2], g[3]);
        *reinterpret_cast<float4*>(o2) =
            make_float4(bl[0], bl[1], bl[2], bl[3]);
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          if (i < n) {
            o0[i] = r[i];
            o1[i] = g[i];
            o2[i] = bl[i];
          }
        }
      }
    }
    if (rgb8) {
      uint8_t* o = rgb8 + size_t(y) * rgb8_stride + 3 * size_t(x0);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        if (i < n) {
          o[3 * i + 0] = Srgb8(r[i]);
          o[3 * i + 1] = Srgb8(g[i]);
          o[3 * i + 2] = Srgb8(bl[i]);
        }
      }
    }
  }
}

}  // namespace pikgpu
