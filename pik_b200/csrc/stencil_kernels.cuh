// Shared-memory tile forms of the two full-frame 3x3 stencil passes:
//  * k_gaborish_tile: ConvolveGaborish (pik/gaborish.cc:137-159) of one
//    plane into `out` (skipped when `out` is null: the EPF recomputes the
//    smoothed values it needs), plus the plane's min/max (MinMax,
//    pik/epf_target.cc:980-1006) for the EPF guide (skipped when `mm` is
//    null);
//  * k_gaborish_minmax: the same min/max without staging (the frame path);
//  * k_final_direct: gaborish #2 (or a copy), ShrinkTo(xsize, ysize),
//    XybToRgb (pik/opsin_inverse.cc:38-123) and optional sRGB-8
//    (pik/color_management.cc:323-345, pik/external_image.cc:1205).
//
// k_gaborish_tile stages a 128 x TH output tile with its 1-pixel halo (rows y0 - 1 ..
// y0 + TH, columns x0 - 4 .. x0 + 131, widened to 16-byte boundaries) in
// shared memory: interior tiles with independent 128-bit loads (many in
// flight per thread), border tiles with mirrored scalar loads. Each thread
// then computes 4 adjacent columns of TH / 8 rows, reading 128-bit row
// segments and taking the left/right neighbours from the adjacent lanes.
// The arithmetic of each output is Sym3's, in the same order, so results are
// bit-identical to it. The padded plane width must be a multiple of 4 (it is
// 8 Bx).
// Included by recon_kernels.cu.
#pragma once

namespace pikgpu {

constexpr int kTileW = 128, kTileThreads = 256;
constexpr int kTileSW = kTileW + 8;  // staged columns x0 - 4 .. x0 + 131
constexpr int kGabTileH = 64;        // rows per CTA, min/max pass

// Symmetric 3x3 stencil of output column i (0..3) from three 6-value rows
// (columns x - 1 .. x + 4), in Sym3's operation order.
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

// Asynchronous 16-byte global -> shared copies: interior tiles are staged
// without passing through registers, every copy of a tile (all planes) in
// flight at once, and one wait before the CTA's barrier. The hardware
// tracks completion per thread, so the wait is no spin loop.
__device__ __forceinline__ void CpAsync16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                   uint32_t(__cvta_generic_to_shared(smem))),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void CpAsync4(void* smem, const void* gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                   uint32_t(__cvta_generic_to_shared(smem))),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void CpAsyncWaitAll() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" :::
                   "memory");
}

// Stages plane `p` (w x h, row stride w) around (x0, y0) into `t`
// (TH + 2 rows). Interior tiles are copied asynchronously: the caller
// calls CpAsyncWaitAll before its barrier.
template <int TH>
__device__ __forceinline__ void StageTile(const float* p, int w, int h,
                                          int x0, int y0,
                                          float (*t)[kTileSW]) {
  constexpr int kTileSH = TH + 2;
  const bool interior =
      x0 >= 4 && x0 + kTileW + 4 <= w && y0 >= 1 && y0 + TH + 1 <= h;
  if (interior) {
    constexpr int Q = kTileSW / 4;
    for (int i = threadIdx.x; i < kTileSH * Q; i += kTileThreads) {
      const int r = i / Q, q = i % Q;
      CpAsync16(&t[r][4 * q], p + size_t(y0 - 1 + r) * w + x0 - 4 + 4 * q);
    }
  } else {
    for (int i = threadIdx.x; i < kTileSH * kTileSW; i += kTileThreads) {
      const int r = i / kTileSW, col = i % kTileSW;
      t[r][col] = p[size_t(MirrorIdx(y0 - 1 + r, h)) * w +
                    MirrorIdx(x0 - 4 + col, w)];
    }
  }
}

// Staged row r as 6 values: columns 4 lane - 1 .. 4 lane + 4 of the tile.
__device__ __forceinline__ void TileRow6(const float (*t)[kTileSW], int r,
                                         int lane, float v[6]) {
  const float4 q = *reinterpret_cast<const float4*>(&t[r][4 + 4 * lane]);
  float left = __shfl_up_sync(0xFFFFFFFFu, q.w, 1);
  float right = __shfl_down_sync(0xFFFFFFFFu, q.x, 1);
  if (lane == 0) left = t[r][3];
  if (lane == 31) right = t[r][4 + kTileW];
  v[0] = left;
  v[1] = q.x, v[2] = q.y, v[3] = q.z, v[4] = q.w;
  v[5] = right;
}

__global__ void __launch_bounds__(kTileThreads)
    k_gaborish_tile(const float* in, int w, int h, int strength, float* out,
                    uint32_t* mm) {
  constexpr int TH = kGabTileH, R = TH / 8;
  __shared__ __align__(16) float t[TH + 2][kTileSW];
  __shared__ uint32_t s_lo[kTileThreads / 32], s_hi[kTileThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = blockIdx.z;
  const size_t plane = size_t(w) * h;
  const int x0 = blockIdx.x * kTileW, y0 = blockIdx.y * TH;
  StageTile<TH>(in + c * plane, w, h, x0, y0, t);
  CpAsyncWaitAll();
  __syncthreads();
  const float* wt = c_t.gaborish[strength];
  const float w0 = wt[0], w1 = wt[1], w2 = wt[2];
  const int x = x0 + 4 * lane;
  uint32_t lo = 0xFFFFFFFFu, hi = 0u;
  float a[6], m[6], b[6];
  TileRow6(t, R * warp, lane, a);
  TileRow6(t, R * warp + 1, lane, m);
#pragma unroll
  for (int j = 0; j < R; ++j) {
    TileRow6(t, R * warp + j + 2, lane, b);
    const int y = y0 + R * warp + j;
    if (x < w && y < h) {
      float r[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        r[i] = Sym3Rows(a, m, b, i, w0, w1, w2);
        const uint32_t ob = OrderedBits(r[i]);
        lo = min(lo, ob);
        hi = max(hi, ob);
      }
      if (out) {
        *reinterpret_cast<float4*>(out + c * plane + size_t(y) * w + x) =
            make_float4(r[0], r[1], r[2], r[3]);
      }
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      a[i] = m[i];
      m[i] = b[i];
    }
  }
  if (!mm) return;
  for (int off = 16; off; off >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, off));
    hi = max(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, off));
  }
  if (lane == 0) {
    s_lo[warp] = lo;
    s_hi[warp] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < kTileThreads / 32; ++i) {
      lo = min(lo, s_lo[i]);
      hi = max(hi, s_hi[i]);
    }
    if (lo <= hi) {
      atomicMin(&mm[c], lo);
      atomicMax(&mm[3 + c], hi);
    }
  }
}

// Min/max of gaborish #1 without staging or barriers: each warp owns 128
// columns (4 per lane) of kGmmRows rows and loads its kGmmRows + 2 input
// rows as independent 16-byte loads (all in flight at once); lanes take
// their left/right neighbours from the adjacent lanes, lane 0 and the
// warp's last lane by scalar loads. Coordinates mirror at the image border
// and each output follows Sym3's operation order, so the min/max equal
// those of k_gaborish_tile. Grid: (warps of a plane / 8, 3).
constexpr int kGmmRows = 8;
__global__ void __launch_bounds__(256, 3)
    k_gaborish_minmax(const float* in, int w, int h, int strength,
                      uint32_t* mm) {
  PdlLaunchDependents();  // the EPF may start on free SMs
  constexpr int R = kGmmRows;
  __shared__ uint32_t s_lo[8], s_hi[8];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int c = blockIdx.y;
  const int tiles_x = (w + 127) / 128;
  const int wg = blockIdx.x * 8 + wib;
  const int x0 = (wg % tiles_x) * 128, y0 = (wg / tiles_x) * R;
  const int x = x0 + 4 * lane;
  uint32_t lo = 0xFFFFFFFFu, hi = 0u;
  if (y0 < h) {  // warp-uniform
    const float* p = in + c * size_t(w) * h;
    const bool xv = x < w;
    // Lanes whose right neighbour is not in the next lane's registers.
    const bool own_right = lane == 31 || x + 4 >= w;
    const int xl = MirrorIdx(x0 - 1, w), xr = MirrorIdx(x + 4, w);
    float4 q[R + 2];
    float el[R + 2], er[R + 2];
#pragma unroll
    for (int r = 0; r < R + 2; ++r) {
      const float* row = p + size_t(MirrorIdx(y0 - 1 + r, h)) * w;
      q[r] = xv ? *reinterpret_cast<const float4*>(row + x)
                : make_float4(0.f, 0.f, 0.f, 0.f);
      el[r] = lane == 0 ? row[xl] : 0.f;
      er[r] = own_right && xv ? row[xr] : 0.f;
    }
    const float* wt = c_t.gaborish[strength];
    const float w0 = wt[0], w1 = wt[1], w2 = wt[2];
    auto row6 = [&](int r, float v[6]) {
      const float left = __shfl_up_sync(0xFFFFFFFFu, q[r].w, 1);
      const float right = __shfl_down_sync(0xFFFFFFFFu, q[r].x, 1);
      v[0] = lane == 0 ? el[r] : left;
      v[1] = q[r].x, v[2] = q[r].y, v[3] = q[r].z, v[4] = q[r].w;
      v[5] = own_right ? er[r] : right;
    };
    float a[6], m[6], b[6];
    row6(0, a);
    row6(1, m);
#pragma unroll
    for (int j = 0; j < R; ++j) {
      row6(j + 2, b);
      if (xv) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const uint32_t ob = OrderedBits(Sym3Rows(a, m, b, i, w0, w1, w2));
          lo = min(lo, ob);
          hi = max(hi, ob);
        }
      }
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        a[i] = m[i];
        m[i] = b[i];
      }
    }
  }
  for (int off = 16; off; off >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, off));
    hi = max(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, off));
  }
  if (lane == 0) {
    s_lo[wib] = lo;
    s_hi[wib] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < 8; ++i) {
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

// The final pass without staging or barriers: each warp owns 128 columns x
// kFinRows output rows of the three planes and loads its input rows
// (kFinRows + 2 per plane with gaborish, kFinRows without) as independent
// 16-byte loads up front;
// horizontal neighbours come from the adjacent lanes, lane 0's and the
// row's last lane's by scalar loads. Coordinates mirror at the padded
// plane's border (pw x ph). `vec_lin`: the linear outputs may be written as
// float4 (width, stride and base all multiples of 4 floats / 16 bytes).
// Grid: warps / 8.
constexpr int kFinRows = 2;
template <bool kGab>
__global__ void __launch_bounds__(256)
    k_final_direct(const float* in, int pw, int ph, int w, int h,
                   int strength, float* pre, float* lin, size_t lin_stride,
                   int vec_lin, uint8_t* rgb8, size_t rgb8_stride) {
  constexpr int R = kFinRows, NR = kGab ? R + 2 : R;
  const int lane = threadIdx.x & 31;
  const int wg = blockIdx.x * 8 + (threadIdx.x >> 5);
  const int tiles_x = (w + 127) / 128;
  const int x0 = (wg % tiles_x) * 128, y0 = (wg / tiles_x) * R;
  if (y0 >= h) return;  // warp-uniform; no barriers below
  const size_t plane = size_t(pw) * ph;
  const int x = x0 + 4 * lane;
  const bool xv = x < pw;
  const bool own_right = lane == 31 || x + 4 >= pw;
  const int xl = MirrorIdx(x0 - 1, pw), xr = MirrorIdx(x + 4, pw);
  float4 q[3][NR];
  float el[3][NR], er[3][NR];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      const int y = kGab ? y0 - 1 + r : y0 + r;
      const float* row = in + c * plane + size_t(MirrorIdx(y, ph)) * pw;
      q[c][r] = xv ? *reinterpret_cast<const float4*>(row + x)
                   : make_float4(0.f, 0.f, 0.f, 0.f);
      if (kGab) {
        el[c][r] = lane == 0 ? row[xl] : 0.f;
        er[c][r] = own_right && xv ? row[xr] : 0.f;
      }
    }
  const float* wt = c_t.gaborish[strength];
  const float w0 = wt[0], w1 = wt[1], w2 = wt[2];
  auto row6 = [&](int c, int r, float v[6]) {
    const float left = __shfl_up_sync(0xFFFFFFFFu, q[c][r].w, 1);
    const float right = __shfl_down_sync(0xFFFFFFFFu, q[c][r].x, 1);
    v[0] = lane == 0 ? el[c][r] : left;
    v[1] = q[c][r].x, v[2] = q[c][r].y, v[3] = q[c][r].z, v[4] = q[c][r].w;
    v[5] = own_right ? er[c][r] : right;
  };
#pragma unroll
  for (int j = 0; j < R; ++j) {
    const int y = y0 + j;
    float v[3][4];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (kGab) {
        float a[6], m[6], b[6];
        row6(c, j, a);
        row6(c, j + 1, m);
        row6(c, j + 2, b);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          v[c][i] = Sym3Rows(a, m, b, i, w0, w1, w2);
        }
      } else {
        v[c][0] = q[c][j].x, v[c][1] = q[c][j].y;
        v[c][2] = q[c][j].z, v[c][3] = q[c][j].w;
      }
    }
    if (x >= w || y >= h) continue;
    const int n = min(4, w - x);
    if (pre) {
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if (i < n) pre[(size_t(c) * h + y) * w + x + i] = v[c][i];
    }
    float r[4], g[4], bl[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      XybToRgb(v[0][i], v[1][i], v[2][i], &r[i], &g[i], &bl[i]);
    }
    if (lin) {
      float* o0 = lin + size_t(y) * lin_stride + x;
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
      uint8_t* o = rgb8 + size_t(y) * rgb8_stride + 3 * size_t(x);
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
