// Edge-preserving filter (AdaptiveFilter + WeightedSum,
// pik/epf_target.cc:526-801, 1113-1278) on packed guide bytes.
//
// One CTA filters a 64 x 32 pixel tile with 16 warps. Lane l of warp w owns
// the pixels (x0 + 32 (w mod 2) + l, y0 + 4 (w / 2) + j), j = 0..3: one
// column (the 32 lanes of a warp read 32 consecutive values of every
// shared-memory row), four rows inside one 8x8 block row.
//
// The u8 guide is staged in shared memory as one 32-bit word per byte
// offset: word o of a row holds the guide bytes o .. o + 3. The 4 guide bytes
// of a patch row at any offset are then one 32-bit load (and the 32 lanes'
// loads of 32 consecutive offsets hit 32 consecutive words, free of bank
// conflicts), and the sum of absolute differences against the centre
// pixel's patch row is one __vsadu4. For every displacement (cy, cx) of the 7 x 8 neighbourhood and
// every channel, a lane forms the 6 patch-row SADs of each of its columns and
// sums them vertically into the 3 x 4 patch SADs of its 4 rows; the SAD is
// the maximum over the channels. The SADs are exact integers; the weights
// (WeightFast's bit construction) and the weighted sums follow the
// reference's neighbour order (cy = -3..3, cx = -3..4) with separately
// rounded products and sums, so the output equals the per-pixel formulation
// bit for bit.
//
// The guide is quantised from one of three sources: the verification
// override (bytes), a plane (`guide_src`: the sharpened guide, a frame
// without gaborish, the DC image), or -- the common case -- gaborish of
// `in` computed here from the staged input tile (the smoothed plane is then
// never written to memory; `gab` > 0 selects it and its strength).
// Included by recon_kernels.cu.
#pragma once

namespace pikgpu {

constexpr int kEpfW = 64, kEpfH = 32;   // output tile
// Columns per lane: 1 (512 threads, each lane 4 pixels of one column, two
// warps per 4-row band) keeps a thread at <= 64 registers, so two CTAs of
// 16 warps share an SM; 2 (256 threads, 8 pixels per lane) needs ~123.
constexpr int kEpfLaneCols = 1;
constexpr int kEpfThreads = 256 * 2 / kEpfLaneCols;
constexpr int kEpfGH = kEpfH + 8;       // guide rows: y0 - 4 .. y0 + 35
constexpr int kEpfGBytes = 80;          // guide bytes x0 - 8 .. x0 + 71
constexpr int kEpfGRow = kEpfGBytes;    // words per guide row (one per byte)
constexpr int kEpfGPlane = kEpfGH * kEpfGRow;
// Input tile with a 5-pixel halo (enough for gaborish at the guide's
// 4-pixel halo): rows y0 - 5 .. y0 + 36, cols x0 - 12 .. x0 + 75 (the
// column range is widened to 16-byte boundaries for vector loads).
constexpr int kEpfTH = kEpfH + 10;
constexpr int kEpfTW = kEpfW + 24;
constexpr int kEpfTS = kEpfTW;               // row stride in floats
constexpr int kEpfTRow0 = 2, kEpfTCol0 = 9;  // tile index of (y0-3, x0-3)
constexpr size_t kEpfGuideWords = size_t(3) * kEpfGPlane;
constexpr size_t kEpfSmemBytes =
    kEpfGuideWords * 4 + size_t(3) * kEpfTH * kEpfTS * 4;
// Shared memory of k_epf_box with a tile of `th` rows.
constexpr size_t EpfSmemBytes(int th) {
  return size_t(3) * (th + 8) * kEpfGRow * 4 + size_t(3) * (th + 10) * kEpfTS * 4;
}

// WeightFast (pik/epf_target.cc:304-428) as 4 integer operations:
// ((int16(min(sad, 507) << 6) * mul) >> 16 + (127 << 7)) in the high half of
// a float equals ((min(sad, 507) * 64 mul) & 0xFFFF0000) + 0x3F800000 for
// every sad >= 0 and -32768 <= mul < 0 (the product fits in int32).
__device__ __forceinline__ float EpfWeight(int mul64, int sad) {
  const int t = min(sad, 507) * mul64;
  return __uint_as_float((uint32_t(t) & 0xFFFF0000u) + 0x3F800000u);
}

// kFma: the weighted sums with fused multiply-adds (the tensor-core forms,
// which are not bound to the reference's rounding); otherwise every product
// and sum is rounded separately, as the reference does.
// TH: tile rows (32 for frames; 8 for small images such as the DC image,
// which would otherwise be a few CTAs of a full tile's latency each).
template <bool kFma, int TH>
__global__ void __launch_bounds__(16 * TH, TH == 16 ? 3 : 2)
    k_epf_box(const float* in, const float* guide_src,
              const uint8_t* guide_ovr, int gab, int w, int h,
              const uint32_t* mm, const int32_t* sigma, float* out) {
  constexpr int kH = TH, kGH = TH + 8, kTH = TH + 10;
  constexpr int kGPlane = kGH * kEpfGRow, kThreads = 16 * TH;
  constexpr size_t kGuideWords = size_t(3) * kGPlane;
  extern __shared__ __align__(16) uint32_t epf_smem[];
  uint32_t* sg = epf_smem;  // [3][kGH][kEpfGRow]
  float(*tile)[kTH][kEpfTS] =
      reinterpret_cast<float(*)[kTH][kEpfTS]>(epf_smem + kGuideWords);
  const int x0 = blockIdx.x * kEpfW, y0 = blockIdx.y * kH;
  const int tid = threadIdx.x;
  constexpr int LC = kEpfLaneCols;
  const int lane = tid & 31, wp = tid >> 5;
  // 4-row band of the warp and its first column (tile-local).
  const int band = wp / (2 / LC), col0 = 32 * (wp % (2 / LC));
  const size_t plane = size_t(w) * h;
  const int bw = w / 8;
  const int py0 = y0 + 4 * band;  // first row; w and h are multiples of 8
  bool inside[LC], filtered[LC], any_filtered = false;
  int sig[LC];
#pragma unroll
  for (int i = 0; i < LC; ++i) {
    const int px = x0 + lane + col0 + 32 * i;
    inside[i] = px < w && py0 < h;
    sig[i] = inside[i] ? sigma[(py0 >> 3) * bw + (px >> 3)] : 0;
    filtered[i] = sig[i] >= kMinSigma;
    any_filtered |= filtered[i];
  }

  // Tiles without filtered blocks are copies (CopyOriginalBlock).
  if (!__syncthreads_or(any_filtered)) {
#pragma unroll
    for (int i = 0; i < LC; ++i) {
      if (!inside[i]) continue;
      const int px = x0 + lane + col0 + 32 * i;
      for (int c = 0; c < 3; ++c)
        for (int j = 0; j < 4; ++j) {
          const size_t o = c * plane + size_t(py0 + j) * w + px;
          out[o] = in[o];
        }
    }
    return;
  }

  float amin, mul, stretch;
  GuideParams(mm, &amin, &mul, &stretch);
  // Tiles whose halo lies inside the image take vector loads and no
  // mirroring; border tiles mirror every coordinate.
  const bool interior = x0 >= 12 && x0 + kEpfW + 12 <= w && y0 >= 5 &&
                        y0 + kH + 5 <= h;
  if (interior) {
    constexpr int Q = kEpfTW / 4;
    for (int i = tid; i < 3 * kTH * Q; i += kThreads) {
      const int c = i / (kTH * Q);
      const int r = (i / Q) % kTH, q = i % Q;
      CpAsync16(&tile[c][r][4 * q],
                in + c * plane + size_t(y0 - 5 + r) * w + x0 - 12 + 4 * q);
    }
    CpAsyncWaitAll();
  } else {
    for (int i = tid; i < 3 * kTH * kEpfTW; i += kThreads) {
      const int c = i / (kTH * kEpfTW);
      const int r = (i / kEpfTW) % kTH, col = i % kEpfTW;
      const int gx = x0 - 12 + col, gy = y0 - 5 + r;
      tile[c][r][col] =
          in[c * plane + size_t(MirrorIdx(gy, h)) * w + MirrorIdx(gx, w)];
    }
  }
  if (gab) __syncthreads();  // the guide is computed from the tile
  const float* gw = c_t.gaborish[gab];
  auto quant = [&](float v) {
    return uint32_t(uint8_t(uint32_t(__float2int_rz((v - amin) * mul))));
  };
  // Gaborish (Sym3 order) at tile position (ly, lx) from the tile.
  auto smooth = [&](int c, int ly, int lx) {
    const float* t = &tile[c][ly - 1][lx];
    const float* m = &tile[c][ly][lx];
    const float* bt = &tile[c][ly + 1][lx];
    const float sum_tb = t[0] + bt[0];
    const float mul0 = m[0] * gw[0];
    const float sum_lr = m[-1] + m[1];
    const float x1 = sum_tb + sum_lr;
    const float mul1 = x1 * gw[1] + mul0;
    const float sum_t2 = t[-1] + t[1];
    const float sum_b2 = bt[-1] + bt[1];
    const float x2 = sum_t2 + sum_b2;
    return x2 * gw[2] + mul1;
  };
  // u8 guide (MakeGuide, pik/epf_target.cc:1009-1070): the aligned words
  // (offsets 4 wd) first.
  constexpr int kAligned = kEpfGBytes / 4;
  for (int i = tid; i < 3 * kGH * kAligned; i += kThreads) {
    const int c = i / (kGH * kAligned);
    const int r = (i / kAligned) % kGH, wd = i % kAligned;
    const int gy = y0 - 4 + r;
    uint32_t word = 0;
    if (interior && !guide_ovr) {
      if (gab) {
        // Four smoothed values from float4 row segments: tile row r + 1,
        // cols 4 wd + 4 .. 4 wd + 7 (gx = x0 - 8 + 4 wd ..).
        const int lx = 4 * wd + 4;
        float v[3][6];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const float* row = &tile[c][r + k][lx];
          const float4 q = *reinterpret_cast<const float4*>(row);
          v[k][0] = row[-1];
          v[k][1] = q.x, v[k][2] = q.y, v[k][3] = q.z, v[k][4] = q.w;
          v[k][5] = row[4];
        }
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          word |= quant(Sym3Rows(v[0], v[1], v[2], b, gw[0], gw[1], gw[2]))
                  << (8 * b);
        }
      } else {
        const float4 q = *reinterpret_cast<const float4*>(
            guide_src + c * plane + size_t(gy) * w + x0 - 8 + 4 * wd);
        word = quant(q.x) | quant(q.y) << 8 | quant(q.z) << 16 |
               quant(q.w) << 24;
      }
    } else {
      for (int b = 0; b < 4; ++b) {
        const int gx = x0 - 8 + 4 * wd + b;
        uint32_t v = 0;
        if (guide_ovr) {
          const bool ok = gx >= -6 && gx < w + 6 && gy >= -6 && gy < h + 6;
          v = ok ? guide_ovr[(size_t(c) * (h + 12) + gy + 6) * (w + 12) +
                             gx + 6]
                 : 0u;
        } else if (gab) {
          // Smoothed value at the mirrored position, from the tile;
          // positions whose mirror leaves the tile are never read.
          const int ly = MirrorIdx(gy, h) - (y0 - 5);
          const int lx = MirrorIdx(gx, w) - (x0 - 12);
          if (ly >= 1 && ly < kTH - 1 && lx >= 1 && lx < kEpfTW - 1) {
            v = quant(smooth(c, ly, lx));
          }
        } else {
          v = quant(guide_src[c * plane + size_t(MirrorIdx(gy, h)) * w +
                              MirrorIdx(gx, w)]);
        }
        word |= v << (8 * b);
      }
    }
    sg[c * kGPlane + r * kEpfGRow + 4 * wd] = word;
  }
  __syncthreads();
  // The other offsets 4 wd + s, s = 1..3, from the two aligned neighbours
  // (bytes past the row end read as 0).
  for (int i = tid; i < 3 * kGH * kAligned * 3; i += kThreads) {
    const int s = 1 + i % 3;
    const int j = i / 3;
    const int c = j / (kGH * kAligned);
    const int r = (j / kAligned) % kGH, wd = j % kAligned;
    const uint32_t* row = sg + c * kGPlane + r * kEpfGRow;
    const uint32_t lo = row[4 * wd];
    const uint32_t hi = wd + 1 < kAligned ? row[4 * wd + 4] : 0u;
    sg[c * kGPlane + r * kEpfGRow + 4 * wd + s] =
        __funnelshift_r(lo, hi, 8 * s);
  }
  __syncthreads();

  // Warps (half a block row of 8 blocks) without filtered blocks copy.
  if (!__any_sync(0xFFFFFFFFu, any_filtered)) {
#pragma unroll
    for (int i = 0; i < LC; ++i) {
      if (!inside[i]) continue;
      const int px = x0 + lane + col0 + 32 * i;
      for (int c = 0; c < 3; ++c)
        for (int j = 0; j < 4; ++j)
          out[c * plane + size_t(py0 + j) * w + px] =
              tile[c][4 * band + j + 3 + kEpfTRow0]
                  [lane + col0 + 32 * i + 3 + kEpfTCol0];
    }
    return;
  }
  int m64[LC];
#pragma unroll
  for (int i = 0; i < LC; ++i) {
    m64[i] = c_t.mul_table[filtered[i] ? sig[i] : kMinSigma] * 64;
  }

  // Centre patch rows: guide rows py0 - 1 .. py0 + 4, bytes px - 1 .. px + 2.
  const int gr0 = 4 * band + 3;  // guide smem row of py0 - 1
  uint32_t ref[3][6][LC];
  {
    // Byte offset of px - 1 from x0 - 8 (column i is 32 further).
    const uint32_t* g = sg + gr0 * kEpfGRow + lane + col0 + 7;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int i = 0; i < LC; ++i)
          ref[c][r][i] = g[c * kGPlane + r * kEpfGRow + 32 * i];
  }

  float ws[3][4 * LC], sw[4 * LC];
#pragma unroll
  for (int p = 0; p < 4 * LC; ++p) {
    ws[0][p] = ws[1][p] = ws[2][p] = 0.f;
    sw[p] = 0.f;
  }
  if constexpr (kFma && LC == 1) {
    // Tensor-core forms: cx outermost. For one cx the 7 vertical offsets
    // read 12 distinct guide rows per channel (one load each), and each
    // staged input row serves every pixel of the lane it reaches: about
    // 84 shared-memory loads per cx and lane instead of 210. Each pixel's
    // sums run cx-major, not in the reference's cy-major order (these
    // forms are not bound to its rounding).
#pragma unroll 1
    for (int cx = -3; cx <= 4; ++cx) {
      const uint32_t* g = sg + (gr0 - 3) * kEpfGRow + lane + col0 + 7 + cx;
      int sad[4][7];
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int k = 0; k < 7; ++k) sad[j][k] = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        uint32_t wd[12];  // guide rows gr0 - 3 .. gr0 + 8 at this cx
#pragma unroll
        for (int t = 0; t < 12; ++t) wd[t] = g[c * kGPlane + t * kEpfGRow];
        // The centre patch words again from shared memory (registers are
        // the limit at two 512-thread CTAs per SM).
        uint32_t rf[6];
#pragma unroll
        for (int r = 0; r < 6; ++r) {
          rf[r] = sg[c * kGPlane + (gr0 + r) * kEpfGRow + lane + col0 + 7];
        }
#pragma unroll
        for (int k = 0; k < 7; ++k) {  // cy = k - 3: rows k .. k + 5
          int hs[6];
#pragma unroll
          for (int r = 0; r < 6; ++r) hs[r] = int(__vsadu4(rf[r], wd[k + r]));
          const int p12 = hs[1] + hs[2], p34 = hs[3] + hs[4];
          sad[0][k] = max(sad[0][k], hs[0] + p12);
          sad[1][k] = max(sad[1][k], p12 + hs[3]);
          sad[2][k] = max(sad[2][k], hs[2] + p34);
          sad[3][k] = max(sad[3][k], p34 + hs[5]);
        }
      }
      float wt[4][7];
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int k = 0; k < 7; ++k) {
          float wgt = EpfWeight(m64[0], sad[j][k]);
          if (!(wgt >= 0.05f)) wgt = 0.0f;
          wt[j][k] = wgt;
          sw[j] += wgt;
        }
      // Input rows band + R - 3 (R = j + cy + 3 = 0..9) at column px + cx.
      const int col = lane + col0 + 3 + cx + kEpfTCol0;
#pragma unroll
      for (int R = 0; R < 10; ++R) {
        const int ir = 4 * band + R + kEpfTRow0;
        const float v0 = tile[0][ir][col], v1 = tile[1][ir][col],
                    v2 = tile[2][ir][col];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int k = R - j;  // cy + 3
          if (k < 0 || k > 6) continue;
          ws[0][j] = fmaf(v0, wt[j][k], ws[0][j]);
          ws[1][j] = fmaf(v1, wt[j][k], ws[1][j]);
          ws[2][j] = fmaf(v2, wt[j][k], ws[2][j]);
        }
      }
    }
  } else {
  #pragma unroll 1
    for (int cy = -3; cy <= 3; ++cy) {
  #pragma unroll 1
      for (int cx = -3; cx <= 4; ++cx) {
        // Window byte offset (column 0): the patch start moved by cx.
        const uint32_t* g = sg + (gr0 + cy) * kEpfGRow + lane + col0 + 7 + cx;
        int sad[4 * LC];  // [j * LC + i]
  #pragma unroll
        for (int p = 0; p < 4 * LC; ++p) sad[p] = 0;
  #pragma unroll
        for (int c = 0; c < 3; ++c) {
  #pragma unroll
          for (int i = 0; i < LC; ++i) {
            int hs[6];
  #pragma unroll
            for (int r = 0; r < 6; ++r) {
              hs[r] = int(__vsadu4(
                  ref[c][r][i], g[c * kGPlane + r * kEpfGRow + 32 * i]));
            }
            const int p12 = hs[1] + hs[2], p34 = hs[3] + hs[4];
            sad[0 * LC + i] = max(sad[0 * LC + i], hs[0] + p12);
            sad[1 * LC + i] = max(sad[1 * LC + i], p12 + hs[3]);
            sad[2 * LC + i] = max(sad[2 * LC + i], hs[2] + p34);
            sad[3 * LC + i] = max(sad[3 * LC + i], p34 + hs[5]);
          }
        }
  #pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int ir = 4 * band + j + 3 + cy + kEpfTRow0;
  #pragma unroll
          for (int i = 0; i < LC; ++i) {
            const int p = j * LC + i;
            const int col = lane + col0 + 32 * i + 3 + cx + kEpfTCol0;
            float wgt = EpfWeight(m64[i], sad[p]);
            if (!(wgt >= 0.05f)) wgt = 0.0f;
            if (kFma) {
              ws[0][p] = fmaf(tile[0][ir][col], wgt, ws[0][p]);
              ws[1][p] = fmaf(tile[1][ir][col], wgt, ws[1][p]);
              ws[2][p] = fmaf(tile[2][ir][col], wgt, ws[2][p]);
            } else {
              ws[0][p] += tile[0][ir][col] * wgt;
              ws[1][p] += tile[1][ir][col] * wgt;
              ws[2][p] += tile[2][ir][col] * wgt;
            }
            sw[p] += wgt;
          }
        }
      }
    }
  }
#pragma unroll
  for (int i = 0; i < LC; ++i) {
    if (!inside[i]) continue;
    const int px = x0 + lane + col0 + 32 * i;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int p = j * LC + i;
        out[c * plane + size_t(py0 + j) * w + px] =
            filtered[i] ? ws[c][p] / sw[p]
                        : tile[c][4 * band + j + 3 + kEpfTRow0]
                              [lane + col0 + 32 * i + 3 + kEpfTCol0];
      }
  }
}

}  // namespace pikgpu
