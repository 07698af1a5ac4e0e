// Edge-preserving filter (AdaptiveFilter + WeightedSum,
// pik/epf_target.cc:526-801, 1113-1278) on packed guide bytes.
//
// A CTA filters 64 x TH pixel tiles with 2 TH / 4 warps. Lane l of warp w
// owns the pixels (x0 + 32 (w mod 2) + l, y0 + 4 (w / 2) + j), j = 0..3: one
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

constexpr int kEpfW = 64, kEpfH = 32;   // output tile (TH = kEpfH)
constexpr int kEpfThreads = 16 * kEpfH;  // two warps per 4-row band
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
constexpr int kEpfAligned = kEpfGBytes / 4;  // aligned guide words per row
// Shared memory of k_epf_box with a tile of `th` rows: the guide words (one
// per byte offset), the input tile and the aligned guide words.
constexpr size_t EpfSmemBytes(int th) {
  return size_t(3) * (th + 8) * kEpfGRow * 4 +
         size_t(3) * (th + 10) * kEpfTS * 4 +
         size_t(3) * (th + 8) * kEpfAligned * 4 + 16;  // + the TMA mbarrier
}
// Bytes of one tile's TMA copy (three planes of TH + 10 rows of kEpfTW).
__host__ __device__ constexpr uint32_t EpfTileBytes(int th) {
  return uint32_t(3 * (th + 10) * kEpfTW * 4);
}
constexpr size_t kEpfSmemBytes = EpfSmemBytes(kEpfH);

// WeightFast (pik/epf_target.cc:304-428) as 4 integer operations:
// ((int16(min(sad, 507) << 6) * mul) >> 16 + (127 << 7)) in the high half of
// a float equals ((min(sad, 507) * 64 mul) & 0xFFFF0000) + 0x3F800000 for
// every sad >= 0 and -32768 <= mul < 0 (the product fits in int32).
__device__ __forceinline__ float EpfWeight(int mul64, int sad) {
  const int t = min(sad, 507) * mul64;
  return __uint_as_float((uint32_t(t) & 0xFFFF0000u) + 0x3F800000u);
}

// The weight with the reference's cut-off (weights below 0.05 are 0) in
// four integer operations. EpfWeight falls as the SAD grows (mul < 0), so
// the cut-off is a SAD threshold `thr` per sigma (c_t.epf_thr); above it
// the weight is `cap`: 0, or EpfWeight(507) when even the largest clamped
// SAD keeps its weight (then thr = 507). For sad <= thr <= 507 the product
// has no wrap and the clamp is the identity; larger SADs only select `cap`.
struct EpfCut {
  uint32_t thr;
  float cap;
};
__device__ __forceinline__ EpfCut EpfCutOf(int sigma, int mul64) {
  EpfCut k;
  k.thr = uint32_t(c_t.epf_thr[sigma]);
  k.cap = k.thr == 507u ? EpfWeight(mul64, 507) : 0.0f;
  return k;
}
__device__ __forceinline__ float EpfCutWeight(int mul64, EpfCut k,
                                              uint32_t sad) {
  const uint32_t u = sad * uint32_t(mul64) + 0x3F800000u;
  return sad <= k.thr ? __uint_as_float(u & 0xFFFF0000u) : k.cap;
}

// Sum of the absolute differences of the four bytes of a and b, plus c
// (the accumulating form of __vsadu4).
__device__ __forceinline__ uint32_t Sad4(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t d;
  asm("vabsdiff4.u32.u32.u32.add %0, %1, %2, %3;"
      : "=r"(d)
      : "r"(a), "r"(b), "r"(c));
  return d;
}

// The 3-row patch SADs of 4 pixel rows from 6 patch-row pairs (centre row
// r against window row r): six byte-SADs (rows 1 + 2 and 3 + 4 accumulated
// onto rows 2 and 3, rows 0 and 5 onto those pairs) and two adds, which
// need not run on the integer ALU. c0: the first channel (no maximum).
template <bool c0>
__device__ __forceinline__ void PatchSads4(const uint32_t* rf,
                                           const uint32_t* wd, uint32_t* sad) {
  const uint32_t h2 = Sad4(rf[2], wd[2], 0u);
  const uint32_t h3 = Sad4(rf[3], wd[3], 0u);
  const uint32_t p12 = Sad4(rf[1], wd[1], h2);
  const uint32_t p34 = Sad4(rf[4], wd[4], h3);
  const uint32_t s0 = Sad4(rf[0], wd[0], p12);
  const uint32_t s1 = p12 + h3;
  const uint32_t s2 = p34 + h2;
  const uint32_t s3 = Sad4(rf[5], wd[5], p34);
  if (c0) {
    sad[0] = s0, sad[1] = s1, sad[2] = s2, sad[3] = s3;
  } else {
    sad[0] = max(sad[0], s0), sad[1] = max(sad[1], s1);
    sad[2] = max(sad[2], s2), sad[3] = max(sad[3], s3);
  }
}

// Where the per-block sigma comes from. It is computed in the kernel from
// the guide's stretch (SigmaFromQuant, pik/epf_target.cc:1072-1111):
// `ovr` (the verification override) if set; else `fixed` if >= 0 (the
// fixed-sigma EPF, pik/epf_target.cc:1342-1386); else from qf, strategy
// and LUT per block; or, qf NULL (the DC image), from the constant
// `const_qf` with a DCT strategy and LUT 0 (AdaptiveDCReconstruction,
// pik/adaptive_reconstruction.cc:300-318). The sigma used is written to
// `out` (NULL: not written) by one lane per block.
struct EpfSigma {
  const int32_t* ovr;
  const int32_t* qf;
  const uint8_t* acs;
  const uint8_t* lut;
  int const_qf;
  int fixed;
  int32_t* out;
};

// The DC image's output: instead of storing the filtered value, the clamp
// of AdaptiveDCReconstruction (pik/adaptive_reconstruction.cc:319-331),
// dc = max(dc - hs, min(filtered, dc + hs)), into the w x h planes at `dc`
// (the padding is dropped). dc NULL: the frame EPF, which stores `out`.
struct EpfDc {
  float* dc;
  int w, h;
  float hs0, hs1, hs2;
};

// Sigma of this thread's block in the tile at (x0, y0); 0 outside the image.
// Sigma of the block holding pixel (px, py0) (0 outside the image); `store`:
// also write it to s.out.
__device__ __forceinline__ int EpfBlockSigma(const EpfSigma& s, float stretch,
                                             int w, int h, int px, int py0,
                                             bool store) {
  if (px >= w || py0 >= h) return 0;
  const int bi = (py0 >> 3) * (w / 8) + (px >> 3);
  int sg;
  if (s.ovr) {
    sg = s.ovr[bi];
  } else if (s.fixed >= 0) {
    sg = s.fixed;
  } else if (s.qf) {
    sg = SigmaFromQuant(float(s.qf[bi]), ARQuantScaleOf(s.acs[bi] >> 4),
                        s.lut[bi], stretch);
  } else {
    sg = SigmaFromQuant(float(s.const_qf), 1.0f, 0, stretch);
  }
  if (s.out && store) s.out[bi] = sg;
  return sg;
}

__device__ __forceinline__ int EpfLaneSigma(const EpfSigma& s, float stretch,
                                            int w, int h, int x0, int y0) {
  const int t = threadIdx.x;
  const int px = x0 + (t & 31) + 32 * ((t >> 5) & 1), py0 = y0 + 4 * (t >> 6);
  return EpfBlockSigma(s, stretch, w, h, px, py0,
                       (px & 7) == 0 && (py0 & 7) == 0);
}

// Stores the value of channel c at pixel (px, y) of the tile's output.
__device__ __forceinline__ void EpfStore(float* out, const EpfDc& dco,
                                         size_t plane, int w, int c, int px,
                                         int y, float v) {
  if (dco.dc) {
    if (px < dco.w && y < dco.h) {
      float& d = dco.dc[(size_t(c) * dco.h + y) * dco.w + px];
      const float hs = c == 0 ? dco.hs0 : c == 1 ? dco.hs1 : dco.hs2;
      const float lo = d - hs, hi = d + hs;
      const float m = v < hi ? v : hi;
      d = lo < m ? m : lo;
    }
  } else {
    out[c * plane + size_t(y) * w + px] = v;
  }
}

// Tiles whose halo lies inside the image take vector copies and no
// mirroring; border tiles mirror every coordinate.
template <int TH>
__device__ __forceinline__ bool EpfInterior(int w, int h, int x0, int y0) {
  return x0 >= 12 && x0 + kEpfW + 12 <= w && y0 >= 5 && y0 + TH + 5 <= h;
}

// Stages input rows y0 - 5 .. y0 + TH + 4, columns x0 - 12 .. x0 + 75 of
// the three planes into `tile` by asynchronous copies: 16 bytes each for
// interior tiles, 4 bytes per mirrored coordinate at the image border. The
// caller commits them and waits.
template <int TH, int NT = 16 * TH>
__device__ __forceinline__ void EpfStage(const float* in, int w, int h, int x0,
                                         int y0,
                                         float (*tile)[TH + 10][kEpfTS],
                                         int tid) {
  constexpr int kTH = TH + 10, kThreads = NT;
  const size_t plane = size_t(w) * h;
  if (EpfInterior<TH>(w, h, x0, y0)) {
    constexpr int Q = kEpfTW / 4;
    for (int i = tid; i < 3 * kTH * Q; i += kThreads) {
      const int c = i / (kTH * Q);
      const int r = (i / Q) % kTH, q = i % Q;
      CpAsync16(&tile[c][r][4 * q],
                in + c * plane + size_t(y0 - 5 + r) * w + x0 - 12 + 4 * q);
    }
  } else {
    for (int i = tid; i < 3 * kTH * kEpfTW; i += kThreads) {
      const int c = i / (kTH * kEpfTW);
      const int r = (i / kEpfTW) % kTH, col = i % kEpfTW;
      const int gx = x0 - 12 + col, gy = y0 - 5 + r;
      CpAsync4(&tile[c][r][col],
               in + c * plane + size_t(MirrorIdx(gy, h)) * w + MirrorIdx(gx, w));
    }
  }
}

// Builds the tile's u8 guide (MakeGuide, pik/epf_target.cc:1009-1070) in
// shared memory: the aligned words into `sa`, then one word per byte offset
// into `sg`. NT threads take part (this thread is `tid` of them), and
// `sync` is their barrier; the tile's copies are complete and published.
// Returns after the last barrier.
template <int TH, int NT, typename Sync>
__device__ __forceinline__ void EpfBuildGuide(
    int tid, Sync sync, const float* guide_src, const uint8_t* guide_ovr,
    int gab, int w, int h, float amin, float mul, uint32_t* sg, uint32_t* sa,
    float (*tile)[TH + 10][kEpfTS], int x0, int y0) {
  constexpr int kGH = TH + 8, kTH = TH + 10;
  const size_t plane = size_t(w) * h;
  const bool interior = EpfInterior<TH>(w, h, x0, y0);
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
  // (bytes 4 wd .. 4 wd + 3 of a row) first, into `sa` (row-major, one
  // row of kEpfAligned words per channel and guide row).
  constexpr int kAligned = kEpfAligned;
  // Interior tiles with the smoothed guide: each thread takes a vertical
  // strip of kStrip words of one channel and column, with its three input
  // rows rolling down the strip, so that each input row is loaded once and
  // its pair sums v[i] + v[i + 2] (Sym3's left/right and corner sums) are
  // formed once for the three output rows that use them. The arithmetic of
  // each value is Sym3Rows', in its order.
  constexpr int kStrip = (3 * kGH * kAligned + NT - 1) / NT;
  static_assert(kGH % kStrip == 0, "whole strips");
  constexpr int kStrips = kGH / kStrip;
  const bool strips = interior && !guide_ovr && gab;
  if (strips && tid < 3 * kAligned * kStrips) {
    const int wd = tid % kAligned, c = (tid / kAligned) % 3;
    const int r0 = (tid / (3 * kAligned)) * kStrip;
    const int lx = 4 * wd + 4;
    float t[6], m[6], b[6], ht[4], hm[4], hb[4];
    auto load = [&](int r, float* v, float* hv) {
      const float* row = &tile[c][r][lx];
      const float4 q = *reinterpret_cast<const float4*>(row);
      v[0] = row[-1];
      v[1] = q.x, v[2] = q.y, v[3] = q.z, v[4] = q.w;
      v[5] = row[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) hv[i] = v[i] + v[i + 2];
    };
    load(r0, t, ht);
    load(r0 + 1, m, hm);
#pragma unroll
    for (int j = 0; j < kStrip; ++j) {
      load(r0 + j + 2, b, hb);
      uint32_t word = 0;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float sum_tb = t[i + 1] + b[i + 1];
        const float mul0 = m[i + 1] * gw[0];
        const float x1 = sum_tb + hm[i];
        const float mul1 = x1 * gw[1] + mul0;
        const float x2 = ht[i] + hb[i];
        word |= quant(x2 * gw[2] + mul1) << (8 * i);
      }
      sa[(c * kGH + r0 + j) * kAligned + wd] = word;
#pragma unroll
      for (int i = 0; i < 6; ++i) t[i] = m[i], m[i] = b[i];
#pragma unroll
      for (int i = 0; i < 4; ++i) ht[i] = hm[i], hm[i] = hb[i];
    }
  }
  for (int i = tid; i < 3 * kGH * kAligned && !strips; i += NT) {
    const int cr = i / kAligned, wd = i - cr * kAligned;
    const int c = cr / kGH, r = cr - c * kGH;
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
    sa[i] = word;
  }
  sync();
  // The words of offsets 4 wd .. 4 wd + 3 from the two aligned neighbours
  // (bytes past the row end read as 0), one 16-byte store each.
  for (int i = tid; i < 3 * kGH * kAligned; i += NT) {
    const int cr = i / kAligned, wd = i - cr * kAligned;
    const uint32_t lo = sa[i];
    const uint32_t hi = wd + 1 < kAligned ? sa[i + 1] : 0u;
    *reinterpret_cast<uint4*>(sg + cr * kEpfGRow + 4 * wd) =
        make_uint4(lo, __funnelshift_r(lo, hi, 8), __funnelshift_r(lo, hi, 16),
                   __funnelshift_r(lo, hi, 24));
  }
  sync();

}

// Filters the tile from its staged input and guide (this thread's pixels:
// `tid` < 16 TH of the tile's filtering threads), with `sig` the sigma of
// this thread's block, and stores the result. No CTA barrier.
template <bool kFma, int TH>
__device__ __forceinline__ void EpfFilterCore(
    int tid, int sig, float* out, const EpfDc& dco, int w, int h,
    const uint32_t* sg, float (*tile)[TH + 10][kEpfTS], int x0, int y0) {
  constexpr int kGH = TH + 8;
  constexpr int kGPlane = kGH * kEpfGRow;
  const int lane = tid & 31, wp = tid >> 5;
  // 4-row band of the warp and its first column (tile-local).
  const int band = wp >> 1, col0 = 32 * (wp & 1);
  const size_t plane = size_t(w) * h;
  const int px = x0 + lane + col0, py0 = y0 + 4 * band;
  const bool inside = px < w && py0 < h;  // w and h are multiples of 8
  const bool filtered = sig >= kMinSigma;
  // Tile position of the pixel (px, py0).
  const int tr0 = 4 * band + 3 + kEpfTRow0, tc0 = lane + col0 + 3 + kEpfTCol0;

  // Warps (half a block row of 8 blocks) without filtered blocks copy.
  if (!__any_sync(0xFFFFFFFFu, filtered)) {
    if (inside) {
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int j = 0; j < 4; ++j)
          EpfStore(out, dco, plane, w, c, px, py0 + j, tile[c][tr0 + j][tc0]);
    }
    return;
  }
  const int m64 = c_t.mul_table[filtered ? sig : kMinSigma] * 64;
  const EpfCut cut = EpfCutOf(filtered ? sig : kMinSigma, m64);

  // Centre patch rows: guide rows py0 - 1 .. py0 + 4, bytes px - 1 .. px + 2
  // (byte offset of px - 1 from x0 - 8).
  const int gr0 = 4 * band + 3;  // guide smem row of py0 - 1
  const int gc0 = lane + col0 + 7;
  float ws[3][4], sw[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    ws[0][j] = ws[1][j] = ws[2][j] = 0.f;
    sw[j] = 0.f;
  }
  if constexpr (kFma) {
    // Tensor-core forms: cx outermost. For one cx the 7 vertical offsets
    // read 12 distinct guide rows per channel (one load each), and each
    // staged input row serves every pixel of the lane it reaches: about
    // 84 shared-memory loads per cx and lane instead of 210. Each pixel's
    // sums run cx-major, not in the reference's cy-major order (these
    // forms are not bound to its rounding).
#pragma unroll 1
    for (int cx = -3; cx <= 4; ++cx) {
      const uint32_t* g = sg + (gr0 - 3) * kEpfGRow + gc0 + cx;
      uint32_t sad[7][4];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        uint32_t wd[12];  // guide rows gr0 - 3 .. gr0 + 8 at this cx
#pragma unroll
        for (int t = 0; t < 12; ++t) wd[t] = g[c * kGPlane + t * kEpfGRow];
        // The centre patch words again from shared memory (registers are
        // the limit).
        uint32_t rf[6];
#pragma unroll
        for (int r = 0; r < 6; ++r) {
          rf[r] = sg[c * kGPlane + (gr0 + r) * kEpfGRow + gc0];
        }
#pragma unroll
        for (int k = 0; k < 7; ++k) {  // cy = k - 3: rows k .. k + 5
          if (c == 0) {
            PatchSads4<true>(rf, wd + k, sad[k]);
          } else {
            PatchSads4<false>(rf, wd + k, sad[k]);
          }
        }
      }
      float wt[4][7];
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int k = 0; k < 7; ++k) {
          const float wgt = EpfCutWeight(m64, cut, sad[k][j]);
          wt[j][k] = wgt;
          sw[j] += wgt;
        }
      // Input rows band + R - 3 (R = j + cy + 3 = 0..9) at column px + cx.
      const int col = tc0 + cx;
#pragma unroll
      for (int R = 0; R < 10; ++R) {
        const int ir = tr0 - 3 + R;
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
    // The reference's order: cy-major, products and sums rounded separately.
    uint32_t ref[3][6];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int r = 0; r < 6; ++r)
        ref[c][r] = sg[c * kGPlane + (gr0 + r) * kEpfGRow + gc0];
#pragma unroll 1
    for (int cy = -3; cy <= 3; ++cy) {
#pragma unroll 1
      for (int cx = -3; cx <= 4; ++cx) {
        // Window byte offset: the patch start moved by cx.
        const uint32_t* g = sg + (gr0 + cy) * kEpfGRow + gc0 + cx;
        uint32_t sad[4];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          uint32_t wd[6];
#pragma unroll
          for (int r = 0; r < 6; ++r) wd[r] = g[c * kGPlane + r * kEpfGRow];
          if (c == 0) {
            PatchSads4<true>(ref[c], wd, sad);
          } else {
            PatchSads4<false>(ref[c], wd, sad);
          }
        }
        const int col = tc0 + cx;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int ir = tr0 + j + cy;
          const float wgt = EpfCutWeight(m64, cut, sad[j]);
          ws[0][j] += tile[0][ir][col] * wgt;
          ws[1][j] += tile[1][ir][col] * wgt;
          ws[2][j] += tile[2][ir][col] * wgt;
          sw[j] += wgt;
        }
      }
    }
  }
  if (!inside) return;
  // The normalisation: an IEEE division in the FP32 form (the reference's
  // rounding); in the tensor-core forms one reciprocal per row (the weight
  // sum is in [1, 56]) and a multiply per channel, within 2 ulp.
  float inv[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) inv[j] = kFma ? __frcp_rn(sw[j]) : 0.f;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float v = kFma ? ws[c][j] * inv[j] : ws[c][j] / sw[j];
      EpfStore(out, dco, plane, w, c, px, py0 + j,
               filtered ? v : tile[c][tr0 + j][tc0]);
    }
}

// Filters the staged tile at (x0, y0) into `out` (or, for the DC image,
// into dco's clamp), with every thread of the CTA: the guide, then the
// filter. The tile's copies are complete in every thread (the first
// barrier below publishes them); `sig` is EpfLaneSigma of this thread;
// (amin, mul) quantise the guide (GuideParams). `sa` holds the aligned
// guide words while the guide is built.
//
// kFma: the weighted sums with fused multiply-adds (the tensor-core forms,
// which are not bound to the reference's rounding); otherwise every product
// and sum is rounded separately, as the reference does.
template <bool kFma, int TH>
__device__ __forceinline__ void EpfFilterTile(
    const float* guide_src, const uint8_t* guide_ovr, int gab, int w, int h,
    float amin, float mul, int sig, float* out, const EpfDc& dco,
    uint32_t* sg, uint32_t* sa, float (*tile)[TH + 10][kEpfTS], int x0,
    int y0) {
  const int tid = threadIdx.x;
  // Tiles without filtered blocks are copies (CopyOriginalBlock).
  if (!__syncthreads_or(sig >= kMinSigma)) {
    const int lane = tid & 31, wp = tid >> 5;
    const int band = wp >> 1, col0 = 32 * (wp & 1);
    const size_t plane = size_t(w) * h;
    const int px = x0 + lane + col0, py0 = y0 + 4 * band;
    const int tr0 = 4 * band + 3 + kEpfTRow0;
    const int tc0 = lane + col0 + 3 + kEpfTCol0;
    if (px < w && py0 < h) {
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int j = 0; j < 4; ++j)
          EpfStore(out, dco, plane, w, c, px, py0 + j, tile[c][tr0 + j][tc0]);
    }
    return;
  }
  EpfBuildGuide<TH, 16 * TH>(tid, [] { __syncthreads(); }, guide_src,
                             guide_ovr, gab, w, h, amin, mul, sg, sa, tile,
                             x0, y0);
  EpfFilterCore<kFma, TH>(tid, sig, out, dco, w, h, sg, tile, x0, y0);
}

// One CTA per 64 x TH tile (1-D grid, row-major tile order). More CTAs
// than resident slots balance the uneven tiles (copies, border tiles)
// better than CTAs that loop over tiles.
//
// Interior tiles are staged by the Tensor Memory Accelerator when `tmap`
// is valid (use_tma): one thread issues a 3-D tiled bulk copy
// (cp.async.bulk.tensor, a tensor map over this GPU's input planes, no
// multicast) of the tile's rows y0 - 5 .. y0 + TH + 4, columns
// x0 - 12 .. x0 + 75 of the three planes, straight into `tile` (whose
// layout is the copy's box), completing on an mbarrier with the byte count.
// The innermost coordinate x0 - 12 is a multiple of 4 floats (x0 is a
// multiple of 64), as the copy requires. The wait is bounded (`polls`, the
// context's PIKGPU_OPT_TC_WAIT_POLLS): if it runs out, the kernel sets
// *err = 2 (the host reports the frame as failed) and waits once more,
// bounded, so that no copy is in flight when the CTA exits. Border tiles, and all tiles without a tensor map, are staged with
// cp.async (EpfStage).
template <bool kFma, int TH>
__global__ void __launch_bounds__(16 * TH, TH == 16 ? 3 : 2)
    k_epf_box(const float* in, const float* guide_src,
              const uint8_t* guide_ovr, int gab, int w, int h,
              const uint32_t* mm, EpfSigma sgs, float* out, EpfDc dco,
              const __grid_constant__ CUtensorMap tmap, int use_tma,
              int* err, uint32_t polls) {
  extern __shared__ __align__(128) uint32_t epf_smem[];
  uint32_t* sg = epf_smem;  // [3][TH + 8][kEpfGRow]
  auto* tile = reinterpret_cast<float(*)[TH + 10][kEpfTS]>(
      epf_smem + 3 * (TH + 8) * kEpfGRow);
  uint32_t* sa = epf_smem + 3 * (TH + 8) * kEpfGRow + 3 * (TH + 10) * kEpfTS;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sa + 3 * (TH + 8) * kEpfAligned);
  PdlLaunchDependents();  // the active-block pass may start on free SMs
  const int tiles_x = (w + kEpfW - 1) / kEpfW;
  const int x0 = (blockIdx.x % tiles_x) * kEpfW;
  const int y0 = (blockIdx.x / tiles_x) * TH;
  const uint32_t tile_s = tc::SmemU32(tile), mbar_s = tc::SmemU32(mbar);
  const bool tma = use_tma && EpfInterior<TH>(w, h, x0, y0) &&
                   (tile_s & 127u) == 0;
  if (tma) {
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_s)
                   : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      asm volatile(
          "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
              mbar_s),
          "r"(EpfTileBytes(TH))
          : "memory");
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::"
          "complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(tile_s),
          "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(x0 - 12), "r"(y0 - 5),
          "r"(0), "r"(mbar_s)
          : "memory");
    }
  } else {
    EpfStage<TH>(in, w, h, x0, y0, tile, threadIdx.x);
  }
  // The input is complete before the min/max pass starts; the guide range
  // in `mm` is that pass's output (the previous kernel on the stream, under
  // a programmatic dependent launch still running until here).
  PdlWait();
  float amin, mul, stretch;
  GuideParams(mm, &amin, &mul, &stretch);
  const int sig = EpfLaneSigma(sgs, stretch, w, h, x0, y0);
  if (tma) {
    __syncthreads();  // the mbarrier is initialised before anyone waits
    // (tc::WaitMma is the bounded mbarrier wait of the tensor-core kernels)
    if (!tc::WaitMma(mbar_s, 0, polls) && threadIdx.x == 0) {
      atomicExch(err, 2);
    }
  } else {
    CpAsyncWaitAll();
  }
  EpfFilterTile<kFma, TH>(guide_src, guide_ovr, gab, w, h, amin, mul, sig,
                          out, dco, sg, sa, tile, x0, y0);
}

}  // namespace pikgpu
