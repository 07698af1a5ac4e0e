// Edge-preserving filter (AdaptiveFilter + WeightedSum,
// pik/epf_target.cc:526-801, 1113-1278) with packed-byte box sums.
//
// One CTA filters a 64 x 32 pixel tile; each thread owns a 4 x 2 pixel
// micro-tile (inside one 8 x 8 block, so sigma is uniform per thread). For
// every displacement (cy, cx) of the 7 x 8 neighbourhood and every channel,
// the 3 x 4 patch SADs of the micro-tile's 16 pixels are formed from packed
// u8 guide words: byte-wise |ref - window| (__vabsdiffu4) over the 7
// columns x-1 .. x+5 of the four patch rows, horizontal 4-sums by __dp4a on
// funnel-shifted words, then vertical 3-sums. The SADs are exact integers;
// weights and the weighted sums follow the reference's neighbour order
// (cy = -3..3, cx = -3..4) with separately rounded products and sums, so
// the output equals the per-pixel formulation bit for bit.
// Included by recon_kernels.cu.
#pragma once

namespace pikgpu {

constexpr int kEpfW = 64, kEpfH = 32;      // output tile
constexpr int kEpfGW = kEpfW + 16;         // guide bytes: x0 - 8 .. x0 + 71
constexpr int kEpfGWords = kEpfGW / 4;     // 20 words per guide row
constexpr int kEpfGH = kEpfH + 8;          // guide rows: y0 - 4 .. y0 + 35
constexpr int kEpfIW = kEpfW + 8;          // in cols: x0 - 3 .. x0 + 68
constexpr int kEpfIH = kEpfH + 6;          // in rows: y0 - 3 .. y0 + 34
constexpr int kEpfMH = 2;                  // micro-tile rows
constexpr int kEpfThreads = 16 * (kEpfH / kEpfMH);

__device__ __forceinline__ uint32_t Shr8(uint32_t lo, uint32_t hi, int sh) {
  // Bytes sh .. sh+3 of the 8-byte little-endian pair (hi:lo).
  return sh == 0 ? lo : __funnelshift_r(lo, hi, 8 * sh);
}

__global__ void __launch_bounds__(kEpfThreads)
    k_epf_box(const float* in, const float* guide_src,
              const uint8_t* guide_ovr, int w, int h, const uint32_t* mm,
              const int32_t* sigma, float* out) {
  // One spare word per row: the last window read may touch it (unused).
  __shared__ uint32_t sg[3][kEpfGH][kEpfGWords + 1];
  __shared__ float si[3][kEpfIH][kEpfIW];
  const int x0 = blockIdx.x * kEpfW, y0 = blockIdx.y * kEpfH;
  const int tid = threadIdx.x;
  const size_t plane = size_t(w) * h;
  const int bw = w / 8;
  const int tx = tid & 15, ty = tid >> 4;  // micro-tile column / row
  const int px = x0 + 4 * tx, py = y0 + kEpfMH * ty;
  const bool inside = px < w && py < h;
  const int sig = inside ? sigma[(py >> 3) * bw + (px >> 3)] : 0;
  const bool filtered = sig >= kMinSigma;

  // Tiles without filtered blocks are copies (CopyOriginalBlock).
  if (!__syncthreads_or(filtered)) {
    if (inside) {
      for (int c = 0; c < 3; ++c) {
        for (int j = 0; j < kEpfMH; ++j) {
          const size_t o = c * plane + size_t(py + j) * w + px;
          *reinterpret_cast<float4*>(out + o) =
              *reinterpret_cast<const float4*>(in + o);
        }
      }
    }
    return;
  }

  float amin, mul, stretch;
  GuideParams(mm, &amin, &mul, &stretch);
  // u8 guide (MakeGuide, pik/epf_target.cc:1009-1070), 4 bytes per word.
  for (int i = tid; i < 3 * kEpfGH * kEpfGWords; i += kEpfThreads) {
    const int c = i / (kEpfGH * kEpfGWords);
    const int r = (i / kEpfGWords) % kEpfGH, wd = i % kEpfGWords;
    const int gy = y0 - 4 + r;
    uint32_t word = 0;
    for (int b = 0; b < 4; ++b) {
      const int gx = x0 - 8 + 4 * wd + b;
      uint32_t v;
      if (guide_ovr) {
        const bool ok = gx >= -6 && gx < w + 6 && gy >= -6 && gy < h + 6;
        v = ok ? guide_ovr[(size_t(c) * (h + 12) + gy + 6) * (w + 12) + gx + 6]
               : 0u;
      } else {
        const float s = guide_src[c * plane + size_t(MirrorIdx(gy, h)) * w +
                                  MirrorIdx(gx, w)];
        v = uint8_t(uint32_t(__float2int_rz((s - amin) * mul)));
      }
      word |= v << (8 * b);
    }
    sg[c][r][wd] = word;
  }
  for (int i = tid; i < 3 * kEpfIH * kEpfIW; i += kEpfThreads) {
    const int c = i / (kEpfIH * kEpfIW);
    const int r = (i / kEpfIW) % kEpfIH, col = i % kEpfIW;
    const int gx = x0 - 3 + col, gy = y0 - 3 + r;
    si[c][r][col] =
        in[c * plane + size_t(MirrorIdx(gy, h)) * w + MirrorIdx(gx, w)];
  }
  __syncthreads();

  // Warps (one block row of 8 blocks) without filtered blocks copy.
  if (!__any_sync(0xFFFFFFFFu, filtered)) {
    if (inside) {
      for (int c = 0; c < 3; ++c) {
        for (int j = 0; j < kEpfMH; ++j) {
          float* o = out + c * plane + size_t(py + j) * w + px;
          const float* s = &si[c][kEpfMH * ty + j + 3][4 * tx + 3];
          o[0] = s[0], o[1] = s[1], o[2] = s[2], o[3] = s[3];
        }
      }
    }
    return;
  }
  const int m = c_t.mul_table[filtered ? sig : kMinSigma];

  // Reference words: rows py-1 .. py+MH, bytes px-4 .. px+7 (words tx+1..3).
  constexpr int R = kEpfMH + 2, NP = 4 * kEpfMH;
  const int gr0 = kEpfMH * ty + 3;  // smem guide row of py - 1
  uint32_t ref[3][R][3];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int k = 0; k < 3; ++k) ref[c][r][k] = sg[c][gr0 + r][tx + 1 + k];

  float ws[3][NP], sw[NP];
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    ws[0][p] = ws[1][p] = ws[2][p] = 0.f;
    sw[p] = 0.f;
  }
#pragma unroll 1
  for (int cy = -3; cy <= 3; ++cy) {
#pragma unroll 2
    for (int cx = -3; cx <= 4; ++cx) {
      // Window byte offset of column px - 4 + cx from the row start.
      const int o = 4 * tx + 4 + cx;
      const int k = o >> 2;
      const int sh = (cx + 4) & 3;
      int sad[NP];
#pragma unroll
      for (int p = 0; p < NP; ++p) sad[p] = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        int hs[R][4];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const uint32_t* row = sg[c][gr0 + r + cy];
          const uint32_t w0 = row[k], w1 = row[k + 1], w2 = row[k + 2],
                         w3 = row[k + 3];
          const uint32_t da = __vabsdiffu4(ref[c][r][0], Shr8(w0, w1, sh));
          const uint32_t db = __vabsdiffu4(ref[c][r][1], Shr8(w1, w2, sh));
          const uint32_t dc = __vabsdiffu4(ref[c][r][2], Shr8(w2, w3, sh));
          hs[r][0] = (int)__dp4a((unsigned)__funnelshift_r(da, db, 24), 0x01010101u, 0u);
          hs[r][1] = (int)__dp4a((unsigned)db, 0x01010101u, 0u);
          hs[r][2] = (int)__dp4a((unsigned)__funnelshift_r(db, dc, 8), 0x01010101u, 0u);
          hs[r][3] = (int)__dp4a((unsigned)__funnelshift_r(db, dc, 16), 0x01010101u, 0u);
        }
#pragma unroll
        for (int j = 0; j < kEpfMH; ++j)
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int s = hs[j][i] + hs[j + 1][i] + hs[j + 2][i];
            sad[j * 4 + i] = max(sad[j * 4 + i], s);
          }
      }
#pragma unroll
      for (int j = 0; j < kEpfMH; ++j) {
        const int ir = kEpfMH * ty + j + 3 + cy;
        const float* i0 = &si[0][ir][4 * tx + 3 + cx];
        const float* i1 = &si[1][ir][4 * tx + 3 + cx];
        const float* i2 = &si[2][ir][4 * tx + 3 + cx];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int p = j * 4 + i;
          float wgt = WeightFast(m, sad[p]);
          if (!(wgt >= 0.05f)) wgt = 0.0f;
          ws[0][p] += i0[i] * wgt;
          ws[1][p] += i1[i] * wgt;
          ws[2][p] += i2[i] * wgt;
          sw[p] += wgt;
        }
      }
    }
  }
  if (!inside) return;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int j = 0; j < kEpfMH; ++j) {
      float v[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int p = j * 4 + i;
        v[i] = filtered ? ws[c][p] / sw[p]
                        : si[c][kEpfMH * ty + j + 3][4 * tx + 3 + i];
      }
      *reinterpret_cast<float4*>(out + c * plane + size_t(py + j) * w + px) =
          make_float4(v[0], v[1], v[2], v[3]);
    }
  }
}

}  // namespace pikgpu
