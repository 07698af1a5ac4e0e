// Adjoint of the reconstruction (pikgpu_adjoint): the gradient of
//   L = sum over the xsize x ysize pixels and X, Y, B of
//       (pre_opsin - target)^2
// with respect to the dequantised AC coefficients (the output of
// Dequant::DoAC, pik/compressed_image.cc:586-707, frame layout) and the
// per-cell quant field taken as a real number. pre_opsin is the frame after
// gaborish #2, before OpsinToLinear (pik/compressed_image.cc:1144-1181).
//
// The EPF's discrete decisions -- the u8 guide and the per-block sigma of
// MakeGuide / SigmaFromQuant (pik/epf_target.cc:1009-1111) -- are piecewise
// constant in every input, so they are held at their forward values (their
// derivative is zero almost everywhere). With them fixed the reconstruction
// is linear in the coefficients except for AdaptiveReconstruction's clamp
// (pik/adaptive_reconstruction.cc:72-244), whose ratio
// (interval / 2) / |correction| is differentiated where it is active. The
// quant field enters through the dequantisation (a cell's coefficients
// scale with 1 / qf) and the clamp intervals (half a step, also 1 / qf).
//
// The forward pass runs first (LaunchAll, keeping the dequantised AC, the
// EPF output and pre_opsin); the backward pass then transposes each stage:
//   k_adj_loss      2 (pre - target) on the padded frame, loss partials
//   k_adj_gab       gaborish #2 transposed (mirrored stencil, gathered)
//   k_adj_ar*       the clamp, per first block: DCT of (EPF - IDCT) again,
//                   the branch of every coefficient from the clamp tape the
//                   forward's clamp kernels wrote (which channel set the
//                   minimum ratio, or none, or a +0.0 correction), the
//                   gradients of the correction and of the quant field
//   k_adj_epf       the EPF with frozen weights: each filtered pixel's
//                   normalised weights scattered back to its (mirrored)
//                   neighbours through a shared-memory tile
//   k_adj_topix*    TransformToPixels transposed per first block, and for HF
//                   prediction TransformFromPixels transposed of the masked
//                   coefficient gradient (the upsampled prediction's
//                   gradient)
//   k_adj_upsample  UpSample4x4BlurDCT transposed into the group's pred2x2
//   k_adj_lf        DC2x2FromLowFrequencies transposed into each block's LF
//                   corner (pik/ac_predictions.cc:560-635); LLF gets zero
//                   (it is overwritten from DC)
//   k_adj_qf        the quant field: -sum(g * ac) / qf per cell
// Square DCT blocks of 16 and 32 use the separable transforms with
// transposed matrices; the 8x8 types use dense 64 x 64 Jacobians built on
// the device from the forward transforms applied to unit vectors
// (k_adj_build_jac). The backward arithmetic is FP32 (sums of the quant
// field gradient and the loss in FP64).
//
// Included by pikgpu.cu (single translation unit).

namespace pikgpu {
namespace {

constexpr int kJTypes = 5;  // DCT8, IDENTITY, DCT2X2, DCT4X4, LINES

__host__ __device__ inline int JIndex(int type) {
  switch (type) {
    case kDCT:
    case kDCT_NOHF:
      return 0;
    case kIDENTITY:
      return 1;
    case kDCT2X2:
      return 2;
    case kDCT4X4:
    case kDCT4X4_NOHF:
      return 3;
    case kLINES:
      return 4;
  }
  return -1;
}

struct AdjJac {
  float j0[kJTypes][64][64];   // TransformToPixels, [pixel][coefficient]
  float j1[kJTypes][64][64];   // TransformFromPixels, [coefficient][pixel]
  float j1t[kJTypes][64][64];  // j1 transposed, [pixel][coefficient]
  float j2[9][64][64];         // DC2x2 of the LF corner, [cell][LF input]
};

// TransformToPixels of an 8x8 type (AcStrategy::TransformToPixels,
// pik/ac_strategy.cc:741-849): coefficients and pixels 8x8 row-major.
__device__ void ToPixels8(int type, const float* co, float* px) {
  if (type == kDCT || type == kDCT_NOHF) {
    TsIdct1(8, co, 8, px, 8);
  } else if (type == kDCT4X4 || type == kDCT4X4_NOHF) {
    const float b00 = co[0], b01 = co[1], b10 = co[8], b11 = co[9];
    const float d[4] = {b00 + b01 + b10 + b11, b00 + b01 - b10 - b11,
                        b00 - b01 + b10 - b11, b00 - b01 - b10 + b11};
    for (int sy = 0; sy < 2; ++sy) {
      for (int sx = 0; sx < 2; ++sx) {
        float in4[16], out4[16];
        for (int iy = 0; iy < 4; ++iy)
          for (int ix = 0; ix < 4; ++ix)
            in4[iy * 4 + ix] = (iy == 0 && ix == 0)
                                   ? d[sy * 2 + sx]
                                   : co[(sy + iy * 2) * 8 + sx + ix * 2];
        TsIdct1(4, in4, 4, out4, 4);
        for (int py = 0; py < 4; ++py)
          for (int q = 0; q < 4; ++q)
            px[(sy * 4 + py) * 8 + sx * 4 + q] = out4[py * 4 + q];
      }
    }
  } else {
    SmallInverse(type, co, px, 8);
  }
}

// TransformFromPixels of an 8x8 type (pik/ac_strategy.cc:531-663).
__device__ void FromPixels8(int type, const float* px, float* co) {
  if (type == kDCT || type == kDCT_NOHF) {
    TsDct1(8, px, 8, co, 8);
  } else if (type == kDCT4X4 || type == kDCT4X4_NOHF) {
    for (int sy = 0; sy < 2; ++sy) {
      for (int sx = 0; sx < 2; ++sx) {
        float in4[16], r4[16];
        for (int py = 0; py < 4; ++py)
          for (int q = 0; q < 4; ++q)
            in4[py * 4 + q] = px[(sy * 4 + py) * 8 + sx * 4 + q];
        TsDct1(4, in4, 4, r4, 4);
        for (int iy = 0; iy < 4; ++iy)
          for (int ix = 0; ix < 4; ++ix)
            co[(sy + iy * 2) * 8 + sx + ix * 2] = r4[iy * 4 + ix];
      }
    }
    const float b00 = co[0], b01 = co[1], b10 = co[8], b11 = co[9];
    co[0] = (b00 + b01 + b10 + b11) * 0.25f;
    co[1] = (b00 + b01 - b10 - b11) * 0.25f;
    co[8] = (b00 - b01 + b10 - b11) * 0.25f;
    co[9] = (b00 - b01 - b10 + b11) * 0.25f;
  } else {
    SmallForward(type, px, 8, co);
  }
}

// Block 2 kJTypes + 9 CTAs of 64 threads; thread j builds column j.
__global__ void k_adj_build_jac(AdjJac* J) {
  const int which = blockIdx.x, j = threadIdx.x;
  const int kTypes[kJTypes] = {kDCT, kIDENTITY, kDCT2X2, kDCT4X4, kLINES};
  float in[64], out[64];
  for (int i = 0; i < 64; ++i) {
    in[i] = i == j ? 1.0f : 0.0f;
    out[i] = 0.0f;
  }
  if (which < kJTypes) {
    ToPixels8(kTypes[which], in, out);
    for (int r = 0; r < 64; ++r) J->j0[which][r][j] = out[r];
  } else if (which < 2 * kJTypes) {
    const int t = which - kJTypes;
    FromPixels8(kTypes[t], in, out);
    for (int r = 0; r < 64; ++r) {
      J->j1[t][r][j] = out[r];
      J->j1t[t][j][r] = out[r];
    }
  } else {
    const int type = which - 2 * kJTypes;
    const int cov = Covered(type), n = 8 * cov, m = 2 * cov;
    if (j < m * m) {
      const int idx = (j / m) * n + j % m;
      DC2x2FromLowFreq(type, [&](int i) { return i == idx ? 1.0f : 0.0f; },
                       out, m);
    }
    for (int r = 0; r < 64; ++r) {
      J->j2[type][r][j] = (j < m * m && r < m * m) ? out[r] : 0.0f;
    }
  }
}

constexpr int kAdjLossBlocks = 592, kAdjThreads = 256;

// g_pre = 2 (pre - target) inside xsize x ysize, 0 in the padding; the loss
// partial sums of each CTA in FP64.
__global__ void __launch_bounds__(kAdjThreads)
    k_adj_loss(const float* pre, const float* target, int w, int h, int pw,
               int ph, float* g_pre, double* partial) {
  __shared__ double s_sum[kAdjThreads / 32];
  const size_t plane = size_t(pw) * ph, n = 3 * plane;
  double acc = 0.0;
  for (size_t i = blockIdx.x * size_t(kAdjThreads) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * kAdjThreads) {
    const int c = int(i / plane);
    const size_t rem = i % plane;
    const int y = int(rem / pw), x = int(rem % pw);
    float gv = 0.0f;
    if (x < w && y < h) {
      const size_t o = (size_t(c) * h + y) * w + x;
      const double d = double(pre[o]) - double(target[o]);
      acc += d * d;
      gv = 2.0f * (pre[o] - target[o]);
    }
    g_pre[i] = gv;
  }
  for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(~0u, acc, off);
  if ((threadIdx.x & 31) == 0) s_sum[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < kAdjThreads / 32; ++i) t += s_sum[i];
    partial[blockIdx.x] = t;
  }
}

__global__ void k_adj_sum(const double* partial, int n, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double t = 0.0;
  for (int i = 0; i < n; ++i) t += partial[i];
  *out = t;
}

// Transpose of Symmetric3 with mirrored borders (the forward stencil is
// symmetric, so interior pixels gather with the same weights; border pixels
// collect every tap whose mirrored source is them).
__global__ void k_adj_gab(const float* gin, int pw, int ph, int strength,
                          float* gout) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int c = blockIdx.z;
  if (x >= pw || y >= ph) return;
  const float* wt = c_t.gaborish[strength];
  const float* p = gin + size_t(c) * pw * ph;
  float s = 0.0f;
  if (x >= 1 && x + 1 < pw && y >= 1 && y + 1 < ph) {
    const float* t = p + size_t(y - 1) * pw + x;
    const float* m = p + size_t(y) * pw + x;
    const float* b = p + size_t(y + 1) * pw + x;
    s = m[0] * wt[0] + (t[0] + b[0] + m[-1] + m[1]) * wt[1] +
        (t[-1] + t[1] + b[-1] + b[1]) * wt[2];
  } else {
    for (int yy = max(y - 1, 0); yy <= min(y + 1, ph - 1); ++yy) {
      for (int dy = -1; dy <= 1; ++dy) {
        if (MirrorIdx(yy + dy, ph) != y) continue;
        for (int xx = max(x - 1, 0); xx <= min(x + 1, pw - 1); ++xx) {
          for (int dx = -1; dx <= 1; ++dx) {
            if (MirrorIdx(xx + dx, pw) != x) continue;
            const int k = abs(dx) + abs(dy);
            s += wt[k == 0 ? 0 : k == 1 ? 1 : 2] * p[size_t(yy) * pw + xx];
          }
        }
      }
    }
  }
  gout[size_t(c) * pw * ph + size_t(y) * pw + x] = s;
}

// Clamp backward of one coefficient, on the branch the forward took (its
// clamp tape code, ClampTapeCode). co: the correction per channel, iv: the
// interval, gs: the gradient of the scaled correction. Writes the
// correction gradient; for a clamped non-LLF coefficient adds the quant
// field's share to *gq: the ratio is (interval / 2) / |co| and
// d interval / d qf = -interval / qf.
__device__ __forceinline__ void ClampBackward(int code, const float co[3],
                                              const float iv[3],
                                              const float gs[3], bool llf,
                                              float qf_eff, float gc[3],
                                              float* gq) {
  const int arg = code >= 1 && code <= 3 ? code - 1 : -1;
  const float mr =
      arg >= 0 ? ClampRatio(co[arg], iv[arg]) : code == 0 ? 1.0f : 0.0f;
  float gmr = 0.0f;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    gmr += gs[c] * co[c];
    gc[c] = gs[c] * mr;
  }
  if (arg >= 0 && co[arg] != 0.0f) {
    gc[arg] += gmr * (-mr / co[arg]);
    if (!llf) *gq += -gmr * mr / qf_eff;
  }
}

__device__ __forceinline__ float QfEff(const Geo& g, const DevFrame& f,
                                       int bx, int by) {
  const int cell = by * g.Bx + bx;
  const float q = float(f.qf[cell]);
  return f.clamp_scale ? q / f.clamp_scale[cell] : q;
}

constexpr int kAdj8Blocks = 4;  // 8x8 blocks per CTA, 64 threads each

// Clamp backward of 8x8 blocks (all cov = 1 types) from the dense
// Jacobians. Blocks the EPF left unfiltered have EPF output == IDCT output,
// a zero correction and ratio 0: the gradient passes to the IDCT output.
__global__ void __launch_bounds__(kAdjThreads)
    k_adj_ar8(Geo g, DevFrame f, FrameScalars s, const AdjJac* J,
              const uint32_t* list, int count, const int32_t* sigma,
              const uint8_t* tape, const float* epf, const float* g_cur,
              float* g_filt, float* g_idct, float* g_qf) {
  __shared__ float s_a[kAdj8Blocks][3][64];  // diff, then g_corr
  __shared__ float s_o[kAdj8Blocks][3][64];  // gradient of the output
  __shared__ float s_q[kAdj8Blocks][2];
  const int lb = threadIdx.x >> 6, e = threadIdx.x & 63;
  const int item = blockIdx.x * kAdj8Blocks + lb;
  const bool valid = item < count;
  int bx = 0, by = 0, type = 0;
  bool active = false;
  if (valid) {
    const uint32_t pk = list[item];
    bx = pk & 0xFFFF;
    by = pk >> 16;
    type = f.acs[by * g.Bx + bx] >> 4;
    active = sigma[by * g.Bx + bx] >= kMinSigma;
  }
  const size_t plane = size_t(g.PW) * g.PH;
  const size_t o = size_t(by * 8 + e / 8) * g.PW + bx * 8 + e % 8;
  if (valid) {
    for (int c = 0; c < 3; ++c) {
      s_o[lb][c][e] = g_cur[c * plane + o];
      s_a[lb][c][e] =
          active ? epf[c * plane + o] - f.idct[c * plane + o] : 0.0f;
    }
  }
  __syncthreads();
  const int t = JIndex(type);
  float gq = 0.0f, gc[3] = {0.0f, 0.0f, 0.0f};
  if (valid && active) {
    float co[3], gs[3], iv[3];
    for (int c = 0; c < 3; ++c) {
      float a = 0.0f, b = 0.0f;
      for (int p = 0; p < 64; ++p) {
        a += J->j1t[t][p][e] * s_a[lb][c][p];
        b += J->j0[t][p][e] * s_o[lb][c][p];
      }
      co[c] = a;
      gs[c] = b;
    }
    const ArBlockInfo info = ArInfo(g, f, s, bx, by, type);
    for (int c = 0; c < 3; ++c) {
      iv[c] = e == 0 ? 1.0f * s.mul_dc[c] : info.dm[c][e] * info.inv_quant_ac;
    }
    ClampBackward(tape[CoefOffset(g, bx, by, 1, e)], co, iv, gs, e == 0,
                  QfEff(g, f, bx, by), gc, &gq);
  }
  __syncthreads();
  if (valid && active) {
    for (int c = 0; c < 3; ++c) s_a[lb][c][e] = gc[c];
  }
  for (int off = 16; off; off >>= 1) gq += __shfl_xor_sync(~0u, gq, off);
  if ((threadIdx.x & 31) == 0) s_q[lb][(threadIdx.x >> 5) & 1] = gq;
  __syncthreads();
  if (!valid) return;
  if (e == 0 && active) g_qf[by * g.Bx + bx] = s_q[lb][0] + s_q[lb][1];
  for (int c = 0; c < 3; ++c) {
    float gd = 0.0f;
    if (active) {
      for (int k = 0; k < 64; ++k) gd += J->j1[t][k][e] * s_a[lb][c][k];
    }
    g_filt[c * plane + o] = gd;
    g_idct[c * plane + o] = s_o[lb][c][e] - gd;
  }
}

// Square-DCT matrices staged in shared memory for the transposed-matrix
// transforms (CoopTsIdctT / CoopTsDctT, which take M^T to apply M): `a` =
// A (applies A^T, the transpose of the IDCT), `b` = B (applies B^T, the
// transpose of the scaled DCT), `bt` = B^T (applies B, the DCT).
template <int N>
__device__ __forceinline__ void StageMatrices(float* a, float* b, float* bt) {
  for (int i = threadIdx.x; i < N * N; i += blockDim.x) {
    const int r = i / N, c = i % N;
    a[i] = IdctMat(N)[i];
    b[i] = DctMat(N)[i];
    if (bt) bt[i] = DctMat(N)[c * N + r];
  }
}

// Clamp backward of one DCT16 / DCT32 block per CTA (separable transforms:
// the transpose of the IDCT is the IDCT routine with A^T, that of the
// scaled DCT the DCT routine with B^T).
template <int N>
__global__ void __launch_bounds__(kAdjThreads)
    k_adj_ar_sq(Geo g, DevFrame f, FrameScalars s, const uint32_t* list,
                int count, const int32_t* sigma, const uint8_t* tape,
                const float* epf, const float* g_cur, float* g_filt,
                float* g_idct, float* g_qf) {
  constexpr int NN = N * N, cov = N / 8;
  __shared__ float s_b[NN], s_a[NN], s_bt[NN];
  __shared__ float s_co[3][NN], s_g[3][NN], s_t[NN];
  __shared__ float s_q[kAdjThreads / 32];
  const int item = blockIdx.x;
  if (item >= count) return;
  const uint32_t pk = list[item];
  const int bx = pk & 0xFFFF, by = pk >> 16;
  const int type = f.acs[by * g.Bx + bx] >> 4;
  bool active = false;
  for (int y = 0; y < cov; ++y)
    for (int x = 0; x < cov; ++x)
      active |= sigma[(by + y) * g.Bx + bx + x] >= kMinSigma;
  const size_t plane = size_t(g.PW) * g.PH;
  auto pix = [&](int c, int e) {
    return c * plane + size_t(by * 8 + e / N) * g.PW + bx * 8 + e % N;
  };
  if (!active) {  // CTA-uniform
    for (int i = threadIdx.x; i < 3 * NN; i += blockDim.x) {
      const size_t o = pix(i / NN, i % NN);
      g_idct[o] = g_cur[o];
      g_filt[o] = 0.0f;
    }
    return;
  }
  StageMatrices<N>(s_a, s_b, s_bt);
  for (int i = threadIdx.x; i < 3 * NN; i += blockDim.x) {
    const int c = i / NN, e = i % NN;
    const size_t o = pix(c, e);
    s_co[c][e] = epf[o] - f.idct[o];
    s_g[c][e] = g_cur[o];
  }
  __syncthreads();
  for (int c = 0; c < 3; ++c) {
    CoopTsDctT(N, 1, s_bt, s_co[c], s_t, s_co[c]);   // B
    CoopTsIdctT(N, 1, s_a, s_g[c], s_t, s_g[c]);    // A^T
  }
  const ArBlockInfo info = ArInfo(g, f, s, bx, by, type);
  const float qf_eff = QfEff(g, f, bx, by);
  float gq = 0.0f;
  for (int e = threadIdx.x; e < NN; e += blockDim.x) {
    const int y = e / N, x = e % N;
    const bool llf = y < cov && x < cov;
    float co[3], gs[3], iv[3], gc[3];
    for (int c = 0; c < 3; ++c) {
      co[c] = s_co[c][e];
      gs[c] = s_g[c][e];
      iv[c] = llf ? LlfScale(type, x, y) * s.mul_dc[c]
                  : info.dm[c][e] * info.inv_quant_ac;
    }
    ClampBackward(tape[CoefOffset(g, bx, by, cov, e)], co, iv, gs, llf,
                  qf_eff, gc, &gq);
    for (int c = 0; c < 3; ++c) s_g[c][e] = gc[c];
  }
  __syncthreads();
  for (int c = 0; c < 3; ++c) {
    CoopTsDctT(N, 1, s_b, s_g[c], s_t, s_g[c]);  // B^T
  }
  for (int i = threadIdx.x; i < 3 * NN; i += blockDim.x) {
    const int c = i / NN, e = i % NN;
    const size_t o = pix(c, e);
    const float gd = s_g[c][e];
    g_filt[o] = gd;
    g_idct[o] = g_cur[o] - gd;
  }
  for (int off = 16; off; off >>= 1) gq += __shfl_xor_sync(~0u, gq, off);
  if ((threadIdx.x & 31) == 0) s_q[threadIdx.x >> 5] = gq;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int i = 0; i < kAdjThreads / 32; ++i) t += s_q[i];
    g_qf[by * g.Bx + bx] = t;
  }
}

// EPF with frozen weights, transposed. The forward pass computes, for a
// filtered pixel p, out(p) = sum_d w(p, d) in(p + d) / sum_d w(p, d) over
// the 7 x 8 window d = (cx, cy), cx in [-3, 4], cy in [-3, 3], where
// w(p, d) = W(mul(p), SAD(p, p + d)) and in() is mirrored at the frame
// border. Its transpose sends g(p) w(p, d) / sum_w(p) to p + d. The patch
// SAD is symmetric, SAD(p, p + d) = SAD(q, q - d) for q = p + d, so the
// transpose is a gather at q over the mirrored window e = -d
// (cx in [-4, 3]) with the weight of the sending pixel p = q + e:
//   pass 1 (k_adj_epf_pass<false>): gv(p) = g(p) / sum_w(p) for filtered
//          pixels, 0 for copied ones;
//   pass 2 (k_adj_epf_pass<true>):  g_idct(q) += sum_e gv(q + e)
//          W(mul(q + e), SAD(q, q + e)) (+ g(q) itself where q was copied),
//          for q + e inside the frame;
//   pass 3 (k_adj_epf_border): the terms whose target p + d lies outside
//          the frame (p within 4 pixels of the border), scattered to the
//          mirrored position.
// Passes 1 and 2 follow the forward kernel's design (k_epf_box): 64 x 32
// tiles, one column of four rows per lane, the u8 guide staged as one
// 32-bit word per byte offset and patch SADs by __vsadu4, summed vertically
// across the lane's rows.
constexpr int kAdjEpfTH = kEpfH + 6;   // gather tile rows y0 - 3 .. y0 + 34
constexpr int kAdjEpfTW = kEpfW + 8;   // gather tile cols x0 - 4 .. x0 + 67
constexpr size_t kAdjEpfSmemBytes =
    kEpfGuideWords * 4 + size_t(3) * kAdjEpfTH * kAdjEpfTW * 4;

template <bool kGather>
__global__ void __launch_bounds__(kEpfThreads, 2)
    k_adj_epf_pass(int w, int h, const uint8_t* guide, const int32_t* sigma,
                   const float* g_filt, const float* gv_in, float* out) {
  extern __shared__ __align__(16) uint32_t adj_epf_smem[];
  uint32_t* sg = adj_epf_smem;  // [3][kEpfGH][kEpfGRow]
  float(*tile)[kAdjEpfTH][kAdjEpfTW] =
      reinterpret_cast<float(*)[kAdjEpfTH][kAdjEpfTW]>(adj_epf_smem +
                                                       kEpfGuideWords);
  __shared__ int s_m64[6][10];  // mul * 64 of blocks y0/8-1.., x0/8-1..
  const int x0 = blockIdx.x * kEpfW, y0 = blockIdx.y * kEpfH;
  const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  const int band = wp >> 1, col0 = 32 * (wp & 1);
  const size_t plane = size_t(w) * h;
  const int bw = w / 8, bh = h / 8;
  const int px = x0 + lane + col0, py0 = y0 + 4 * band;
  const bool inside = px < w && py0 < h;
  const int sig = inside ? sigma[(py0 >> 3) * bw + (px >> 3)] : 0;
  const bool filtered = sig >= kMinSigma;
  // The u8 guide (6-pixel mirrored border) as words: bytes x0 - 8 ..
  // x0 + 71 of rows y0 - 4 .. y0 + 35; bytes outside the buffer read 0.
  const int gwid = w + 12, ght = h + 12;
  constexpr int kAligned = kEpfGBytes / 4;
  for (int i = tid; i < 3 * kEpfGH * kAligned; i += kEpfThreads) {
    const int c = i / (kEpfGH * kAligned);
    const int r = (i / kAligned) % kEpfGH, wd = i % kAligned;
    const int gy = y0 - 4 + r;
    uint32_t word = 0;
    for (int b = 0; b < 4; ++b) {
      const int gx = x0 - 8 + 4 * wd + b;
      const bool ok = gx >= -6 && gx < w + 6 && gy >= -6 && gy < h + 6;
      const uint32_t v =
          ok ? guide[(size_t(c) * ght + gy + 6) * gwid + gx + 6] : 0u;
      word |= v << (8 * b);
    }
    sg[c * kEpfGPlane + r * kEpfGRow + 4 * wd] = word;
  }
  if (kGather) {
    // gv around the tile, 0 outside the frame (those terms are pass 3's).
    for (int i = tid; i < 3 * kAdjEpfTH * kAdjEpfTW; i += kEpfThreads) {
      const int c = i / (kAdjEpfTH * kAdjEpfTW);
      const int r = (i / kAdjEpfTW) % kAdjEpfTH, col = i % kAdjEpfTW;
      const int gx = x0 - 4 + col, gy = y0 - 3 + r;
      tile[c][r][col] = (gx >= 0 && gx < w && gy >= 0 && gy < h)
                            ? gv_in[c * plane + size_t(gy) * w + gx]
                            : 0.0f;
    }
    for (int i = tid; i < 60; i += kEpfThreads) {
      const int by = y0 / 8 - 1 + i / 10, bx = x0 / 8 - 1 + i % 10;
      int m = 0;
      if (by >= 0 && by < bh && bx >= 0 && bx < bw) {
        const int sg_ = sigma[by * bw + bx];
        m = sg_ >= kMinSigma ? c_t.mul_table[sg_] * 64 : 0;
      }
      s_m64[i / 10][i % 10] = m;
    }
  }
  __syncthreads();
  for (int i = tid; i < 3 * kEpfGH * kAligned * 3; i += kEpfThreads) {
    const int sft = 1 + i % 3;
    const int j = i / 3;
    const int c = j / (kEpfGH * kAligned);
    const int r = (j / kAligned) % kEpfGH, wd = j % kAligned;
    const uint32_t* row = sg + c * kEpfGPlane + r * kEpfGRow;
    const uint32_t lo = row[4 * wd];
    const uint32_t hi = wd + 1 < kAligned ? row[4 * wd + 4] : 0u;
    sg[c * kEpfGPlane + r * kEpfGRow + 4 * wd + sft] =
        __funnelshift_r(lo, hi, 8 * sft);
  }
  __syncthreads();
  if (!inside) return;  // no barrier follows
  if (!kGather && !filtered) {
    for (int c = 0; c < 3; ++c)
      for (int j = 0; j < 4; ++j)
        out[c * plane + size_t(py0 + j) * w + px] = 0.0f;
    return;
  }
  const int gr0 = 4 * band + 3;  // guide smem row of py0 - 1
  uint32_t ref[3][6];
  {
    const uint32_t* g = sg + gr0 * kEpfGRow + lane + col0 + 7;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int r = 0; r < 6; ++r) ref[c][r] = g[c * kEpfGPlane + r * kEpfGRow];
  }
  const int m64c = filtered ? c_t.mul_table[sig] * 64 : 0;
  float acc[3][4], sw[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    acc[0][j] = acc[1][j] = acc[2][j] = 0.f;
    sw[j] = 0.f;
  }
  constexpr int kCx0 = kGather ? -4 : -3;
#pragma unroll 1
  for (int cy = -3; cy <= 3; ++cy) {
#pragma unroll 1
    for (int cx = kCx0; cx <= kCx0 + 7; ++cx) {
      const uint32_t* g = sg + (gr0 + cy) * kEpfGRow + lane + col0 + 7 + cx;
      int sad[4] = {0, 0, 0, 0};
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        int hs[6];
#pragma unroll
        for (int r = 0; r < 6; ++r) {
          hs[r] = int(__vsadu4(ref[c][r], g[c * kEpfGPlane + r * kEpfGRow]));
        }
        const int p12 = hs[1] + hs[2], p34 = hs[3] + hs[4];
        sad[0] = max(sad[0], hs[0] + p12);
        sad[1] = max(sad[1], p12 + hs[3]);
        sad[2] = max(sad[2], hs[2] + p34);
        sad[3] = max(sad[3], p34 + hs[5]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (kGather) {
          // The sending pixel q + e and its block's weight multiplier.
          const int sy = py0 + j + cy, sx = px + cx;
          const int m = s_m64[(sy >> 3) - y0 / 8 + 1][(sx >> 3) - x0 / 8 + 1];
          float wgt = EpfWeight(m, sad[j]);
          if (!(wgt >= 0.05f) || m == 0) wgt = 0.0f;
          const int tr = 4 * band + j + 3 + cy, tc = lane + col0 + 4 + cx;
          acc[0][j] = fmaf(tile[0][tr][tc], wgt, acc[0][j]);
          acc[1][j] = fmaf(tile[1][tr][tc], wgt, acc[1][j]);
          acc[2][j] = fmaf(tile[2][tr][tc], wgt, acc[2][j]);
        } else {
          float wgt = EpfWeight(m64c, sad[j]);
          if (!(wgt >= 0.05f)) wgt = 0.0f;
          sw[j] += wgt;
        }
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const size_t o = c * plane + size_t(py0 + j) * w + px;
      if (kGather) {
        out[o] += acc[c][j] + (filtered ? 0.0f : g_filt[o]);
      } else {
        out[o] = g_filt[o] / sw[j];
      }
    }
}

// Pass 3: the EPF terms that the forward mirrored back into the frame
// (p + d outside it), scattered from the 4-pixel border band.
__global__ void k_adj_epf_border(int w, int h, const uint8_t* guide,
                                 const int32_t* sigma, const float* gv,
                                 float* g_idct) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  if (x >= 3 && x < w - 4 && y >= 3 && y < h - 3) return;  // interior
  const int sg = sigma[(y >> 3) * (w / 8) + (x >> 3)];
  if (sg < kMinSigma) return;
  const size_t plane = size_t(w) * h;
  const int gwid = w + 12, ght = h + 12;
  const int m64 = c_t.mul_table[sg] * 64;
  auto gb = [&](int c, int yy, int xx) {
    return int(guide[(size_t(c) * ght + yy + 6) * gwid + xx + 6]);
  };
  float gvp[3];
  for (int c = 0; c < 3; ++c) gvp[c] = gv[c * plane + size_t(y) * w + x];
  for (int cy = -3; cy <= 3; ++cy) {
    for (int cx = -3; cx <= 4; ++cx) {
      const int tx = x + cx, ty = y + cy;
      if (tx >= 0 && tx < w && ty >= 0 && ty < h) continue;  // gathered
      int sad_max = 0;
      for (int c = 0; c < 3; ++c) {
        int sad = 0;
        for (int py = -1; py <= 1; ++py)
          for (int q = -1; q <= 2; ++q)
            sad += abs(gb(c, y + py, x + q) - gb(c, ty + py, tx + q));
        sad_max = max(sad_max, sad);
      }
      float wgt = EpfWeight(m64, sad_max);
      if (!(wgt >= 0.05f)) continue;
      const size_t o = size_t(MirrorIdx(ty, h)) * w + MirrorIdx(tx, w);
      for (int c = 0; c < 3; ++c) atomicAdd(&g_idct[c * plane + o], gvp[c] * wgt);
    }
  }
}

// TransformToPixels transposed for 8x8 blocks; for HF-predicting types the
// masked coefficient gradient (all but 0, 1, 8, 9) through
// TransformFromPixels transposed into the upsampled-prediction gradient.
__global__ void __launch_bounds__(kAdjThreads)
    k_adj_topix8(Geo g, DevFrame f, const AdjJac* J, const uint32_t* list,
                 int count, int predict_hf, const float* g_idct,
                 float* g_coef, float* g_up) {
  __shared__ float s_p[kAdj8Blocks][3][64], s_m[kAdj8Blocks][3][64];
  const int lb = threadIdx.x >> 6, e = threadIdx.x & 63;
  const int item = blockIdx.x * kAdj8Blocks + lb;
  const bool valid = item < count;
  int bx = 0, by = 0, type = 0;
  if (valid) {
    const uint32_t pk = list[item];
    bx = pk & 0xFFFF;
    by = pk >> 16;
    type = f.acs[by * g.Bx + bx] >> 4;
  }
  const size_t plane = size_t(g.PW) * g.PH;
  const size_t plane_ac = size_t(g.ac_stride) * g.By;
  const size_t o = size_t(by * 8 + e / 8) * g.PW + bx * 8 + e % 8;
  if (valid) {
    for (int c = 0; c < 3; ++c) s_p[lb][c][e] = g_idct[c * plane + o];
  }
  __syncthreads();
  const int t = JIndex(type);
  const bool masked = e == 0 || e == 1 || e == 8 || e == 9;
  if (valid) {
    for (int c = 0; c < 3; ++c) {
      float gc = 0.0f;
      for (int p = 0; p < 64; ++p) gc += J->j0[t][p][e] * s_p[lb][c][p];
      g_coef[c * plane_ac + size_t(by) * g.ac_stride + bx * 64 + e] = gc;
      s_m[lb][c][e] = masked ? 0.0f : gc;
    }
  }
  __syncthreads();
  if (!valid || !predict_hf || !PredictHFOf(type)) return;
  for (int c = 0; c < 3; ++c) {
    float gp = 0.0f;
    for (int k = 0; k < 64; ++k) gp += J->j1[t][k][e] * s_m[lb][c][k];
    g_up[c * plane + o] = gp;
  }
}

template <int N>
__global__ void __launch_bounds__(kAdjThreads)
    k_adj_topix_sq(Geo g, DevFrame f, const uint32_t* list, int count,
                   int predict_hf, const float* g_idct, float* g_coef,
                   float* g_up) {
  constexpr int NN = N * N, cov = N / 8, chunk = 64 * cov;
  __shared__ float s_a[NN], s_b[NN], s_x[NN], s_t[NN];
  const int item = blockIdx.x;
  if (item >= count) return;
  const uint32_t pk = list[item];
  const int bx = pk & 0xFFFF, by = pk >> 16;
  const size_t plane = size_t(g.PW) * g.PH;
  const size_t plane_ac = size_t(g.ac_stride) * g.By;
  StageMatrices<N>(s_a, s_b, nullptr);
  for (int c = 0; c < 3; ++c) {
    for (int e = threadIdx.x; e < NN; e += blockDim.x) {
      s_x[e] = g_idct[c * plane + size_t(by * 8 + e / N) * g.PW + bx * 8 +
                      e % N];
    }
    __syncthreads();
    CoopTsIdctT(N, 1, s_a, s_x, s_t, s_x);  // A^T
    float* base = g_coef + c * plane_ac + size_t(by) * g.ac_stride +
                  size_t(bx) * 64;
    for (int e = threadIdx.x; e < NN; e += blockDim.x) {
      base[(e / chunk) * size_t(g.ac_stride) + e % chunk] = s_x[e];
      if (e / N < 2 * cov && e % N < 2 * cov) s_x[e] = 0.0f;
    }
    __syncthreads();
    if (!predict_hf) continue;  // CTA-uniform
    CoopTsDctT(N, 1, s_b, s_x, s_t, s_x);  // B^T
    for (int e = threadIdx.x; e < NN; e += blockDim.x) {
      g_up[c * plane + size_t(by * 8 + e / N) * g.PW + bx * 8 + e % N] =
          s_x[e];
    }
    __syncthreads();
  }
}

// UpSample4x4BlurDCT (pik/ac_predictions.cc:263-374) transposed: the
// gradient of each block-interior pred2x2 cell of a group gathered from the
// 12 x 12 upsampled pixels that read it.
__global__ void k_adj_upsample(Geo g, const float* g_up, float* g_pred) {
  const int gi = blockIdx.z / 3, c = blockIdx.z % 3;
  int x0, y0, gxs, gys;
  GroupDims(g, gi, &x0, &y0, &gxs, &gys);
  const int Q = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int R = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  if (Q >= 2 * gxs + 2 || R >= 2 * gys + 2) return;
  const float* up =
      g_up + size_t(c) * g.PW * g.PH + size_t(8 * y0) * g.PW + 8 * x0;
  float s = 0.0f;
  for (int j = 0; j < 3; ++j) {
    const int r = R - 1 - j;
    if (r < 0 || r >= 2 * gys) continue;
    for (int iy = 0; iy < 4; ++iy) {
      const float* row = up + size_t(4 * r + iy) * g.PW;
      float hsum = 0.0f;
      for (int i = 0; i < 3; ++i) {
        const int q = Q - 1 - i;
        if (q < 0 || q >= 2 * gxs) continue;
        for (int ix = 0; ix < 4; ++ix) {
          hsum += c_t.ub4[i][ix] * row[4 * q + ix];
        }
      }
      s += c_t.ub4[j][iy] * hsum;
    }
  }
  g_pred[gi * kG2GroupFloats + c * kG2 * kG2 + R * kG2 + Q] = s;
}

// Per first block and channel: DC2x2FromLowFrequencies transposed into the
// LF corner (HF prediction), then the LLF coefficients' gradient is zeroed
// (they are overwritten by values from DC).
__global__ void k_adj_lf(Geo g, DevFrame f, const AdjJac* J, int predict_hf,
                         const float* g_pred, float* g_coef) {
  const int bx = blockIdx.x * blockDim.x + threadIdx.x;
  const int by = blockIdx.y * blockDim.y + threadIdx.y;
  const int c = blockIdx.z;
  if (bx >= g.Bx || by >= g.By) return;
  const int a = f.acs[by * g.Bx + bx];
  if (a & 0xF) return;
  const int type = a >> 4, cov = Covered(type), n = 8 * cov, m = 2 * cov;
  const int chunk = 64 * cov;
  float* base = g_coef + c * size_t(g.ac_stride) * g.By +
                size_t(by) * g.ac_stride + size_t(bx) * 64;
  auto at = [&](int i) -> float& {
    return base[(i / chunk) * size_t(g.ac_stride) + i % chunk];
  };
  if (predict_hf) {
    const int gi = (by >> 6) * g.Gx + (bx >> 6);
    const int lbx = bx & 63, lby = by & 63;
    const float* gp = g_pred + gi * kG2GroupFloats + c * kG2 * kG2 +
                      2 * (lby + 1) * kG2 + 2 * (lbx + 1);
    float cell[64];
    for (int r = 0; r < m * m; ++r) cell[r] = gp[(r / m) * kG2 + r % m];
    for (int u = 0; u < m * m; ++u) {
      float sum = 0.0f;
      for (int r = 0; r < m * m; ++r) sum += J->j2[type][r][u] * cell[r];
      at((u / m) * n + u % m) += sum;
    }
  }
  for (int y = 0; y < cov; ++y)
    for (int x = 0; x < cov; ++x) at(y * n + x) = 0.0f;
}

// Quant field: every coefficient of a cell scales with 1 / qf, so
// d L / d qf += -sum(g * ac) / qf (FP64 sum).
__global__ void k_adj_qf(Geo g, DevFrame f, const float* ac0,
                         const float* g_coef, float* g_qf) {
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= g.Bx * g.By) return;
  const int bx = cell % g.Bx, by = cell / g.Bx;
  const size_t plane_ac = size_t(g.ac_stride) * g.By;
  const size_t o = size_t(by) * g.ac_stride + size_t(bx) * 64;
  double s = 0.0;
  for (int c = 0; c < 3; ++c)
    for (int k = 0; k < 64; ++k)
      s += double(g_coef[c * plane_ac + o + k]) *
           double(ac0[c * plane_ac + o + k]);
  double q = double(f.qf[cell]);
  if (f.clamp_scale) q /= double(f.clamp_scale[cell]);
  g_qf[cell] += float(-s / q);
}

}  // namespace
}  // namespace pikgpu

namespace {

// The backward launches; the forward pass (with the stages it reads) has
// run on ctx->stream.
int LaunchAdjoint(pikgpu_ctx* ctx, const float* target) {
  const Geo& g = ctx->g;
  const FrameScalars& s = ctx->s;
  cudaStream_t st = ctx->stream;
  const size_t npx = size_t(g.PW) * g.PH;
  const size_t nac = size_t(g.ac_stride) * g.By;
  const int nb = g.Bx * g.By;
  DevFrame f{};
  f.acs = P<uint8_t>(ctx->acs);
  f.qf = P<int32_t>(ctx->qf);
  f.dq_cf = P<uint8_t>(ctx->dq_cf);
  f.dq_map = P<uint8_t>(ctx->dq_map);
  f.table = P<float>(ctx->table);
  f.offsets = P<uint32_t>(ctx->offsets);
  f.idct = P<float>(ctx->idct);
  f.clamp_scale = ctx->use_clamp_scale ? P<float>(ctx->clamp_scale) : nullptr;
  const AdjJac* J = P<AdjJac>(ctx->adj_jac);
  float* ga = P<float>(ctx->adj_a);  // g_pre, then g_filt
  float* gb = P<float>(ctx->adj_b);  // g_cur, then g_up
  float* gc = P<float>(ctx->adj_c);  // g_idct
  float* g_coef = P<float>(ctx->adj_coef);
  float* g_qf = P<float>(ctx->adj_qf);
  const uint32_t* L[kNumClasses];
  int n[kNumClasses];
  for (int k = 0; k < kNumClasses; ++k) {
    L[k] = P<uint32_t>(ctx->list[k]);
    n[k] = int(ctx->lists[k].size());
  }

  k_adj_loss<<<kAdjLossBlocks, kAdjThreads, 0, st>>>(
      P<float>(ctx->dbg_pre), target, g.W, g.H, g.PW, g.PH, ga,
      P<double>(ctx->adj_partial));
  k_adj_sum<<<1, 32, 0, st>>>(P<double>(ctx->adj_partial), kAdjLossBlocks,
                              P<double>(ctx->adj_partial) + kAdjLossBlocks);
  ctx->launches += 2;
  const float* g_cur = ga;
  if (s.gaborish) {
    dim3 b(32, 8), gr(Blocks(g.PW, 32), Blocks(g.PH, 8), 3);
    k_adj_gab<<<gr, b, 0, st>>>(ga, g.PW, g.PH, s.gaborish, gb);
    ++ctx->launches;
    g_cur = gb;
  }
  CUDA_TRY(ctx, cudaMemsetAsync(g_qf, 0, sizeof(float) * nb, st));
  const float* g_idct = g_cur;
  if (s.have_ar) {
    // Guide bytes of the forward pass (the override, or MakeGuide again).
    const uint8_t* guide = P<uint8_t>(ctx->guide_ovr);
    if (!ctx->use_guide_ovr) {
      const bool smoothed = s.gaborish && !s.use_sharpened;
      int rc;
      if (smoothed && (rc = EnsureSmoothed(ctx)) != PIKGPU_OK) return rc;
      const float* src =
          smoothed ? P<float>(ctx->smoothed) : P<float>(ctx->idct);
      dim3 b(32, 8), gr(Blocks(g.PW + 12, 32), Blocks(g.PH + 12, 8), 3);
      k_export_guide<<<gr, b, 0, st>>>(src, g.PW, g.PH, P<uint32_t>(ctx->mm),
                                       P<uint8_t>(ctx->adj_guide));
      ++ctx->launches;
      guide = P<uint8_t>(ctx->adj_guide);
    }
    const int32_t* sig = P<int32_t>(ctx->sigma);
    const uint8_t* tape = P<uint8_t>(ctx->adj_tape);
    const float* epf = P<float>(ctx->dbg_epf);
    // g_filt goes to ga (g_pre is dead once g_cur exists; without
    // gaborish g_cur is ga itself, so g_filt then takes gb).
    float* g_filt = s.gaborish ? ga : gb;
    const int k8[3] = {kC8, kC4, kCSmall};
    for (int k : k8) {
      if (!n[k]) continue;
      k_adj_ar8<<<Blocks(n[k], kAdj8Blocks), kAdjThreads, 0, st>>>(
          g, f, s, J, L[k], n[k], sig, tape, epf, g_cur, g_filt, gc, g_qf);
      ++ctx->launches;
    }
    if (n[kC16]) {
      k_adj_ar_sq<16><<<n[kC16], kAdjThreads, 0, st>>>(
          g, f, s, L[kC16], n[kC16], sig, tape, epf, g_cur, g_filt, gc,
          g_qf);
      ++ctx->launches;
    }
    if (n[kC32]) {
      k_adj_ar_sq<32><<<n[kC32], kAdjThreads, 0, st>>>(
          g, f, s, L[kC32], n[kC32], sig, tape, epf, g_cur, g_filt, gc,
          g_qf);
      ++ctx->launches;
    }
    // gv = g_filt / sum_w in the plane g_cur no longer needs.
    float* gv = g_filt == ga ? gb : ga;
    dim3 gr(Blocks(g.PW, kEpfW), Blocks(g.PH, kEpfH));
    k_adj_epf_pass<false><<<gr, kEpfThreads, kAdjEpfSmemBytes, st>>>(
        g.PW, g.PH, guide, sig, g_filt, nullptr, gv);
    k_adj_epf_pass<true><<<gr, kEpfThreads, kAdjEpfSmemBytes, st>>>(
        g.PW, g.PH, guide, sig, g_filt, gv, gc);
    dim3 b3(32, 8), g3(Blocks(g.PW, 32), Blocks(g.PH, 8));
    k_adj_epf_border<<<g3, b3, 0, st>>>(g.PW, g.PH, guide, sig, gv, gc);
    ctx->launches += 3;
    g_idct = gc;
  }
  // g_up: the upsampled-prediction gradient (zero outside HF blocks), in
  // whichever plane buffer g_idct does not occupy.
  float* g_up = g_idct == gb ? gc : gb;
  if (s.predict_hf) {
    CUDA_TRY(ctx, cudaMemsetAsync(g_up, 0, sizeof(float) * 3 * npx, st));
  }
  const int k8[3] = {kC8, kC4, kCSmall};
  for (int k : k8) {
    if (!n[k]) continue;
    k_adj_topix8<<<Blocks(n[k], kAdj8Blocks), kAdjThreads, 0, st>>>(
        g, f, J, L[k], n[k], s.predict_hf, g_idct, g_coef, g_up);
    ++ctx->launches;
  }
  if (n[kC16]) {
    k_adj_topix_sq<16><<<n[kC16], kAdjThreads, 0, st>>>(
        g, f, L[kC16], n[kC16], s.predict_hf, g_idct, g_coef, g_up);
    ++ctx->launches;
  }
  if (n[kC32]) {
    k_adj_topix_sq<32><<<n[kC32], kAdjThreads, 0, st>>>(
        g, f, L[kC32], n[kC32], s.predict_hf, g_idct, g_coef, g_up);
    ++ctx->launches;
  }
  const int ng = g.Gx * g.Gy;
  if (s.predict_hf) {
    dim3 b(16, 16), gr(Blocks(2 * 64, 16), Blocks(2 * 64, 16), 3 * ng);
    k_adj_upsample<<<gr, b, 0, st>>>(g, g_up, P<float>(ctx->adj_pred));
    ++ctx->launches;
  }
  {
    dim3 b(32, 8), gr(Blocks(g.Bx, 32), Blocks(g.By, 8), 3);
    k_adj_lf<<<gr, b, 0, st>>>(g, f, J, s.predict_hf, P<float>(ctx->adj_pred),
                               g_coef);
    ++ctx->launches;
  }
  const float* ac0 =
      ctx->use_dq_ovr ? P<float>(ctx->dq_ovr) : P<float>(ctx->dbg_dequant);
  k_adj_qf<<<Blocks(nb, 256), 256, 0, st>>>(g, f, ac0, g_coef, g_qf);
  ++ctx->launches;
  (void)nac;
  CUDA_TRY(ctx, cudaGetLastError());
  return PIKGPU_OK;
}

}  // namespace

extern "C" {

int pikgpu_frame_set_dequantized_ac(pikgpu_ctx* ctx, const float* ac,
                                    int on_device) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  PIKGPU_NOT_PENDING(ctx);
  if (!ctx->have_frame) return Fail(ctx, PIKGPU_ERR_STATE, "no frame");
  ++ctx->generation;
  ctx->use_dq_ovr = ac != nullptr;
  if (!ac) return PIKGPU_OK;
  const Geo& g = ctx->g;
  const size_t bytes = sizeof(float) * 3 * size_t(g.ac_stride) * g.By;
  int rc;
  if ((rc = Ensure(ctx, &ctx->dq_ovr, bytes))) return rc;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->dq_ovr.p, ac, bytes,
                                on_device ? cudaMemcpyDeviceToDevice
                                          : cudaMemcpyHostToDevice,
                                ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PIKGPU_OK;
}

int pikgpu_frame_set_clamp_scale(pikgpu_ctx* ctx, const float* scale,
                                 int on_device) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  PIKGPU_NOT_PENDING(ctx);
  if (!ctx->have_frame) return Fail(ctx, PIKGPU_ERR_STATE, "no frame");
  ++ctx->generation;
  ctx->use_clamp_scale = scale != nullptr;
  if (!scale) return PIKGPU_OK;
  const size_t bytes = sizeof(float) * size_t(ctx->g.Bx) * ctx->g.By;
  int rc;
  if ((rc = Ensure(ctx, &ctx->clamp_scale, bytes))) return rc;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->clamp_scale.p, scale, bytes,
                                on_device ? cudaMemcpyDeviceToDevice
                                          : cudaMemcpyHostToDevice,
                                ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PIKGPU_OK;
}

int pikgpu_set_clamp_decisions(pikgpu_ctx* ctx, const uint8_t* tape) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  PIKGPU_NOT_PENDING(ctx);
  if (!ctx->have_frame) return Fail(ctx, PIKGPU_ERR_STATE, "no frame");
  ++ctx->generation;
  ctx->use_tape_in = false;
  if (!tape) return PIKGPU_OK;
  const size_t n = size_t(ctx->g.ac_stride) * ctx->g.By;
  for (size_t i = 0; i < n; ++i) {
    if (tape[i] > 4) {
      return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "clamp tape code %u at %zu",
                  tape[i], i);
    }
  }
  int rc;
  if ((rc = Ensure(ctx, &ctx->tape_in, n))) return rc;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  CUDA_TRY(ctx, cudaMemcpy(ctx->tape_in.p, tape, n, cudaMemcpyHostToDevice));
  ctx->use_tape_in = true;
  return PIKGPU_OK;
}

int pikgpu_get_clamp_decisions(pikgpu_ctx* ctx, uint8_t* tape) {
  if (!ctx || !tape) return PIKGPU_ERR_INVALID_ARG;
  PIKGPU_NOT_PENDING(ctx);
  if (!ctx->have_result || !ctx->tape_valid) {
    return Fail(ctx, PIKGPU_ERR_STATE,
                "no clamp tape: needs a frame with the EPF and a forward pass "
                "with PIKGPU_OPT_KEEP_STAGES (set before frame_begin) or "
                "pikgpu_adjoint");
  }
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  CUDA_TRY(ctx, cudaMemcpy(tape, ctx->adj_tape.p,
                           size_t(ctx->g.ac_stride) * ctx->g.By,
                           cudaMemcpyDeviceToHost));
  return PIKGPU_OK;
}

int pikgpu_adjoint(pikgpu_ctx* ctx, const float* target, double* loss,
                   float* grad_ac, float* grad_qf, int buffers_on_device) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  PIKGPU_NOT_PENDING(ctx);
  if (!ctx->have_frame || !(ctx->have_ac || ctx->use_dq_ovr)) {
    return Fail(ctx, PIKGPU_ERR_STATE, "frame or AC not supplied");
  }
  if (!target) return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "target is NULL");
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const Geo& g = ctx->g;
  const size_t npx = size_t(g.PW) * g.PH;
  const size_t nac = size_t(g.ac_stride) * g.By;
  const size_t nb = size_t(g.Bx) * g.By;
  const size_t ntg = 3 * size_t(g.W) * g.H;
  const int ng = g.Gx * g.Gy;
  int rc;
  if ((rc = Ensure(ctx, &ctx->adj_a, 4 * 3 * npx)) ||
      (rc = Ensure(ctx, &ctx->adj_b, 4 * 3 * npx)) ||
      (rc = Ensure(ctx, &ctx->adj_c, 4 * 3 * npx)) ||
      (rc = Ensure(ctx, &ctx->adj_coef, 4 * 3 * nac)) ||
      (rc = Ensure(ctx, &ctx->adj_pred, 4 * kG2GroupFloats * ng)) ||
      (rc = Ensure(ctx, &ctx->adj_qf, 4 * nb)) ||
      (rc = Ensure(ctx, &ctx->adj_guide,
                   3 * size_t(g.PW + 12) * (g.PH + 12))) ||
      (rc = Ensure(ctx, &ctx->adj_partial,
                   sizeof(double) * (kAdjLossBlocks + 1))) ||
      (rc = Ensure(ctx, &ctx->adj_jac, sizeof(AdjJac))) ||
      (rc = Ensure(ctx, &ctx->adj_tape, nac)) ||
      (rc = Ensure(ctx, &ctx->dbg_dequant, 4 * 3 * nac)) ||
      (rc = Ensure(ctx, &ctx->dbg_epf, 4 * 3 * npx)) ||
      (rc = Ensure(ctx, &ctx->dbg_pre, 4 * ntg))) {
    return rc;
  }
  cudaStream_t st = ctx->stream;
  if (!ctx->adj_jac_built) {
    CUDA_TRY(ctx, cudaFuncSetAttribute(
                      k_adj_epf_pass<false>,
                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                      int(kAdjEpfSmemBytes)));
    CUDA_TRY(ctx, cudaFuncSetAttribute(
                      k_adj_epf_pass<true>,
                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                      int(kAdjEpfSmemBytes)));
    k_adj_build_jac<<<2 * kJTypes + 9, 64, 0, st>>>(P<AdjJac>(ctx->adj_jac));
    CUDA_TRY(ctx, cudaGetLastError());
    ctx->adj_jac_built = true;
  }
  const float* tgt = target;
  if (!buffers_on_device) {
    if ((rc = Ensure(ctx, &ctx->adj_target, 4 * ntg))) return rc;
    CUDA_TRY(ctx, cudaMemcpyAsync(ctx->adj_target.p, target, 4 * ntg,
                                  cudaMemcpyHostToDevice, st));
    tgt = P<float>(ctx->adj_target);
  }
  // Forward pass, keeping the dequantised AC, the EPF output and pre_opsin.
  // The clamp kernels also record their branches (the clamp tape).
  const bool keep = ctx->keep_stages;
  ctx->keep_stages = ctx->record_tape = true;
  rc = LaunchAll(ctx, nullptr, 0, nullptr, 0);
  ctx->keep_stages = keep;
  ctx->record_tape = false;
  if (rc != PIKGPU_OK) return rc;
  if ((rc = LaunchAdjoint(ctx, tgt)) != PIKGPU_OK) return rc;
  const cudaMemcpyKind kind =
      buffers_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (grad_ac) {
    CUDA_TRY(ctx, cudaMemcpyAsync(grad_ac, ctx->adj_coef.p, 4 * 3 * nac, kind,
                                  st));
  }
  if (grad_qf) {
    CUDA_TRY(ctx, cudaMemcpyAsync(grad_qf, ctx->adj_qf.p, 4 * nb, kind, st));
  }
  if (loss) {
    CUDA_TRY(ctx, cudaMemcpyAsync(
                      loss, P<double>(ctx->adj_partial) + kAdjLossBlocks,
                      sizeof(double), kind, st));
  }
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  {
    int code = 0;
    CUDA_TRY(ctx, cudaMemcpy(&code, ctx->tc_err.p, sizeof(int),
                             cudaMemcpyDeviceToHost));
    if (code) {
      cudaMemset(ctx->tc_err.p, 0, sizeof(int));
      return Fail(ctx, PIKGPU_ERR_CUDA, "%s", WaitTimeoutMessage(code));
    }
  }
  ctx->have_result = true;
  return PIKGPU_OK;
}

}  // extern "C"
