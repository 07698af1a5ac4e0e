// Square DCT blocks (8x8, 16x16, 32x32) with one thread per row of the
// N x N block: a "unit" of N lanes holds one block (and channel) in
// registers, the transform matrices are compile-time operands from
// __constant__ memory, and the transpose between the two separable passes
// goes through a padded shared-memory tile with __syncwarp only. Every
// output is the same sequential sum (index 0..N-1, separate multiply and
// add) as the row-major formulation, so results are bit-identical to it.
// Included by recon_kernels.cu.
#pragma once

namespace pikgpu {
namespace square {

// tsIDCT pass 1 on coefficient row c (row = horizontal frequency k):
// t[v] = sum_l c[l] A[v][l].
template <int N>
__device__ __forceinline__ void IdctRow(const float (&c)[N], float (&t)[N]) {
#pragma unroll
  for (int v = 0; v < N; ++v) {
    float s = 0.f;
#pragma unroll
    for (int l = 0; l < N; ++l) s += c[l] * c_t.idct[MatOffset(N) + v * N + l];
    t[v] = s;
  }
}
// tsIDCT pass 2 on column u[k] = tmp[k][v]: out[x] = sum_k A[x][k] u[k].
template <int N>
__device__ __forceinline__ void IdctCol(const float (&u)[N], float (&o)[N]) {
#pragma unroll
  for (int x = 0; x < N; ++x) {
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < N; ++k) s += c_t.idct[MatOffset(N) + x * N + k] * u[k];
    o[x] = s;
  }
}
// tsDCT pass 1 on pixel row p (row y): t[k] = sum_x B[k][x] p[x].
template <int N>
__device__ __forceinline__ void DctRow(const float (&p)[N], float (&t)[N]) {
#pragma unroll
  for (int k = 0; k < N; ++k) {
    float s = 0.f;
#pragma unroll
    for (int x = 0; x < N; ++x) s += c_t.dct[MatOffset(N) + k * N + x] * p[x];
    t[k] = s;
  }
}
// tsDCT pass 2 on q[y] = tmp[k][y]: o[l] = (sum_y q[y] B[l][y]) / N^2.
template <int N>
__device__ __forceinline__ void DctCol(const float (&q)[N], float (&o)[N]) {
  const float scale = 1.0f / float(N * N);
#pragma unroll
  for (int l = 0; l < N; ++l) {
    float s = 0.f;
#pragma unroll
    for (int y = 0; y < N; ++y) s += q[y] * c_t.dct[MatOffset(N) + l * N + y];
    o[l] = s * scale;
  }
}

// Writes `v` as row r of the unit's tile (stride N + 1) ...
template <int N>
__device__ __forceinline__ void PutRow(float* tile, int r, const float (&v)[N]) {
#pragma unroll
  for (int i = 0; i < N; ++i) tile[r * (N + 1) + i] = v[i];
}
template <int N>
__device__ __forceinline__ void PutCol(float* tile, int r, const float (&v)[N]) {
#pragma unroll
  for (int i = 0; i < N; ++i) tile[i * (N + 1) + r] = v[i];
}
template <int N>
__device__ __forceinline__ void GetRow(const float* tile, int r, float (&v)[N]) {
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = tile[r * (N + 1) + i];
}
template <int N>
__device__ __forceinline__ void GetCol(const float* tile, int r, float (&v)[N]) {
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = tile[i * (N + 1) + r];
}

// Pointer to row r of the block's coefficients in the frame layout: row r
// of the N x N matrix lives in block row (by + r / 8) at column offset
// bx * 64 + (r % 8) * N (GatherCoefficients layout, pik/ac_strategy.h:255-272).
__device__ __forceinline__ size_t CoefRowOffset(const Geo& g, int bx, int by,
                                                int n, int r) {
  return size_t(by + r / 8) * g.ac_stride + size_t(bx) * 64 + (r % 8) * n;
}

}  // namespace square

constexpr int kSquareThreads = 128;

// HF prediction + AddBlockExceptLFAndLLFTo + IDCT for square DCT blocks
// (UpSample4x4BlurDCT, pik/ac_predictions.cc:263-374; TransformToPixels,
// pik/ac_strategy.cc:674-848). One unit per (block, channel).
template <int N>
__global__ void __launch_bounds__(kSquareThreads)
    k_square_idct_rows(Geo g, DevFrame f, const uint32_t* list, int count,
                       int predict_hf) {
  PdlLaunchDependents();
  PdlTail pdl_tail;
  using namespace square;
  constexpr int UPW = 32 / N;  // units per warp
  constexpr int cov = N / 8;
  __shared__ float s_tile[kSquareThreads / N][N * (N + 1)];
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int unit = lane / N, r = lane % N;
  const int item = warp * UPW + unit;
  if (warp * UPW >= 3 * count) return;  // warp-uniform
  const bool active = item < 3 * count;
  float* tile = s_tile[threadIdx.x / N];
  const int b = active ? item / 3 : 0, c = active ? item % 3 : 0;
  const uint32_t pk = list[b];
  const int bx = pk & 0xFFFF, by = pk >> 16;
  const size_t plane_ac = size_t(g.ac_stride) * g.By;
  const float* crow = f.ac + c * plane_ac + CoefRowOffset(g, bx, by, N, r);
  float X[N];
#pragma unroll
  for (int i = 0; i < N; i += 4) {
    const float4 v = *reinterpret_cast<const float4*>(crow + i);
    X[i] = v.x, X[i + 1] = v.y, X[i + 2] = v.z, X[i + 3] = v.w;
  }
  if (predict_hf) {
    // DCT_NOHF shares the 8x8 class; its prediction is computed but not
    // added, keeping the warp's control flow uniform.
    const bool hf = PredictHFOf(f.acs[by * g.Bx + bx] >> 4);
    const int gi = (by >> 6) * g.Gx + (bx >> 6);
    const float* pred = f.pred2x2_g + gi * kG2GroupFloats + c * kG2 * kG2;
    const int X0 = (bx & 63) * 8, Y = (by & 63) * 8 + r;
    float P[N], T[N];
    UpsampleRow<N>(pred, X0, Y, P);
    DctRow<N>(P, T);
    PutCol<N>(tile, r, T);  // tmp[k][y = r]
    __syncwarp();
    GetRow<N>(tile, r, P);  // tmp[k = r][y]
    DctCol<N>(P, T);        // predicted coefficients row k = r
    __syncwarp();
#pragma unroll
    for (int l = 0; l < N; ++l) {
      if (hf && !(r < 2 * cov && l < 2 * cov)) X[l] += T[l];
    }
  }
  float T[N];
  IdctRow<N>(X, T);
  PutRow<N>(tile, r, T);  // tmp[k = r][v]
  __syncwarp();
  GetCol<N>(tile, r, X);  // column v = r
  IdctCol<N>(X, T);       // pixel row v = r
  if (active) {
    float* out = f.idct + c * size_t(g.PW) * g.PH +
                 size_t(by * 8 + r) * g.PW + bx * 8;
#pragma unroll
    for (int i = 0; i < N; i += 4) {
      *reinterpret_cast<float4*>(out + i) =
          make_float4(T[i], T[i + 1], T[i + 2], T[i + 3]);
    }
  }
}

// Keeps the blocks of each class's list that the EPF filtered (some cell
// has sigma >= kMinSigma) in that class's active list (counter k); for the
// others the clamp stage is an exact no-op because the filtered block
// equals the original. One thread per block of all the classes.
__global__ void k_active_blocks(Geo g, const int32_t* sigma,
                                const uint8_t* acs, ClassLists cl,
                                int* counters) {
  PdlWait();  // the EPF's sigma
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int k = 0;
  while (k < kMaxClasses && i >= cl.n[k]) i -= cl.n[k++];
  bool any = false;
  uint32_t pk = 0;
  if (k < kMaxClasses) {
    pk = cl.list[k][i];
    const int bx = pk & 0xFFFF, by = pk >> 16;
    const int cov = Covered(acs[by * g.Bx + bx] >> 4);
    for (int y = 0; y < cov; ++y)
      for (int x = 0; x < cov; ++x)
        any |= sigma[(by + y) * g.Bx + bx + x] >= kMinSigma;
  }
  // One atomic per warp and class: the lanes of a class take consecutive
  // slots after the first of them reserves them all.
  const int lane = threadIdx.x & 31;
  for (int kk = 0; kk < kMaxClasses; ++kk) {
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, any && k == kk);
    if (!m) continue;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&counters[kk], __popc(m));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    if (any && k == kk) {
      cl.active[kk][base + __popc(m & ((1u << lane) - 1))] = pk;
    }
  }
}

// AdaptiveReconstruction clamp for square DCT blocks, one unit per block
// (pik/adaptive_reconstruction.cc:128-244, 334-471). `count` is read from
// device memory (the compacted list of k_active_blocks).
template <int N>
__global__ void __launch_bounds__(kSquareThreads)
    k_square_ar_rows(Geo g, DevFrame f, FrameScalars s, const uint32_t* list,
                     const int* count_ptr) {
  PdlLaunchDependents();
  PdlTail pdl_tail;
  using namespace square;
  constexpr int UPW = 32 / N;
  constexpr int cov = N / 8;
  __shared__ float s_tile[kSquareThreads / N][N * (N + 1)];
  const int count = *count_ptr;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int unit = lane / N, r = lane % N;
  const int item = warp * UPW + unit;
  if (warp * UPW >= count) return;  // warp-uniform
  const bool active = item < count;
  float* tile = s_tile[threadIdx.x / N];
  const uint32_t pk = list[active ? item : 0];
  const int bx = pk & 0xFFFF, by = pk >> 16;
  const int type = f.acs[by * g.Bx + bx] >> 4;
  const size_t plane = size_t(g.PW) * g.PH;
  const size_t row0 = size_t(by * 8 + r) * g.PW + bx * 8;
  float Y[3][N];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float D[N], T[N];
#pragma unroll
    for (int x = 0; x < N; x += 4) {
      const float4 a =
          *reinterpret_cast<const float4*>(f.filt + c * plane + row0 + x);
      const float4 o =
          *reinterpret_cast<const float4*>(f.idct + c * plane + row0 + x);
      D[x] = a.x - o.x, D[x + 1] = a.y - o.y;
      D[x + 2] = a.z - o.z, D[x + 3] = a.w - o.w;
    }
    DctRow<N>(D, T);
    PutCol<N>(tile, r, T);
    __syncwarp();
    GetRow<N>(tile, r, D);
    DctCol<N>(D, Y[c]);
    __syncwarp();
  }
  // Clamp ratios of coefficient row k = r, minimum over the channels.
  const int qac = f.qf[by * g.Bx + bx];
  const float inv_quant_ac =
      ClampInvQuantAc(g, f, s.inv_global_scale, bx, by, qac);
  const int cf = f.dq_cf[(by >> 3) * g.Tx + (bx >> 3)];
  const int table = f.dq_map[cf * 256 + (qac - 1)];
  const int kind = QuantKindOf(type);
  const float* dm0 = f.table + f.offsets[(table * 7 + kind) * 3 + 0] + r * N;
  const float* dm1 = f.table + f.offsets[(table * 7 + kind) * 3 + 1] + r * N;
  const float* dm2 = f.table + f.offsets[(table * 7 + kind) * 3 + 2] + r * N;
  const size_t tape_row = CoefOffset(g, bx, by, cov, r * N);
  uint8_t* tape = f.clamp_tape && active ? f.clamp_tape + tape_row : nullptr;
  const uint8_t* tin =
      f.clamp_tape_in && active ? f.clamp_tape_in + tape_row : nullptr;
#pragma unroll
  for (int l = 0; l < N; ++l) {
    const bool llf = r < cov && l < cov;
    const float ls = llf ? LlfScale(type, l, r) : 0.f;
    float mr = 1.0f;
    int arg = -1;
    const float rt0 =
        ClampRatio(Y[0][l], llf ? ls * s.mul_dc[0] : dm0[l] * inv_quant_ac);
    if (rt0 < mr) mr = rt0, arg = 0;
    const float rt1 =
        ClampRatio(Y[1][l], llf ? ls * s.mul_dc[1] : dm1[l] * inv_quant_ac);
    if (rt1 < mr) mr = rt1, arg = 1;
    const float rt2 =
        ClampRatio(Y[2][l], llf ? ls * s.mul_dc[2] : dm2[l] * inv_quant_ac);
    if (rt2 < mr) mr = rt2, arg = 2;
    uint8_t code = arg < 0 ? 0 : mr == 0.0f ? 4 : uint8_t(arg + 1);
    if (tin) {
      code = tin[l];
      mr = TapeRatio(code, rt0, rt1, rt2);
    }
    if (tape) tape[l] = code;
    Y[0][l] = Y[0][l] * mr;
    Y[1][l] = Y[1][l] * mr;
    Y[2][l] = Y[2][l] * mr;
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float T[N], U[N];
    IdctRow<N>(Y[c], T);
    PutRow<N>(tile, r, T);
    __syncwarp();
    GetCol<N>(tile, r, U);
    IdctCol<N>(U, T);
    __syncwarp();
    if (active) {
#pragma unroll
      for (int x = 0; x < N; x += 4) {
        const float4 o =
            *reinterpret_cast<const float4*>(f.idct + c * plane + row0 + x);
        *reinterpret_cast<float4*>(f.filt + c * plane + row0 + x) =
            make_float4(T[x] + o.x, T[x + 1] + o.y, T[x + 2] + o.z,
                        T[x + 3] + o.w);
      }
    }
  }
}

}  // namespace pikgpu
