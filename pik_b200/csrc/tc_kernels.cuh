// Split-BF16 tensor-core form of the square-block transforms (the
// ComputeTransposedScaledIDCT / DCT passes of TransformToPixels and the HF
// prediction's TransformFromPixels, pik/ac_strategy.cc:531-848,
// pik/dct.h:362-507) on the 5th-generation tensor cores (tcgen05).
//
// Each separable pass over a batch of 128 / N blocks of N x N is one GEMM
// D[128 x N] = A[128 x K] * B[N x K]^T with K = N: the rows of A are the
// batch's block rows (row m = N * block + r), B is the transform matrix, D
// accumulates in FP32 in tensor memory. The operands are split into BF16
// terms. With S = 2, x = hi + lo (about 16 significant bits) and
// D = A_hi B_hi + A_hi B_lo + A_lo B_hi (three MMAs): about 1e-5 relative
// error per product. With S = 3, x = hi + mid + lo (the full 24 bits) and
// six MMAs (hi hi, hi mid, mid hi, hi lo, lo hi, mid mid): FP32-level
// error. The transpose
// between the two passes of a 2-D transform costs nothing: each thread reads
// its row of D from tensor memory and writes it back to shared memory as the
// M-major A operand of the next pass.
//
// Operand layouts are the tcgen05 "no swizzle" canonical forms: 8 x 8 BF16
// core matrices of 128 contiguous bytes (8 rows of 16 bytes), the K groups
// of a row group 128 bytes apart and the row groups KC * 128 bytes apart
// (KC = K / 8). One thread issues the MMAs and commits them to an mbarrier;
// every wait on it is bounded and reports a timeout through `err` instead of
// hanging.
// Included by recon_kernels.cu.
#pragma once

#include <cuda_bf16.h>

namespace pikgpu {
namespace tc {

constexpr int kThreads = 128;            // one row of D per thread
constexpr uint32_t kMaxPolls = 1u << 22;  // bounded mbarrier wait

__device__ __forceinline__ uint32_t SmemU32(const void* p) {
  return uint32_t(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (no swizzle): start, leading (K-group)
// and stride (row-group) byte offsets, descriptor version 1.
__device__ __forceinline__ uint64_t Desc(const void* base, uint32_t lbo,
                                         uint32_t sbo) {
  const uint64_t a = SmemU32(base);
  return ((a >> 4) & 0x3FFFull) | (uint64_t((lbo >> 4) & 0x3FFF) << 16) |
         (uint64_t((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: BF16 x BF16 -> F32, M x N, B K-major,
// A K-major (a_mn = 0) or M-major (a_mn = 1).
__host__ __device__ constexpr uint32_t Idesc(int m, int n, int a_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(a_mn) << 15) |
         (uint32_t(n >> 3) << 17) | (uint32_t(m >> 4) << 24);
}

__device__ __forceinline__ void Mma(uint32_t d, uint64_t a, uint64_t b,
                                    uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void FenceBefore() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void FenceAfter() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ bool TryWait(uint32_t mbar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(phase)
      : "memory");
  return ok != 0;
}

// Waits for the commit of the MMAs just issued: at most `polls` polls. If
// they run out, the wait has failed (the caller reports it through its error
// flag), and a second wait of at most kMaxPolls polls follows, so that no
// MMA is left in flight when the caller goes on: its operands and
// accumulators are reused, and its tensor memory is freed at the end.
__device__ __forceinline__ bool WaitMma(uint32_t mbar, uint32_t phase,
                                        uint32_t polls) {
  for (uint32_t it = 0; it < polls; ++it) {
    if (TryWait(mbar, phase)) return true;
  }
  for (uint32_t it = 0; it < kMaxPolls; ++it) {
    if (TryWait(mbar, phase)) break;
  }
  return false;
}

// 16 consecutive FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void Ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,"
      "%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]),
        "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
        "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Splits 8 floats into S BF16 terms (each the rounded remainder of the
// previous ones), stored as one 16-byte chunk in each term's array
// (the arrays are `stride` bytes apart).
template <int S>
__device__ __forceinline__ void PutChunk(uint8_t* base, uint32_t stride,
                                         uint32_t off, const float* v) {
  float rest[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) rest[i] = v[i];
#pragma unroll
  for (int t = 0; t < S; ++t) {
    uint32_t w[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      // One conversion for two values; element 2i in the low half.
      const __nv_bfloat162 h =
          __floats2bfloat162_rn(rest[2 * i], rest[2 * i + 1]);
      w[i] = *reinterpret_cast<const uint32_t*>(&h);
      if (t + 1 < S) {
        const float2 b = __bfloat1622float2(h);
        rest[2 * i] -= b.x;
        rest[2 * i + 1] -= b.y;
      }
    }
    *reinterpret_cast<uint4*>(base + t * stride + off) =
        make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// Row m of a K-major operand (K = N): v[k], k = 0..N-1.
template <int N, int S>
__device__ __forceinline__ void PutRowK(uint8_t* base, int m, const float* v) {
#pragma unroll
  for (int kc = 0; kc < N / 8; ++kc) {
    PutChunk<S>(base, 128 * N * 2,
                (m >> 3) * (N / 8) * 128 + kc * 128 + (m & 7) * 16, v + 8 * kc);
  }
}

// Column k of an M-major operand for rows m0 .. m0 + N - 1: v[i] is element
// (m0 + i, k); m0 is a multiple of 8.
template <int N, int S>
__device__ __forceinline__ void PutColMN(uint8_t* base, int m0, int k,
                                         const float* v) {
#pragma unroll
  for (int g = 0; g < N / 8; ++g) {
    PutChunk<S>(base, 128 * N * 2,
                ((m0 >> 3) + g) * (N / 8) * 128 + (k >> 3) * 128 + (k & 7) * 16,
                v + 8 * g);
  }
}

// Shared state of one CTA: the A operand of each channel (its S split
// terms; K-major or M-major depending on the pass -- each pass's input is
// consumed before the next is written) and the transform matrices.
template <int N, int S>
struct Smem {
  static constexpr int kOpBytes = 128 * N * 2;  // 128 x N BF16
  static constexpr int kMatBytes = N * N * 2;
  alignas(128) uint8_t a[3][S * kOpBytes];
  alignas(128) uint8_t idct[S * kMatBytes];
  alignas(128) uint8_t dct[S * kMatBytes];
  alignas(8) uint64_t mbar;
  uint32_t tmem;
};

// Tensor-memory column of channel c's accumulator j (0 or 1).
template <int N>
__device__ __forceinline__ uint32_t AccCol(int c, int j) {
  return uint32_t(c * 2 * N + j * N);
}

// One split-BF16 GEMM pass for the three channels: D(c, j) = A(c) * B^T over
// K = N, then waits for it. Called by all threads after writing their rows
// of the A operands.
template <int N, int S>
__device__ __forceinline__ bool Pass(Smem<N, S>& s, int j, bool a_mn,
                                     const uint8_t* b, uint32_t& phase,
                                     uint32_t polls) {
  using Sm = Smem<N, S>;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  FenceBefore();
  __syncthreads();
  if (threadIdx.x == 0) {
    FenceAfter();
    const uint32_t idesc = Idesc(128, N, a_mn ? 1 : 0);
    constexpr uint32_t sbo = (N / 8) * 128;
    // Split-term pairs (i, k) with i + k <= S - 1 (S = 2: three products;
    // S = 3: six), largest first.
    constexpr int kPairs = S == 2 ? 3 : 6;
    constexpr int pi[6] = {0, 0, 1, 0, 2, 1};
    constexpr int pk[6] = {0, 1, 0, 2, 0, 1};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const uint32_t d = s.tmem + AccCol<N>(c, j);
#pragma unroll
      for (int kk = 0; kk < N / 16; ++kk) {
#pragma unroll
        for (int p = 0; p < kPairs; ++p) {
          Mma(d, Desc(s.a[c] + pi[p] * Sm::kOpBytes + kk * 256, 128, sbo),
              Desc(b + pk[p] * Sm::kMatBytes + kk * 256, 128, sbo), idesc,
              (kk > 0 || p > 0) ? 1u : 0u);
        }
      }
    }
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster."
        "b64 [%0];" ::"r"(SmemU32(&s.mbar))
        : "memory");
  }
  const bool ok = WaitMma(SmemU32(&s.mbar), phase, polls);
  phase ^= 1u;
  FenceAfter();
  return ok;
}

// This thread's row of D (N FP32 columns from dcol).
template <int N, int S>
__device__ __forceinline__ void LoadRow(const Smem<N, S>& s, uint32_t dcol,
                                        float* v) {
  const uint32_t lane_base = (threadIdx.x & ~31u) << 16;
#pragma unroll
  for (int c = 0; c < N; c += 16) Ld16(s.tmem + lane_base + dcol + c, v + c);
}

// Transform matrix (row-major n x k in constant memory) as a K-major BF16
// hi/lo B operand.
template <int N, int S>
__device__ __forceinline__ void PutMatrix(uint8_t* base, const float* m) {
  for (int i = threadIdx.x; i < N * N / 8; i += kThreads) {
    const int n = i / (N / 8), kc = i % (N / 8);
    float v[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) v[e] = m[n * N + kc * 8 + e];
    PutChunk<S>(base, N * N * 2,
                (n >> 3) * (N / 8) * 128 + kc * 128 + (n & 7) * 16, v);
  }
}

// One-channel operands: a CTA transforms one channel of a batch (the
// channels of a block are independent in the IDCT), so a thread holds a
// third of the registers of the three-channel kernels and more CTAs share
// an SM, each with its own MMA round trips.
// Side of a block's window of 2x2-cell prediction values: the block's 2 cov
// cells and one on each side (the upsampling's 3 taps).
template <int N>
__host__ __device__ constexpr int HfWin() {
  return N / 4 + 2;
}
template <int N, int S>
struct Smem1 {
  static constexpr int kOpBytes = 128 * N * 2;
  static constexpr int kMatBytes = N * N * 2;
  alignas(128) uint8_t a[S * kOpBytes];
  alignas(128) uint8_t idct[S * kMatBytes];
  // HF prediction: each block's window of cell values.
  float win[128 / N][HfWin<N>() * HfWin<N>()];
  alignas(8) uint64_t mbar;
  uint32_t tmem;
};
// Tensor-memory columns: the one-channel kernel's 2 accumulators of N
// columns, the three-channel kernel's 6 (rounded up to a power of two).
template <int N>
__host__ __device__ constexpr int TmemCols1() {
  return 2 * N;
}
template <int N>
__host__ __device__ constexpr int TmemCols3() {
  return N == 16 ? 128 : 256;
}
// The HF corner table of an N x N block: 2 cov rows of HfWin<N>() taps.
template <int N>
__device__ __forceinline__ const float* HfCorner() {
  return N == 16 ? &c_t.hf_corner16[0][0] : &c_t.hf_corner32[0][0];
}

// This thread's row of D (N FP32 columns from dcol).
template <int N, int S>
__device__ __forceinline__ void LoadRow1(const Smem1<N, S>& s, uint32_t dcol,
                                         float* v) {
  const uint32_t lane_base = (threadIdx.x & ~31u) << 16;
#pragma unroll
  for (int c = 0; c < N; c += 16) Ld16(s.tmem + lane_base + dcol + c, v + c);
}

// One split-BF16 GEMM pass of the CTA's channel: D(j) = A * B^T over K = N
// (tensor-memory columns j N ..), then waits for it (bounded).
template <int N, int S>
__device__ __forceinline__ bool Pass1(Smem1<N, S>& s, int j, bool a_mn,
                                      const uint8_t* b, uint32_t& phase,
                                      uint32_t polls) {
  using Sm = Smem1<N, S>;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  FenceBefore();
  __syncthreads();
  if (threadIdx.x == 0) {
    FenceAfter();
    const uint32_t idesc = Idesc(128, N, a_mn ? 1 : 0);
    constexpr uint32_t sbo = (N / 8) * 128;
    constexpr int kPairs = S == 2 ? 3 : 6;
    constexpr int pi[6] = {0, 0, 1, 0, 2, 1};
    constexpr int pk[6] = {0, 1, 0, 2, 0, 1};
    const uint32_t d = s.tmem + uint32_t(j * N);
#pragma unroll
    for (int kk = 0; kk < N / 16; ++kk) {
#pragma unroll
      for (int p = 0; p < kPairs; ++p) {
        Mma(d, Desc(s.a + pi[p] * Sm::kOpBytes + kk * 256, 128, sbo),
            Desc(b + pk[p] * Sm::kMatBytes + kk * 256, 128, sbo), idesc,
            (kk > 0 || p > 0) ? 1u : 0u);
      }
    }
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster."
        "b64 [%0];" ::"r"(SmemU32(&s.mbar))
        : "memory");
  }
  const bool ok = WaitMma(SmemU32(&s.mbar), phase, polls);
  phase ^= 1u;
  FenceAfter();
  return ok;
}

}  // namespace tc

// AdaptiveReconstruction clamp for square DCT blocks on the tensor cores
// (split-BF16 form of k_square_ar_rows, pik/adaptive_reconstruction.cc:
// 128-244, 334-471): DCT of (filtered - original) for the three channels,
// the clamp ratio of each coefficient (minimum over X, Y, B) in registers,
// then the IDCT of the scaled correction added to the original. `count` is
// read from device memory (the compacted list of k_active_blocks).
// Dynamic shared memory of k_square_ar_tc: its Smem and room to align it
// to 128 bytes.
template <int N, int S>
constexpr size_t ArTcSmemBytes() {
  return sizeof(tc::Smem<N, S>) + 128;
}

template <int N, int S>
__global__ void __launch_bounds__(tc::kThreads, N == 16 ? 4 : 2)
    k_square_ar_tc(Geo g, DevFrame f, FrameScalars sc, const uint32_t* list,
                   const int* count_ptr, int* work, int* err) {
  PdlLaunchDependents();
  PdlTail pdl_tail;
  using namespace tc;
  constexpr int BPB = 128 / N;
  constexpr int cov = N / 8;
  constexpr int kCols = TmemCols3<N>();
  extern __shared__ uint8_t ar_tc_smem[];
  Smem<N, S>& s = *reinterpret_cast<Smem<N, S>*>(
      (reinterpret_cast<uintptr_t>(ar_tc_smem) + 127) & ~uintptr_t(127));
  __shared__ int s_next[2];
  const int t = threadIdx.x, bl = t / N, r = t % N;
  const int count = *count_ptr;
  const int nbat = (count + BPB - 1) / BPB;
  // Batches are taken from a work counter, one at a time: a CTA that
  // starts late (its SM busy with another class's kernel) takes fewer. The
  // first is taken before the set-up, which a CTA without work skips (the
  // grid is sized for all of the class's blocks, the active ones are
  // counted on the device). The next batch is fetched at the start of a
  // batch and read after the batch's last barrier.
  if (t == 0) s_next[0] = atomicAdd(work, 1);
  __syncthreads();
  int batch = s_next[0];
  if (batch >= nbat) return;
  if (t < 32) {
    asm volatile(
        "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::
            "r"(SmemU32(&s.tmem)),
        "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(
        SmemU32(&s.mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  PutMatrix<N, S>(s.idct, c_t.idct + MatOffset(N));
  PutMatrix<N, S>(s.dct, c_t.dct + MatOffset(N));
  FenceBefore();
  __syncthreads();
  FenceAfter();
  uint32_t phase = 0;
  const size_t plane = size_t(g.PW) * g.PH;
  const float inv_nn = 1.0f / float(N * N);
  bool ok = true;
  for (int k = 1; batch < nbat && ok; ++k) {
    if (t == 0) s_next[k & 1] = atomicAdd(work, 1);
    const int idx = batch * BPB + bl;
    const bool active = idx < count;
    const uint32_t pkd = list[active ? idx : 0];
    const int bx = pkd & 0xFFFF, by = pkd >> 16;
    const size_t row0 = size_t(by * 8 + r) * g.PW + bx * 8;
    // The block's clamp intervals (a chain of dependent table loads) are
    // looked up first, so that the loads resolve during the DCT passes. The
    // class holds only blocks of one type.
    static_assert(N == 16 || N == 32, "DCT16X16 or DCT32X32");
    constexpr int type = N == 16 ? kDCT16X16 : kDCT32X32;
    const int qac = f.qf[by * g.Bx + bx];
    const float inv_quant_ac =
        ClampInvQuantAc(g, f, sc.inv_global_scale, bx, by, qac);
    const int cf = f.dq_cf[(by >> 3) * g.Tx + (bx >> 3)];
    const int table = f.dq_map[cf * 256 + (qac - 1)];
    uint32_t dm_off[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      dm_off[c] = f.offsets[(table * 7 + QuantKindOf(type)) * 3 + c] + r * N;
    }
    float T[N];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
      for (int x = 0; x < N; x += 4) {
        float4 a = make_float4(0.f, 0.f, 0.f, 0.f), o = a;
        if (active) {
          a = *reinterpret_cast<const float4*>(f.filt + c * plane + row0 + x);
          o = *reinterpret_cast<const float4*>(f.idct + c * plane + row0 + x);
        }
        T[x] = a.x - o.x, T[x + 1] = a.y - o.y;
        T[x + 2] = a.z - o.z, T[x + 3] = a.w - o.w;
      }
      PutRowK<N, S>(s.a[c], t, T);  // pixel row y = r of the correction
    }
    ok = Pass<N, S>(s, 0, false, s.dct, phase, f.tc_polls);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      LoadRow<N, S>(s, AccCol<N>(c, 0), T);  // t_y[k]
      PutColMN<N, S>(s.a[c], N * bl, r, T);
    }
    ok = Pass<N, S>(s, 1, true, s.dct, phase, f.tc_polls) && ok;
    float Y[3][N];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      LoadRow<N, S>(s, AccCol<N>(c, 1), Y[c]);  // coefficient row k = r
#pragma unroll
      for (int l = 0; l < N; ++l) Y[c][l] *= inv_nn;
    }
    // Clamp ratios of coefficient row k = r, minimum over the channels.
    {
      const float* dm[3];
      bool dm_vec = true;  // rows 16-byte aligned: float4 loads
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        dm[c] = f.table + dm_off[c];
        dm_vec = dm_vec && (reinterpret_cast<uintptr_t>(dm[c]) & 15) == 0;
      }
      const size_t tape_row = CoefOffset(g, bx, by, cov, r * N);
      uint8_t* tape =
          f.clamp_tape && active ? f.clamp_tape + tape_row : nullptr;
      const uint8_t* tin =
          f.clamp_tape_in && active ? f.clamp_tape_in + tape_row : nullptr;
      float dq[3][4];  // dm[c][l0 .. l0 + 3]
#pragma unroll
      for (int l = 0; l < N; ++l) {
        if ((l & 3) == 0) {
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            if (dm_vec) {
              const float4 q = *reinterpret_cast<const float4*>(dm[c] + l);
              dq[c][0] = q.x, dq[c][1] = q.y, dq[c][2] = q.z, dq[c][3] = q.w;
            } else {
#pragma unroll
              for (int e = 0; e < 4; ++e) dq[c][e] = dm[c][l + e];
            }
          }
        }
        const bool llf = r < cov && l < cov;
        const float ls = llf ? LlfScale(type, l, r) : 0.f;
        float mr = 1.0f, rt[3];
        int arg = -1;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          rt[c] = ClampRatio(
              Y[c][l], llf ? ls * sc.mul_dc[c] : dq[c][l & 3] * inv_quant_ac);
          if (rt[c] < mr) mr = rt[c], arg = c;
        }
        uint8_t code = arg < 0 ? 0 : mr == 0.0f ? 4 : uint8_t(arg + 1);
        if (tin) {
          code = tin[l];
          mr = TapeRatio(code, rt[0], rt[1], rt[2]);
        }
        if (tape) tape[l] = code;
#pragma unroll
        for (int c = 0; c < 3; ++c) Y[c][l] = Y[c][l] * mr;
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) PutRowK<N, S>(s.a[c], t, Y[c]);
    ok = Pass<N, S>(s, 0, false, s.idct, phase, f.tc_polls) && ok;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      LoadRow<N, S>(s, AccCol<N>(c, 0), T);
      PutColMN<N, S>(s.a[c], N * bl, r, T);
    }
    ok = Pass<N, S>(s, 1, true, s.idct, phase, f.tc_polls) && ok;
    ok = __syncthreads_and(ok);
    const int next = s_next[k & 1];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      LoadRow<N, S>(s, AccCol<N>(c, 1), T);  // pixel row v = r
      if (active && ok) {
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
    batch = next;
  }
  if (!ok && t == 0) atomicExch(err, 1);
  FenceBefore();
  __syncthreads();
  if (t < 32) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(
                     s.tmem),
                 "r"(kCols));
  }
}

// HF prediction + AddBlockExceptLFAndLLFTo + IDCT for 16x16 and 32x32 DCT
// blocks on the tensor cores (split-BF16 form of k_square_idct_rows and
// k_square_idct). Persistent CTAs of 128 threads; an item is one channel
// of a batch of 128 / N blocks ((batch, channel) pairs, batch-major; the
// channels of a block are independent here). A thread holds one row of one
// channel, so several CTAs share an SM (eight for N = 16, four for
// N = 32), each with its own MMA round trips; the next item's coefficient
// row is loaded while this item's passes run.
template <int N, int S>
__global__ void __launch_bounds__(tc::kThreads, N == 16 ? 8 : 4)
    k_square_idct_tc1(Geo g, DevFrame f, const uint32_t* list, int count,
                      int predict_hf, int* work, int* err) {
  PdlLaunchDependents();
  PdlTail pdl_tail;
  using namespace tc;
  using square::CoefRowOffset;
  static_assert(N == 16 || N == 32, "DCT16X16 or DCT32X32");
  constexpr int BPB = 128 / N;  // blocks per batch
  constexpr int cov = N / 8;
  constexpr int W = HfWin<N>();  // prediction window side (cells)
  constexpr int kCols = TmemCols1<N>();
  __shared__ Smem1<N, S> s;
  __shared__ int s_first[2], s_next[2];
  const int t = threadIdx.x, bl = t / N, r = t % N;
  const int nitems = 3 * ((count + BPB - 1) / BPB);
  // Items are taken from a work counter, so that a CTA that starts late
  // (its SM busy with another class's kernel) takes fewer; a CTA without
  // work skips the set-up. Two are known ahead: the current one and the
  // next, whose coefficient row is loaded during the current item's
  // passes; the one after that is fetched during the current item and read
  // after its first pass's barrier.
  if (t == 0) {
    s_first[0] = atomicAdd(work, 1);
    s_first[1] = atomicAdd(work, 1);
  }
  __syncthreads();
  int item = s_first[0], item_next = s_first[1];
  if (item >= nitems) return;
  if (t < 32) {
    asm volatile(
        "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::
            "r"(SmemU32(&s.tmem)),
        "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(
        SmemU32(&s.mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  PutMatrix<N, S>(s.idct, c_t.idct + MatOffset(N));
  FenceBefore();
  __syncthreads();
  FenceAfter();
  uint32_t phase = 0;
  const size_t plane_ac = size_t(g.ac_stride) * g.By;
  const size_t plane_px = size_t(g.PW) * g.PH;
  const float inv_nn = 1.0f / float(N * N);
  // This lane's row of the HF corner table (rows r < 2 cov).
  const float* ctab = HfCorner<N>();
  float cr[W];
#pragma unroll
  for (int m = 0; m < W; ++m) cr[m] = ctab[(r & (2 * cov - 1)) * W + m];
  bool ok = true;
  // The next item's coefficient row is loaded while this item's passes
  // run (the CTAs of an SM otherwise wait for their loads in step).
  float X[N];
  auto load_row = [&](int it) {
    const int bt = it / 3, ch = it - 3 * bt;
    const int i = bt * BPB + bl;
    const uint32_t pk = list[i < count ? i : 0];
    const float* crow = f.ac + ch * plane_ac +
                        CoefRowOffset(g, pk & 0xFFFF, pk >> 16, N, r);
#pragma unroll
    for (int j = 0; j < N; j += 4) {
      const float4 v = i < count ? *reinterpret_cast<const float4*>(crow + j)
                                 : make_float4(0.f, 0.f, 0.f, 0.f);
      X[j] = v.x, X[j + 1] = v.y, X[j + 2] = v.z, X[j + 3] = v.w;
    }
    return pk;
  };
  uint32_t pkd_next = item < nitems ? load_row(item) : 0u;
  for (int k = 0; item < nitems && ok; ++k) {
    const int batch = item / 3, c = item - 3 * batch;
    const int idx = batch * BPB + bl;
    const bool active = idx < count;
    const uint32_t pkd = pkd_next;
    const int bx = pkd & 0xFFFF, by = pkd >> 16;
    // HF prediction: adding the predicted coefficients outside the
    // 2cov x 2cov corner and transforming back equals transforming the
    // coefficients minus that corner of DCT(P) and adding P (IDCT(DCT(P))
    // = P). The upsampled prediction P of this pixel row is the 3-tap
    // vertical blend of three rows of the 2x2-cell grid (W columns), then
    // the 3-tap horizontal blend; its DCT corner is C Pred C^T over the
    // block's W x W cell window (C = HfCorner<N>), of which lanes
    // r < 2 cov subtract row r. The class holds only DCT16X16 (DCT32X32)
    // blocks, which predict HF. The block's N lanes first stage its cell
    // window in shared memory (a few loads per lane instead of tens of
    // scalar loads of cells that the lanes share).
    float P[N];
    const bool hf = active && predict_hf;
    if (predict_hf) {
      const int gi = (by >> 6) * g.Gx + (bx >> 6);
      const int rb = (by & 63) * 2, q0 = (bx & 63) * 2;
      const float* pred = f.pred2x2_g + gi * kG2GroupFloats + c * kG2 * kG2 +
                          (rb + 1) * kG2 + q0 + 1;
      for (int e = r; e < W * W; e += N) {
        s.win[bl][e] = pred[(e / W) * kG2 + e % W];
      }
      __syncwarp();
    }
    if (hf) {
      const float* w = s.win[bl];
      const int iy = r & 3;
      const float* w0 = w + (r >> 2) * W;
      const float v0 = c_t.ub4[0][iy], v1 = c_t.ub4[1][iy],
                  v2 = c_t.ub4[2][iy];
      float col[W];
#pragma unroll
      for (int m = 0; m < W; ++m) {
        col[m] = fmaf(w0[2 * W + m], v2, fmaf(w0[W + m], v1, w0[m] * v0));
      }
#pragma unroll
      for (int x = 0; x < N; ++x) {
        const int q = x >> 2, ix = x & 3;
        P[x] = fmaf(col[q + 2], c_t.ub4[2][ix],
                    fmaf(col[q + 1], c_t.ub4[1][ix], col[q] * c_t.ub4[0][ix]));
      }
      if (r < 2 * cov) {
        float u[W];
#pragma unroll
        for (int rho = 0; rho < W; ++rho) {
          float a = 0.f;
#pragma unroll
          for (int m = 0; m < W; ++m) a = fmaf(w[rho * W + m], cr[m], a);
          u[rho] = a;
        }
#pragma unroll
        for (int l = 0; l < 2 * cov; ++l) {
          float v = 0.f;
#pragma unroll
          for (int rho = 0; rho < W; ++rho) {
            v = fmaf(ctab[l * W + rho], u[rho], v);
          }
          X[l] -= v * inv_nn;
        }
      }
    }
    float T[N];
    PutRowK<N, S>(s.a, t, X);
    if (item_next < nitems) pkd_next = load_row(item_next);
    if (t == 0) s_next[k & 1] = atomicAdd(work, 1);
    ok = Pass1<N, S>(s, 0, false, s.idct, phase, f.tc_polls) && ok;
    const int item_after = s_next[k & 1];
    LoadRow1<N, S>(s, 0, T);  // T[k = r][v]
    PutColMN<N, S>(s.a, N * bl, r, T);
    ok = Pass1<N, S>(s, 1, true, s.idct, phase, f.tc_polls) && ok;
    ok = __syncthreads_and(ok);
    LoadRow1<N, S>(s, N, T);  // pixel row v = r
    if (hf) {
#pragma unroll
      for (int i = 0; i < N; ++i) T[i] += P[i];
    }
    if (active && ok) {
      float* out = f.idct + c * plane_px + size_t(by * 8 + r) * g.PW + bx * 8;
#pragma unroll
      for (int i = 0; i < N; i += 4) {
        *reinterpret_cast<float4*>(out + i) =
            make_float4(T[i], T[i + 1], T[i + 2], T[i + 3]);
      }
    }
    item = item_next;
    item_next = item_after;
  }
  if (!ok && t == 0) atomicExch(err, 1);
  FenceBefore();
  __syncthreads();
  if (t < 32) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(
                     s.tmem),
                 "r"(kCols));
  }
}

}  // namespace pikgpu
