// C ABI of the B200 reconstruction path (include/pikgpu.h): validation,
// device memory, uploads and the launch sequence that replaces
// Dequant::DoAC + ReconOpsinImage (per group) + FinalizeFrameDecoding
// (pik/compressed_image.cc:586-707, 936-1106, 1144-1181) and
// DequantDC + AdaptiveDCReconstruction (pik/compressed_dc.cc:181-231,
// pik/adaptive_reconstruction.cc:300-332).
//
// Single translation unit: the kernels are included so that the
// __constant__ tables need no relocatable device code.

#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "../../include/pikgpu.h"
#include "recon_kernels.cu"
#include "tables.cc"

using namespace pikgpu;

namespace {

// Block classes launched by separate kernels.
enum Class { kC8 = 0, kC16, kC32, kC4, kCSmall, kNumClasses };
// Device counters, zeroed at the start of every frame: the clamp's active
// blocks per class, then the work counters of the persistent tensor-core
// transform and clamp kernels.
constexpr int kWorkIdct = kNumClasses, kWorkAr = kNumClasses + 1;
constexpr int kWorkIdct32 = kNumClasses + 2, kWorkAr32 = kNumClasses + 3;
constexpr int kNumCounters = kNumClasses + 4;
// Up to this many small-transform blocks per SM, the small classes run one
// CTA per block (short latency: one or two waves); above it, one thread per
// block and channel (throughput).
constexpr int kSmallCtaMax = 16;
static_assert(kNumClasses == kMaxClasses, "ClassLists holds every class");
int ClassOf(int type) {
  switch (type) {
    case kDCT:
    case kDCT_NOHF:
      return kC8;
    case kDCT16X16:
      return kC16;
    case kDCT32X32:
      return kC32;
    case kDCT4X4:
    case kDCT4X4_NOHF:
      return kC4;
    default:
      return kCSmall;
  }
}

// Kernel groups timed with events when profiling is on.
enum Timed {
  kTDc = 0, kTDequant, kTLf, kTIdct, kTGab1, kTEpf, kTAr, kTFinal, kNumTimed
};
const char* kTimedNames[kNumTimed] = {
    "dc_dequant_epf", "dequant_ac", "lf_prediction_update", "hf_idct",
    "gaborish1_minmax", "epf", "ar_clamp", "gaborish2_opsin_srgb"};

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

std::mutex g_table_mutex;
bool g_tables_uploaded[64] = {};

// Persistent tensor-core transform CTAs per SM (default): 4 x 128
// tensor-memory columns fill the SM's 512. A batch's autotuner may lower it
// (pikgpu_batch_autotune).
constexpr int kTcCtasPerSm = 4;

}  // namespace

struct pikgpu_ctx {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  // Last error message; Fail() may run on several host threads at once
  // (concurrent pikgpu_frame_set_group_ac calls).
  std::string err;
  std::mutex err_mu;
  bool have_frame = false, have_result = false;
  // Set by every AC upload; group uploads may run on several host threads.
  std::atomic<bool> have_ac{false};
  // The caller's device AC planes, read in place (pikgpu_frame_set_ac_device
  // with the context's own layout); NULL: the context's copy in `qac`.
  const int16_t* qac_in = nullptr;
  bool keep_stages = false, profile = false;
  int form = PIKGPU_FORM_FP32;
  Geo g{};
  FrameScalars s{};
  // host copies needed after begin
  std::vector<uint32_t> lists[kNumClasses];
  // device buffers
  DevBuf acs, qf, lut, dq_cf, dq_map, ytox, ytob, table, offsets;
  DevBuf qdc, qac, dc, dcpad, ac, pred2x2_g;
  DevBuf idct, smoothed, filt, mm, sigma, dc_sigma, list[kNumClasses];
  DevBuf out_lin, out_rgb8, dbg_dequant, dbg_epf, dbg_pre, guide_ovr, pnm;
  // Linear planes of the last reconstruction (device; NULL if it wrote
  // none), for pikgpu_encode_pnm.
  const float* last_lin = nullptr;
  size_t last_lin_stride = 0;
  DevBuf sigma_ovr, counters, active[kNumClasses], tc_err;
  bool use_guide_ovr = false, use_sigma_ovr = false;
  // Dequantised AC supplied by the caller instead of Dequant::DoAC, and the
  // per-cell clamp scale (pikgpu_frame_set_dequantized_ac / _clamp_scale).
  DevBuf dq_ovr, clamp_scale;
  bool use_dq_ovr = false, use_clamp_scale = false;
  // Adjoint (adjoint.cu): gradient planes, coefficient gradient, group
  // pred2x2 gradient, quant-field gradient, guide bytes, loss partials,
  // per-type Jacobians, host target staging.
  DevBuf adj_a, adj_b, adj_c, adj_coef, adj_pred, adj_qf, adj_guide;
  DevBuf adj_partial, adj_jac, adj_target, adj_tape;
  bool adj_jac_built = false;
  // The clamp kernels record their branches (the clamp tape) in the
  // adjoint's forward pass and with PIKGPU_OPT_KEEP_STAGES; tape_valid: the
  // last forward pass wrote adj_tape. tape_in: branches to follow
  // (pikgpu_set_clamp_decisions).
  bool record_tape = false, tape_valid = false;
  DevBuf tape_in;
  bool use_tape_in = false;
  // The smoothed frame (gaborish #1) is written only when an export asks.
  bool smoothed_valid = false;
  cudaEvent_t ev[kNumTimed + 1] = {};
  // Side streams and fork/join events of the launch sequence's concurrent
  // branches (LaunchAll).
  static constexpr int kSide = 4;
  cudaStream_t side[kSide] = {};
  cudaEvent_t fork_ev[3] = {}, join_ev[3][kSide] = {};
  int num_sms = 148;
  int tc_ctas_per_sm = kTcCtasPerSm;
  // PIKGPU_OPT_TC_WAIT_POLLS.
  uint32_t tc_polls = tc::kMaxPolls;
  float times[kNumTimed] = {};
  float dc_half_step[3] = {};
  int launches = 0;
  // Bumped by every call that changes what the launch sequence does or
  // which buffers it uses, and by every device (re)allocation: a captured
  // graph (single frame or batch) is then stale.
  uint64_t generation = 0;
  // Single-frame graph replay (PIKGPU_OPT_GRAPHS): the launch state of the
  // last pikgpu_reconstruct call, and its graph once a call repeated it.
  struct GraphKey {
    uint64_t generation;
    const int16_t* qac_in;
    float* lin;
    size_t lin_stride;
    uint8_t* rgb8;
    size_t rgb8_stride;
    cudaStream_t stream;
    int tc_ctas;
    bool operator==(const GraphKey& o) const {
      return generation == o.generation && qac_in == o.qac_in &&
             lin == o.lin &&
             lin_stride == o.lin_stride && rgb8 == o.rgb8 &&
             rgb8_stride == o.rgb8_stride && stream == o.stream &&
             tc_ctas == o.tc_ctas;
    }
  };
  bool use_graphs = true, have_key = false;
  GraphKey key{};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  int graph_launches = 0, graph_captures = 0;
  bool graph_tape_valid = false, last_replayed = false;
  // Pinned host word the tensor-core error flag is read back into.
  int* tc_err_host = nullptr;
  // pikgpu_reconstruct_async enqueued work that pikgpu_wait has not yet
  // finished (with the tensor-core flag to check).
  bool pending = false;
};

namespace {

int Fail(pikgpu_ctx* ctx, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) {
    std::lock_guard<std::mutex> lock(ctx->err_mu);
    ctx->err = buf;
  }
  return code;
}

// Every call but pikgpu_wait refuses a context whose asynchronous
// reconstruction has not been waited for.
#define PIKGPU_NOT_PENDING(ctx)                                             \
  do {                                                                      \
    if ((ctx)->pending) {                                                   \
      return Fail(ctx, PIKGPU_ERR_STATE,                                    \
                  "reconstruction in flight: call pikgpu_wait first");      \
    }                                                                       \
  } while (0)

#define CUDA_TRY(ctx, call)                                                 \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) {                                                \
      return Fail(ctx, PIKGPU_ERR_CUDA, "%s: %s", #call,                    \
                  cudaGetErrorString(e_));                                  \
    }                                                                       \
  } while (0)

int Ensure(pikgpu_ctx* ctx, DevBuf* b, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (b->cap >= bytes) return PIKGPU_OK;
  if (b->p) cudaFree(b->p);
  b->p = nullptr;
  b->cap = 0;
  if (ctx) ++ctx->generation;
  const cudaError_t e = cudaMalloc(&b->p, bytes);
  if (e != cudaSuccess) {
    return Fail(ctx, PIKGPU_ERR_NO_MEMORY, "cudaMalloc(%zu): %s", bytes,
                cudaGetErrorString(e));
  }
  b->cap = bytes;
  return PIKGPU_OK;
}

void FreeBuf(DevBuf* b) {
  if (b->p) cudaFree(b->p);
  b->p = nullptr;
  b->cap = 0;
}

template <typename T>
T* P(const DevBuf& b) {
  return static_cast<T*>(b.p);
}

constexpr int kRequiredSize[7] = {1, 1, 1, 1, 2, 4, 1};

// Host-side validation shared by pikgpu_frame_begin and pikgpu_validate.
int Validate(pikgpu_ctx* ctx, const pikgpu_frame_params* p) {
  if (!p) return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "params is NULL");
  if (p->xsize == 0 || p->ysize == 0) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "empty image %ux%u", p->xsize,
                p->ysize);
  }
  if (p->xsize > (1u << 18) || p->ysize > (1u << 18)) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "image %ux%u too large",
                p->xsize, p->ysize);
  }
  if (!p->dequant_table || !p->dequant_offsets || !p->dequant_control_field ||
      !p->dequant_map || !p->ytox_map || !p->ytob_map || !p->ac_strategy ||
      !p->raw_quant_field || !p->ar_sigma_lut_ids || !p->quantized_dc) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "NULL array in params");
  }
  if (p->flags != 0) {
    return Fail(ctx, PIKGPU_ERR_UNSUPPORTED,
                "FrameHeader flags 0x%x (noise/gradient/grayscale/...) are "
                "not supported",
                p->flags);
  }
  if (p->gaborish > PIKGPU_GABORISH_1000) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "gaborish strength %u",
                p->gaborish);
  }
  // Fixed-sigma EPF filters with kMinSigma <= sigma <= kMaxSigma, or copies
  // when sigma is 0 (FilterWorkers and Filter, pik/epf_target.cc:1295,
  // 1357-1361).
  if (p->have_adaptive_reconstruction && !p->epf_enable_adaptive &&
      p->epf_sigma != 0 &&
      (p->epf_sigma < uint32_t(kMinSigma) ||
       p->epf_sigma > uint32_t(kMaxSigma))) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG,
                "fixed EPF sigma %u outside {0} and [%d, %d]", p->epf_sigma,
                kMinSigma, kMaxSigma);
  }
  if (p->global_scale < 1 || p->global_scale > 32768) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "global_scale %d",
                p->global_scale);
  }
  if (p->quant_dc < 1 || p->quant_dc > 256) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "quant_dc %d", p->quant_dc);
  }
  if (p->num_dequant_tables < 1 || p->num_dequant_tables > 256) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "num_dequant_tables %u",
                p->num_dequant_tables);
  }
  for (uint32_t t = 0; t < p->num_dequant_tables; ++t) {
    for (int k = 0; k < 7; ++k) {
      for (int c = 0; c < 3; ++c) {
        const uint64_t off = p->dequant_offsets[(t * 7 + k) * 3 + c];
        const uint64_t need = 64ull * kRequiredSize[k] * kRequiredSize[k];
        if (off + need > p->dequant_table_size) {
          return Fail(ctx, PIKGPU_ERR_INVALID_ARG,
                      "dequant offset %llu (table %u kind %d c %d) beyond "
                      "table of %u floats",
                      (unsigned long long)off, t, k, c,
                      p->dequant_table_size);
        }
      }
    }
  }
  const int bx = (p->xsize + 7) / 8, by = (p->ysize + 7) / 8;
  const int tx = (p->xsize + 63) / 64, ty = (p->ysize + 63) / 64;
  for (int i = 0; i < tx * ty; ++i) {
    if (p->dequant_control_field[i] >= PIKGPU_MAX_QUANT_CONTROL_FIELD) {
      return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "dequant control field %u",
                  p->dequant_control_field[i]);
    }
  }
  for (int i = 0; i < 16 * 256; ++i) {
    if (p->dequant_map[i] >= p->num_dequant_tables) {
      return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "dequant_map entry %u >= %u",
                  p->dequant_map[i], p->num_dequant_tables);
    }
  }
  // AcStrategyImage consistency (pik/ac_strategy.h:95-97, 315-356).
  std::vector<uint8_t> expect(size_t(bx) * by, 0xFF);
  for (int y = 0; y < by; ++y) {
    for (int x = 0; x < bx; ++x) {
      const uint8_t a = p->ac_strategy[y * bx + x];
      const int type = a >> 4, blk = a & 0xF;
      if (type > 8) {
        return Fail(ctx, PIKGPU_ERR_INVALID_ARG,
                    "invalid AcStrategy %d at block (%d, %d)", type, x, y);
      }
      const int q = p->raw_quant_field[y * bx + x];
      if (q < 1 || q > 256) {
        return Fail(ctx, PIKGPU_ERR_INVALID_ARG,
                    "quant field %d at block (%d, %d) outside [1, 256]", q, x,
                    y);
      }
      if (p->ar_sigma_lut_ids[y * bx + x] > 1) {
        return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "EPF LUT id %u at (%d, %d)",
                    p->ar_sigma_lut_ids[y * bx + x], x, y);
      }
      if (blk != 0) continue;
      const int cov = Covered(type);
      if (cov > 1 && ((x % cov) != 0 || (y % cov) != 0)) {
        return Fail(ctx, PIKGPU_ERR_UNSUPPORTED,
                    "%dx%d transform at block (%d, %d) is not aligned to its "
                    "size",
                    8 * cov, 8 * cov, x, y);
      }
      if (x + cov > bx || y + cov > by) {
        return Fail(ctx, PIKGPU_ERR_INVALID_ARG,
                    "transform at (%d, %d) extends past the image", x, y);
      }
      for (int iy = 0; iy < cov; ++iy) {
        for (int ix = 0; ix < cov; ++ix) {
          uint8_t& e = expect[size_t(y + iy) * bx + x + ix];
          if (e != 0xFF) {
            return Fail(ctx, PIKGPU_ERR_INVALID_ARG,
                        "overlapping transforms at block (%d, %d)", x + ix,
                        y + iy);
          }
          e = uint8_t((type << 4) | (iy * cov + ix));
        }
      }
    }
  }
  for (size_t i = 0; i < expect.size(); ++i) {
    if (expect[i] != p->ac_strategy[i]) {
      return Fail(ctx, PIKGPU_ERR_INVALID_ARG,
                  "AcStrategy sub-block index inconsistent at block (%zu, "
                  "%zu)",
                  i % bx, i / bx);
    }
  }
  return PIKGPU_OK;
}

void ComputeScalars(const pikgpu_frame_params* p, FrameScalars* s) {
  // Quantizer::RecomputeFromGlobalScale + Decode (pik/quantizer.h:130-135,
  // pik/quantizer.cc:63-71).
  s->inv_global_scale = static_cast<float>(1.0 * 65536 / p->global_scale);
  s->inv_quant_dc = s->inv_global_scale / p->quant_dc;
  for (int c = 0; c < 3; ++c) {
    s->mul_dc[c] =
        p->dequant_table[p->dequant_offsets[c]] * s->inv_quant_dc;
  }
  s->ytox_dc = 1.0f * float(p->ytox_dc - 128) * (1.0f / 256);
  s->ytob_dc = 1.0f * float(p->ytob_dc) * (1.0f / 128);
  s->gaborish = p->gaborish;
  s->predict_lf = p->predict_lf ? 1 : 0;
  s->predict_hf = p->predict_hf ? 1 : 0;
  s->have_ar = p->have_adaptive_reconstruction ? 1 : 0;
  s->use_sharpened = p->epf_use_sharpened ? 1 : 0;
  s->quant_dc = p->quant_dc;
  s->epf_fixed_sigma = p->epf_enable_adaptive ? -1 : int(p->epf_sigma);
}

int UploadTables(pikgpu_ctx* ctx) {
  std::lock_guard<std::mutex> lock(g_table_mutex);
  if (ctx->device < 64 && g_tables_uploaded[ctx->device]) return PIKGPU_OK;
  DevTables t;
  BuildTables(&t);
  CUDA_TRY(ctx, cudaMemcpyToSymbol(c_t, &t, sizeof(t)));
  CUDA_TRY(ctx, cudaFuncSetAttribute(
                    k_epf_box<false, 32>,
                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                    int(EpfSmemBytes(32))));
  CUDA_TRY(ctx, cudaFuncSetAttribute(
                    k_epf_box<false, 8>,
                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                    int(EpfSmemBytes(8))));
  CUDA_TRY(ctx, cudaFuncSetAttribute(
                    k_epf_box<true, 16>,
                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                    int(EpfSmemBytes(16))));
  CUDA_TRY(ctx, cudaFuncSetAttribute(
                    k_epf_box<true, 8>,
                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                    int(EpfSmemBytes(8))));
  CUDA_TRY(ctx, cudaFuncSetAttribute(
                    k_lf_tile, cudaFuncAttributeMaxDynamicSharedMemorySize,
                    int(kLfSmemBytes)));
  CUDA_TRY(ctx, cudaFuncSetAttribute(
                    k_square_ar_tc<16, 2>,
                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                    int(ArTcSmemBytes<16, 2>())));
  CUDA_TRY(ctx, cudaFuncSetAttribute(
                    k_square_ar_tc<16, 3>,
                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                    int(ArTcSmemBytes<16, 3>())));
  CUDA_TRY(ctx, cudaFuncSetAttribute(
                    k_square_ar_tc<32, 3>,
                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                    int(ArTcSmemBytes<32, 3>())));
  if (ctx->device < 64) g_tables_uploaded[ctx->device] = true;
  return PIKGPU_OK;
}

inline int Blocks(size_t n, int t) { return int((n + t - 1) / t); }


// Writes the smoothed frame (gaborish #1 of the IDCT output) for the stage
// and guide exports; the reconstruction itself never stores it.
int EnsureSmoothed(pikgpu_ctx* ctx) {
  if (ctx->smoothed_valid || !ctx->s.gaborish) return PIKGPU_OK;
  const Geo& g = ctx->g;
  const int rc = Ensure(ctx, &ctx->smoothed, 4 * 3 * size_t(g.PW) * g.PH);
  if (rc != PIKGPU_OK) return rc;
  dim3 gr(Blocks(g.PW, kTileW), Blocks(g.PH, kGabTileH), 3);
  k_gaborish_tile<<<gr, kTileThreads, 0, ctx->stream>>>(
      P<float>(ctx->idct), g.PW, g.PH, ctx->s.gaborish,
      P<float>(ctx->smoothed), nullptr);
  CUDA_TRY(ctx, cudaGetLastError());
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->smoothed_valid = true;
  return PIKGPU_OK;
}

void Mark(pikgpu_ctx* ctx, int i) {
  if (ctx->profile) cudaEventRecord(ctx->ev[i], ctx->stream);
}

// Launches `kernel` on `st`; with `pdl`, as a programmatic dependent of the
// kernel before it on the stream
// (cudaLaunchAttributeProgrammaticStreamSerialization): it may then start
// once every CTA of that kernel has begun (PdlLaunchDependents), and it
// orders itself after that kernel's completion with griddepcontrol.wait
// (PdlWait or PdlTail in the kernel).
template <typename... KArgs, typename... Args>
cudaError_t LaunchPdl(bool pdl, void (*kernel)(KArgs...), int grid, int block,
                      size_t smem, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr = {};
  attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr.val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = pdl ? &attr : nullptr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// The frame EPF or the DC EPF: the min/max of the guide source is expected
// in `mm` already. `sgs`: where the per-block sigma comes from (computed in
// the kernel); `dco`: the DC image's clamped output instead of `out`.
// `gab` > 0: the guide is gaborish (that strength) of `in`, computed inside
// the kernel.
// The wait that ran out, from the context's timeout flag: 1 from the
// tensor-core kernels' MMA completion waits, 2 from the EPF's tile copy.
const char* WaitTimeoutMessage(int code) {
  return code == 2 ? "EPF: TMA tile copy wait timed out"
                   : "tensor-core transform: MMA completion wait timed out";
}

// cuTensorMapEncodeTiled from the driver, found through the runtime's
// entry-point query (no link-time dependency on libcuda); NULL if the
// driver has none.
PFN_cuTensorMapEncodeTiled_v12000 TensorMapEncoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p,
                                cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      return PFN_cuTensorMapEncodeTiled_v12000(nullptr);
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// The EPF's tile map over the three w x h planes at `in` (boxes of th + 10
// rows x kEpfTW columns x 3 planes, the layout of k_epf_box's staged tile).
// False if it cannot be made: no driver entry point, `in` not 16-byte
// aligned, rows not a multiple of 16 bytes, or the encoder refuses.
bool EpfTileMap(CUtensorMap* m, const float* in, int w, int h, int th) {
  const auto enc = TensorMapEncoder();
  if (!enc || (reinterpret_cast<uintptr_t>(in) & 15) || (w % 4) ||
      w < kEpfTW || h < th + 10) {
    return false;
  }
  const cuuint64_t dims[3] = {cuuint64_t(w), cuuint64_t(h), 3};
  const cuuint64_t strides[2] = {cuuint64_t(w) * 4,
                                 cuuint64_t(w) * cuuint64_t(h) * 4};
  const cuuint32_t box[3] = {cuuint32_t(kEpfTW), cuuint32_t(th + 10), 3};
  const cuuint32_t elem[3] = {1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(in),
             dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// `err`: the context's wait-timeout flag (k_epf_box's TMA wait sets 2),
// `polls` the first wait's limit; err NULL: no TMA staging.
void EpfLaunch(cudaStream_t st, int num_sms, int form, const float* in,
               const float* guide_src, int gab, int w, int h,
               const uint32_t* mm, const EpfSigma& sgs, float* out,
               const uint8_t* guide_ovr, const EpfDc& dco, int* err,
               uint32_t polls = tc::kMaxPolls, bool pdl = false) {
  // Images that fill fewer than two CTAs per SM with 32-row tiles (the DC
  // image) take 8-row tiles: four times the CTAs, a quarter of the latency.
  const bool small = Blocks(w, kEpfW) * Blocks(h, kEpfH) < 2 * num_sms;
  const bool fma = form != PIKGPU_FORM_FP32;
  // One CTA per 64 x th tile.
  auto grid = [&](int th) { return Blocks(w, kEpfW) * Blocks(h, th); };
  const int th = small ? 8 : fma ? 16 : kEpfH;
  CUtensorMap map;
  memset(&map, 0, sizeof(map));
  const int tma = err && EpfTileMap(&map, in, w, h, th) ? 1 : 0;
  // Errors of the launch surface through cudaGetLastError.
  if (small) {
    if (fma) {
      LaunchPdl(pdl, k_epf_box<true, 8>, grid(8), 16 * 8, EpfSmemBytes(8), st,
                in, guide_src, guide_ovr, gab, w, h, mm, sgs, out, dco, map,
                tma, err, polls);
    } else {
      LaunchPdl(pdl, k_epf_box<false, 8>, grid(8), 16 * 8, EpfSmemBytes(8),
                st, in, guide_src, guide_ovr, gab, w, h, mm, sgs, out, dco,
                map, tma, err, polls);
    }
  } else {
    if (fma) {
      // 16-row tiles of 256 threads, three CTAs per SM: the cx-major loop
      // of these forms needs ~85 registers.
      LaunchPdl(pdl, k_epf_box<true, 16>, grid(16), 16 * 16,
                EpfSmemBytes(16), st, in, guide_src, guide_ovr, gab, w, h, mm,
                sgs, out, dco, map, tma, err, polls);
    } else {
      LaunchPdl(pdl, k_epf_box<false, kEpfH>, grid(kEpfH), kEpfThreads,
                kEpfSmemBytes, st, in, guide_src, guide_ovr, gab, w, h, mm,
                sgs, out, dco, map, tma, err, polls);
    }
  }
}

// Concurrent branches of the launch sequence. Fork(i, n) makes side streams
// 0..n-1 wait for the main stream's work so far; Join(i, n) makes the main
// stream wait for theirs. Without branches (profiling, whose per-group
// event times need one stream) every branch is the main stream and both
// are no-ops. Events are recorded and waited in stream order, so this also
// holds inside a stream capture (the branches become graph dependencies).
struct Branches {
  pikgpu_ctx* ctx;
  bool on;
  cudaStream_t main;
  cudaStream_t operator[](int i) const {
    return on ? ctx->side[i] : main;
  }
  void Fork(int i, int n) const {
    if (!on) return;
    cudaEventRecord(ctx->fork_ev[i], main);
    for (int k = 0; k < n; ++k) cudaStreamWaitEvent(ctx->side[k], ctx->fork_ev[i], 0);
  }
  void Join(int i, int n) const {
    if (!on) return;
    for (int k = 0; k < n; ++k) {
      cudaEventRecord(ctx->join_ev[i][k], ctx->side[k]);
      cudaStreamWaitEvent(main, ctx->join_ev[i][k], 0);
    }
  }
};

// The transform classes other than DCT8 (and later their clamps) as one
// chain of kernels on one stream. Each kernel after the first is launched
// as a programmatic dependent of the one before it
// (cudaLaunchAttributeProgrammaticStreamSerialization): it may start once
// every CTA of its predecessor has begun, and it waits for the
// predecessor's completion before it exits (PdlLaunchDependents and
// PdlTail in the kernels). The first is an ordinary launch, so the chain
// starts after everything before it. Launched in the order given, the
// few-block classes are resident before the persistent tensor-core kernels
// take the SMs, in a graph replay too, whose branches start in an order of
// the runtime's choosing.
struct ClassChain {
  cudaStream_t st;
  int* launches;
  bool pdl;  // false: ordinary launches, each after the one before
  bool started = false;
  cudaError_t err = cudaSuccess;
  template <typename... KArgs, typename... Args>
  void operator()(void (*kernel)(KArgs...), int grid, int block, size_t smem,
                  Args... args) {
    const cudaError_t e =
        LaunchPdl(pdl && started, kernel, grid, block, smem, st, args...);
    if (e != cudaSuccess && err == cudaSuccess) err = e;
    started = true;
    ++*launches;
  }
};

// The launch sequence of one frame. Its DAG:
//   side 0: DC dequant, DC EPF and clamp
//   main:   AC dequantisation            (both from the inputs only)
//   main:   LLF / LF update, pred2x2      (joins the two)
//   main:   the DCT8 inverse transforms, beside
//   side 0: the other classes' inverse transforms (ClassChain; the classes'
//           blocks are disjoint)
//   main:   gaborish minmax, sigma, EPF
//   main + side 0: the clamp, split the same way
//   main:   gaborish #2, opsin, outputs
//
// `single_stream`: everything on the main stream (the events become no-ops).
// The batch captures its frames that way: the frames themselves run as
// concurrent branches, and without per-frame branches the 64-frame batch
// took 7.23 ms against 7.40.
int LaunchAll(pikgpu_ctx* ctx, float* lin, size_t lin_stride, uint8_t* rgb8,
              size_t rgb8_stride, bool single_stream = false) {
  const Geo& g = ctx->g;
  const FrameScalars& s = ctx->s;
  cudaStream_t st = ctx->stream;
  const Branches br{ctx, !ctx->profile && !single_stream, st};
  DevFrame f;
  f.acs = P<uint8_t>(ctx->acs);
  f.qf = P<int32_t>(ctx->qf);
  f.lut = P<uint8_t>(ctx->lut);
  f.dq_cf = P<uint8_t>(ctx->dq_cf);
  f.dq_map = P<uint8_t>(ctx->dq_map);
  f.ytox = P<int32_t>(ctx->ytox);
  f.ytob = P<int32_t>(ctx->ytob);
  f.table = P<float>(ctx->table);
  f.offsets = P<uint32_t>(ctx->offsets);
  f.qdc = P<int16_t>(ctx->qdc);
  f.qac = ctx->qac_in ? ctx->qac_in : P<int16_t>(ctx->qac);
  f.dc = P<float>(ctx->dc);
  f.ac = P<float>(ctx->ac);
  f.pred2x2_g = P<float>(ctx->pred2x2_g);
  f.idct = P<float>(ctx->idct);
  f.smoothed = P<float>(ctx->smoothed);
  f.filt = P<float>(ctx->filt);
  f.clamp_scale = ctx->use_clamp_scale ? P<float>(ctx->clamp_scale) : nullptr;
  const size_t nac = size_t(g.ac_stride) * g.By;
  const bool rec = (ctx->record_tape || ctx->keep_stages) && s.have_ar &&
                   ctx->adj_tape.cap >= nac;
  f.clamp_tape = rec ? P<uint8_t>(ctx->adj_tape) : nullptr;
  f.clamp_tape_in = ctx->use_tape_in ? P<uint8_t>(ctx->tape_in) : nullptr;
  f.tc_polls = ctx->tc_polls;
  ctx->tape_valid = rec;
  uint32_t* mm = P<uint32_t>(ctx->mm);
  const uint32_t* L[kNumClasses];
  int n[kNumClasses];
  for (int k = 0; k < kNumClasses; ++k) {
    L[k] = P<uint32_t>(ctx->list[k]);
    n[k] = int(ctx->lists[k].size());
  }

  ctx->launches = 0;
  ctx->smoothed_valid = false;
  // Both min/max sets and the clamp's block counters start empty.
  int* counters = P<int>(ctx->counters);
  k_frame_init<<<1, 32, 0, st>>>(mm, counters, kNumCounters); ++ctx->launches;
  br.Fork(0, 1);
  Mark(ctx, kTDc);
  // DC (side stream 0): dequantisation, the 8-padded copy and its min/max;
  // then the EPF on it, which clamps its output into the DC planes.
  cudaStream_t sd = br[0];
  const int dpw = (g.Bx + 7) / 8 * 8, dph = (g.By + 7) / 8 * 8;
  float* dcpad = P<float>(ctx->dcpad);
  uint32_t* mm_dc = mm + 8;
  {
    k_dc_prep<<<dim3(Blocks(dpw, 32), Blocks(dph, 8)), 256, 0, sd>>>(
        g, f, s, dcpad, dpw, dph, mm_dc); ++ctx->launches;
    EpfSigma sgs{};
    sgs.const_qf = s.quant_dc / 2;
    sgs.fixed = -1;
    sgs.out = P<int32_t>(ctx->dc_sigma);
    const EpfDc dco{f.dc, g.Bx, g.By, ctx->dc_half_step[0],
                    ctx->dc_half_step[1], ctx->dc_half_step[2]};
    EpfLaunch(sd, ctx->num_sms, ctx->form, dcpad, dcpad, 0, dpw, dph, mm_dc,
              sgs, nullptr, nullptr, dco, P<int>(ctx->tc_err), ctx->tc_polls);
    ++ctx->launches;
  }
  Mark(ctx, kTDequant);
  {
    // AC dequantisation (main stream, concurrent with DC).
    if (ctx->use_dq_ovr) {
      cudaMemcpyAsync(f.ac, ctx->dq_ovr.p,
                      sizeof(float) * 3 * size_t(g.ac_stride) * g.By,
                      cudaMemcpyDeviceToDevice, st);
    } else {
      dim3 gr(Blocks(g.Bx, kDequantCells), g.By);
      k_dequant_ac<<<gr, 256, 0, st>>>(g, f, s); ++ctx->launches;
    }
    if (ctx->keep_stages) {
      cudaMemcpyAsync(ctx->dbg_dequant.p, f.ac,
                      sizeof(float) * 3 * size_t(g.ac_stride) * g.By,
                      cudaMemcpyDeviceToDevice, st);
    }
    br.Join(0, 1);
  }
  Mark(ctx, kTLf);
  // Per-group LF prediction and the LF update of every block's dequantised
  // coefficients, with its pred2x2 (after DC and the dequantisation): one
  // CTA per tile of 32 x 32 cells of a group and channel.
  const int ng = g.Gx * g.Gy;
  constexpr int kTilesPerGroup = (64 + kLfTile - 1) / kLfTile;
  k_lf_tile<<<dim3(kTilesPerGroup * kTilesPerGroup, ng, 3), kLfThreads,
              kLfSmemBytes, st>>>(g, f, s.predict_lf, s.predict_hf);
  ++ctx->launches;
  Mark(ctx, kTIdct);
  br.Fork(1, 1);
  {
    auto rows_grid = [](int items, int n) {
      const int upw = 32 / n;
      const int warps = (items + upw - 1) / upw;
      return (warps * 32 + kSquareThreads - 1) / kSquareThreads;
    };
    // DCT8 on the main stream; the other classes as one chain on a side
    // stream, the classes with few blocks first, so that their CTAs are
    // resident before the persistent tensor-core kernels fill the SMs
    // (which take their work from a counter and leave those SMs' share to
    // the others).
    if (n[kC8]) {
      k_square_idct_rows<8><<<rows_grid(3 * n[kC8], 8), kSquareThreads, 0,
                              st>>>(g, f, L[kC8], n[kC8], s.predict_hf);
      ++ctx->launches;
    }
    ClassChain ch{br[0], &ctx->launches, !ctx->profile};
    if (n[kCSmall]) {
      if (n[kCSmall] <= kSmallCtaMax * ctx->num_sms) {
        ch(k_small_idct_cta, n[kCSmall], kSmallCtaThreads, 0, g, f,
           L[kCSmall], n[kCSmall]);
      } else {
        ch(k_small_idct, Blocks(3 * n[kCSmall], kSmallIdctThreads),
           kSmallIdctThreads, 0, g, f, L[kCSmall], n[kCSmall]);
      }
    }
    if (n[kC4]) {
      ch(k_dct4_idct, Blocks(3 * n[kC4], kDct4Threads / 8), kDct4Threads, 0,
         g, f, L[kC4], n[kC4], s.predict_hf);
    }
    if (n[kC32] && ctx->form != PIKGPU_FORM_FP32) {
      // One channel per CTA: four blocks of 32 rows per batch, up to
      // tc_ctas_per_sm CTAs per SM (registers). Both tensor-core forms
      // split the 32-point operands in three BF16 terms: with two, a frame
      // without HF prediction reached 3.0e-5 against FP64.
      const int items = 3 * ((n[kC32] + 3) / 4);
      const int grid = std::min(items, ctx->num_sms * ctx->tc_ctas_per_sm);
      ch(k_square_idct_tc1<32, 3>, grid, tc::kThreads, 0, g, f, L[kC32],
         n[kC32], s.predict_hf, counters + kWorkIdct32, P<int>(ctx->tc_err));
    } else if (n[kC32]) {
      // One 256-thread CTA per block.
      ch(k_square_idct<32>, n[kC32], 256, 0, g, f, L[kC32], n[kC32],
         s.predict_hf);
    }
    if (n[kC16] && ctx->form != PIKGPU_FORM_FP32) {
      const int items = (n[kC16] + 7) / 8;
      // One channel per CTA: up to 2 tc_ctas_per_sm CTAs per SM.
      const int grid =
          std::min(3 * items, ctx->num_sms * 2 * ctx->tc_ctas_per_sm);
      // Two BF16 terms hold 2e-5 against FP64 only when the HF prediction
      // carries the bulk of the coefficients (it is added in FP32 outside
      // the tensor cores); frames without it take three terms.
      if (ctx->form == PIKGPU_FORM_SPLIT_BF16 && s.predict_hf) {
        ch(k_square_idct_tc1<16, 2>, grid, tc::kThreads, 0, g, f, L[kC16],
           n[kC16], s.predict_hf, counters + kWorkIdct, P<int>(ctx->tc_err));
      } else {
        ch(k_square_idct_tc1<16, 3>, grid, tc::kThreads, 0, g, f, L[kC16],
           n[kC16], s.predict_hf, counters + kWorkIdct, P<int>(ctx->tc_err));
      }
    } else if (n[kC16]) {
      ch(k_square_idct_rows<16>, rows_grid(3 * n[kC16], 16), kSquareThreads,
         0, g, f, L[kC16], n[kC16], s.predict_hf);
    }
    CUDA_TRY(ctx, ch.err);
  }
  br.Join(1, 1);
  const float* final_in = f.idct;
  Mark(ctx, kTGab1);
  if (s.have_ar) {
    const size_t npx = size_t(g.PW) * g.PH;
    // Guide source: gaborish of the IDCT output (computed inside the EPF;
    // here only its min/max), or the IDCT output itself (sharpened guide,
    // or no gaborish).
    const int gab = s.use_sharpened ? 0 : s.gaborish;
    // The clamp tape starts empty (written by the clamp kernels only).
    if (f.clamp_tape) cudaMemsetAsync(f.clamp_tape, 0, nac, st);
    // The EPF, and after it the active-block pass, as programmatic
    // dependents of the kernel before each (LaunchPdl) when nothing else
    // lies between them on the stream (no per-group events, no stage copy).
    const bool pdl = !ctx->profile && !ctx->keep_stages;
    if (gab) {
      const int warps = Blocks(g.PW, 128) * Blocks(g.PH, kGmmRows);
      k_gaborish_minmax<<<dim3(Blocks(warps, 8), 3), 256, 0, st>>>(
          f.idct, g.PW, g.PH, gab, mm); ++ctx->launches;
    } else {
      k_minmax<<<dim3(Blocks(npx, 256 * 8), 3), 256, 0, st>>>(f.idct, npx,
                                                               mm); ++ctx->launches;
    }
    Mark(ctx, kTEpf);
    int32_t* sig = P<int32_t>(ctx->sigma);
    EpfSigma sgs{};
    sgs.ovr = ctx->use_sigma_ovr ? P<int32_t>(ctx->sigma_ovr) : nullptr;
    sgs.qf = f.qf;
    sgs.acs = f.acs;
    sgs.lut = f.lut;
    sgs.fixed = s.epf_fixed_sigma;
    sgs.out = sig;
    EpfLaunch(st, ctx->num_sms, ctx->form, f.idct, f.idct, gab, g.PW, g.PH,
              mm, sgs, f.filt,
              ctx->use_guide_ovr ? P<uint8_t>(ctx->guide_ovr) : nullptr,
              EpfDc{}, P<int>(ctx->tc_err), ctx->tc_polls, pdl);
    ++ctx->launches;
    if (ctx->keep_stages) {
      cudaMemcpyAsync(ctx->dbg_epf.p, f.filt, sizeof(float) * 3 * npx,
                      cudaMemcpyDeviceToDevice, st);
    }
    Mark(ctx, kTAr);
    // Only blocks the EPF filtered need the clamp (see k_active_blocks).
    // Every class's filtered blocks in one pass (main stream), then the
    // classes' clamps, the ones with few blocks first (see the transforms).
    {
      ClassLists cl{};
      int total = 0;
      for (int k = 0; k < kNumClasses; ++k) {
        cl.list[k] = L[k];
        cl.n[k] = n[k];
        cl.active[k] = P<uint32_t>(ctx->active[k]);
        total += n[k];
      }
      if (total) {
        CUDA_TRY(ctx, LaunchPdl(pdl, k_active_blocks, Blocks(total, 256), 256,
                                0, st, g, sig, f.acs, cl, counters));
        ++ctx->launches;
      }
    }
    br.Fork(2, 1);
    auto rows_grid = [](int items, int nn) {
      const int upw = 32 / nn;
      const int warps = (items + upw - 1) / upw;
      return (warps * 32 + kSquareThreads - 1) / kSquareThreads;
    };
    if (n[kC8]) {
      k_square_ar_rows<8><<<rows_grid(n[kC8], 8), kSquareThreads, 0, st>>>(
          g, f, s, P<uint32_t>(ctx->active[kC8]), counters + kC8);
      ++ctx->launches;
    }
    ClassChain ch{br[0], &ctx->launches, !ctx->profile};
    if (n[kCSmall]) {
      if (n[kCSmall] <= kSmallCtaMax * ctx->num_sms) {
        ch(k_small_ar_cta, n[kCSmall], kSmallCtaThreads, 0, g, f, s,
           P<uint32_t>(ctx->active[kCSmall]), counters + kCSmall);
      } else {
        ch(k_small_ar, Blocks(n[kCSmall], kSmallArBlocks),
           3 * kSmallArBlocks, 0, g, f, s,
           P<uint32_t>(ctx->active[kCSmall]), counters + kCSmall);
      }
    }
    if (n[kC4]) {
      ch(k_dct4_ar, Blocks(n[kC4], kDct4ArThreads / 32), kDct4ArThreads, 0,
         g, f, s, P<uint32_t>(ctx->active[kC4]), counters + kC4);
    }
    if (n[kC32] && ctx->form != PIKGPU_FORM_FP32) {
      // Four blocks per batch; two CTAs per SM (256 tensor-memory columns
      // each); three BF16 terms in both tensor-core forms (see the
      // transforms).
      const int grid = std::min((n[kC32] + 3) / 4, ctx->num_sms * 2);
      ch(k_square_ar_tc<32, 3>, grid, tc::kThreads, ArTcSmemBytes<32, 3>(),
         g, f, s, P<uint32_t>(ctx->active[kC32]), counters + kC32,
         counters + kWorkAr32, P<int>(ctx->tc_err));
    } else if (n[kC32]) {
      ch(k_square_ar<32>, n[kC32], 256, 0, g, f, s,
         P<uint32_t>(ctx->active[kC32]), counters + kC32);
    }
    if (n[kC16] && ctx->form != PIKGPU_FORM_FP32) {
      const int grid =
          std::min((n[kC16] + 7) / 8, ctx->num_sms * ctx->tc_ctas_per_sm);
      if (ctx->form == PIKGPU_FORM_SPLIT_BF16) {
        ch(k_square_ar_tc<16, 2>, grid, tc::kThreads, ArTcSmemBytes<16, 2>(),
           g, f, s, P<uint32_t>(ctx->active[kC16]), counters + kC16,
           counters + kWorkAr, P<int>(ctx->tc_err));
      } else {
        ch(k_square_ar_tc<16, 3>, grid, tc::kThreads, ArTcSmemBytes<16, 3>(),
           g, f, s, P<uint32_t>(ctx->active[kC16]), counters + kC16,
           counters + kWorkAr, P<int>(ctx->tc_err));
      }
    } else if (n[kC16]) {
      ch(k_square_ar_rows<16>, rows_grid(n[kC16], 16), kSquareThreads, 0, g,
         f, s, P<uint32_t>(ctx->active[kC16]), counters + kC16);
    }
    CUDA_TRY(ctx, ch.err);
    br.Join(2, 1);
    final_in = f.filt;
  } else {
    Mark(ctx, kTEpf);
    Mark(ctx, kTAr);
  }
  Mark(ctx, kTFinal);
  {
    const int vec_lin = lin && lin_stride % 4 == 0 && g.W % 4 == 0 &&
                        reinterpret_cast<uintptr_t>(lin) % 16 == 0;
    const int warps = Blocks(g.W, 128) * Blocks(g.H, kFinRows);
    float* pre = ctx->keep_stages ? P<float>(ctx->dbg_pre) : nullptr;
    if (s.gaborish) {
      k_final_direct<true><<<Blocks(warps, 8), 256, 0, st>>>(
          final_in, g.PW, g.PH, g.W, g.H, s.gaborish, pre, lin, lin_stride,
          vec_lin, rgb8, rgb8_stride);
    } else {
      k_final_direct<false><<<Blocks(warps, 8), 256, 0, st>>>(
          final_in, g.PW, g.PH, g.W, g.H, 0, pre, lin, lin_stride, vec_lin,
          rgb8, rgb8_stride);
    }
    ++ctx->launches;
  }
  Mark(ctx, kNumTimed);
  CUDA_TRY(ctx, cudaGetLastError());
  return PIKGPU_OK;
}

void DropFrameGraph(pikgpu_ctx* ctx) {
  if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
  if (ctx->graph) cudaGraphDestroy(ctx->graph);
  ctx->graph_exec = nullptr;
  ctx->graph = nullptr;
}

// The launch sequence of one pikgpu_reconstruct. A call that repeats the
// previous call's launch state (GraphKey: generation, outputs, stream,
// tensor-core CTAs per SM) replays the sequence from a CUDA graph, captured
// on the first repeat; any other call launches kernel by kernel and
// remembers its state.
int RunFrame(pikgpu_ctx* ctx, float* lin, size_t lin_stride, uint8_t* rgb8,
             size_t rgb8_stride) {
  ctx->last_replayed = false;
  if (!ctx->use_graphs || ctx->profile) {
    DropFrameGraph(ctx);
    ctx->have_key = false;
    return LaunchAll(ctx, lin, lin_stride, rgb8, rgb8_stride);
  }
  const pikgpu_ctx::GraphKey key{ctx->generation, ctx->qac_in, lin,
                                 lin_stride,      rgb8,        rgb8_stride,
                                 ctx->stream,     ctx->tc_ctas_per_sm};
  const bool repeat = ctx->have_key && key == ctx->key;
  if (repeat && ctx->graph_exec) {
    CUDA_TRY(ctx, cudaGraphLaunch(ctx->graph_exec, ctx->stream));
    ctx->launches = ctx->graph_launches;
    ctx->smoothed_valid = false;
    ctx->tape_valid = ctx->graph_tape_valid;
    ctx->last_replayed = true;
    return PIKGPU_OK;
  }
  DropFrameGraph(ctx);
  if (!repeat) {
    ctx->key = key;
    ctx->have_key = true;
    return LaunchAll(ctx, lin, lin_stride, rgb8, rgb8_stride);
  }
  // First repeat: capture, instantiate and launch. If capturing is not
  // possible (the stream is being captured by the caller, say), launch
  // directly.
  if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) !=
      cudaSuccess) {
    cudaGetLastError();
    ctx->have_key = false;
    return LaunchAll(ctx, lin, lin_stride, rgb8, rgb8_stride);
  }
  const int rc = LaunchAll(ctx, lin, lin_stride, rgb8, rgb8_stride);
  cudaGraph_t graph = nullptr;
  const cudaError_t end = cudaStreamEndCapture(ctx->stream, &graph);
  cudaGraphExec_t exec = nullptr;
  const cudaError_t inst =
      rc == PIKGPU_OK && end == cudaSuccess
          ? cudaGraphInstantiate(&exec, graph, 0)
          : cudaErrorUnknown;
  if (inst != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    ctx->have_key = false;
    if (rc != PIKGPU_OK) return rc;
    return LaunchAll(ctx, lin, lin_stride, rgb8, rgb8_stride);
  }
  ctx->graph = graph;
  ctx->graph_exec = exec;
  ctx->graph_launches = ctx->launches;
  ctx->graph_tape_valid = ctx->tape_valid;
  ++ctx->graph_captures;
  CUDA_TRY(ctx, cudaGraphLaunch(ctx->graph_exec, ctx->stream));
  ctx->last_replayed = true;
  return PIKGPU_OK;
}

}  // namespace

extern "C" {

int pikgpu_validate(const pikgpu_frame_params* params, char* msg,
                    size_t msg_size) {
  pikgpu_ctx tmp;
  const int rc = Validate(&tmp, params);
  if (msg && msg_size) {
    snprintf(msg, msg_size, "%s", rc == PIKGPU_OK ? "" : tmp.err.c_str());
  }
  return rc;
}

int pikgpu_ctx_create(int device, pikgpu_ctx** out) {
  if (!out) return PIKGPU_ERR_INVALID_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    return PIKGPU_ERR_CUDA;
  }
  pikgpu_ctx* ctx = new pikgpu_ctx;
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) !=
          cudaSuccess) {
    delete ctx;
    return PIKGPU_ERR_CUDA;
  }
  ctx->stream = ctx->own_stream;
  for (auto& e : ctx->ev) cudaEventCreate(&e);
  for (auto& s : ctx->side) {
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
      pikgpu_ctx_destroy(ctx);
      return PIKGPU_ERR_CUDA;
    }
  }
  for (auto& e : ctx->fork_ev) {
    cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  }
  for (auto& row : ctx->join_ev) {
    for (auto& e : row) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  }
  cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount,
                         device);
  if (Ensure(ctx, &ctx->tc_err, sizeof(int)) != PIKGPU_OK ||
      cudaMemset(ctx->tc_err.p, 0, sizeof(int)) != cudaSuccess ||
      cudaMallocHost(&ctx->tc_err_host, sizeof(int)) != cudaSuccess) {
    pikgpu_ctx_destroy(ctx);
    return PIKGPU_ERR_NO_MEMORY;
  }
  if (UploadTables(ctx) != PIKGPU_OK) {
    pikgpu_ctx_destroy(ctx);
    return PIKGPU_ERR_CUDA;
  }
  *out = ctx;
  return PIKGPU_OK;
}

int pikgpu_ctx_destroy(pikgpu_ctx* ctx) {
  if (!ctx) return PIKGPU_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  DevBuf* bufs[] = {&ctx->acs,     &ctx->qf,        &ctx->lut,
                    &ctx->dq_cf,   &ctx->dq_map,    &ctx->ytox,
                    &ctx->ytob,    &ctx->table,     &ctx->offsets,
                    &ctx->qdc,     &ctx->qac,       &ctx->dc,
                    &ctx->dcpad,   &ctx->ac,
                    &ctx->pred2x2_g, &ctx->idct,    &ctx->smoothed,
                    &ctx->filt,    &ctx->mm,        &ctx->sigma,
                    &ctx->dc_sigma, &ctx->out_lin,  &ctx->out_rgb8,
                    &ctx->dbg_dequant, &ctx->dbg_epf, &ctx->dbg_pre,
                    &ctx->guide_ovr, &ctx->sigma_ovr, &ctx->dq_ovr,
                    &ctx->clamp_scale, &ctx->adj_a,  &ctx->adj_b,
                    &ctx->adj_c,   &ctx->adj_coef,  &ctx->adj_pred,
                    &ctx->adj_qf,  &ctx->adj_guide, &ctx->adj_partial,
                    &ctx->adj_jac, &ctx->adj_target, &ctx->adj_tape,
                    &ctx->tape_in, &ctx->pnm};
  for (DevBuf* b : bufs) FreeBuf(b);
  for (auto& b : ctx->list) FreeBuf(&b);
  for (auto& b : ctx->active) FreeBuf(&b);
  FreeBuf(&ctx->counters);
  FreeBuf(&ctx->tc_err);
  DropFrameGraph(ctx);
  if (ctx->tc_err_host) cudaFreeHost(ctx->tc_err_host);
  for (auto& e : ctx->ev) {
    if (e) cudaEventDestroy(e);
  }
  for (auto& e : ctx->fork_ev) {
    if (e) cudaEventDestroy(e);
  }
  for (auto& row : ctx->join_ev) {
    for (auto& e : row) {
      if (e) cudaEventDestroy(e);
    }
  }
  for (auto& s : ctx->side) {
    if (s) cudaStreamDestroy(s);
  }
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return PIKGPU_OK;
}

const char* pikgpu_last_error(const pikgpu_ctx* ctx) {
  return ctx ? ctx->err.c_str() : "NULL context";
}

int pikgpu_set_stream(pikgpu_ctx* ctx, void* stream) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  PIKGPU_NOT_PENDING(ctx);
  ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
  return PIKGPU_OK;
}

int pikgpu_set_option(pikgpu_ctx* ctx, int option, int value) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  PIKGPU_NOT_PENDING(ctx);
  ++ctx->generation;
  switch (option) {
    case PIKGPU_OPT_KEEP_STAGES:
      ctx->keep_stages = value != 0;
      return PIKGPU_OK;
    case PIKGPU_OPT_PROFILE:
      ctx->profile = value != 0;
      return PIKGPU_OK;
    case PIKGPU_OPT_GRAPHS:
      ctx->use_graphs = value != 0;
      return PIKGPU_OK;
    case PIKGPU_OPT_FORM:
      if (value != PIKGPU_FORM_FP32 && value != PIKGPU_FORM_SPLIT_BF16 &&
          value != PIKGPU_FORM_SPLIT_BF16X3) {
        return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "form %d", value);
      }
      ctx->form = value;
      return PIKGPU_OK;
    case PIKGPU_OPT_TC_WAIT_POLLS:
      if (value < -1) {
        return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "wait polls %d", value);
      }
      ctx->tc_polls = value < 0 ? tc::kMaxPolls : uint32_t(value);
      return PIKGPU_OK;
  }
  return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "unknown option %d", option);
}

int pikgpu_frame_begin(pikgpu_ctx* ctx, const pikgpu_frame_params* p) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  PIKGPU_NOT_PENDING(ctx);
  // The launch state before this frame: a frame that leaves it unchanged
  // (and reallocates nothing, which Ensure would record) keeps the
  // generation, so a captured graph stays valid for it.
  const bool had_frame = ctx->have_frame;
  const bool had_overrides = ctx->use_guide_ovr || ctx->use_sigma_ovr ||
                             ctx->use_dq_ovr || ctx->use_clamp_scale ||
                             ctx->use_tape_in;
  const Geo old_g = ctx->g;
  const FrameScalars old_s = ctx->s;
  float old_half[3];
  memcpy(old_half, ctx->dc_half_step, sizeof(old_half));
  size_t old_n[kNumClasses];
  for (int k = 0; k < kNumClasses; ++k) old_n[k] = ctx->lists[k].size();
  ++ctx->generation;  // until the frame is known to keep the state
  const uint64_t gen0 = ctx->generation;
  ctx->have_frame = ctx->have_ac = ctx->have_result = false;
  ctx->qac_in = nullptr;
  ctx->use_guide_ovr = ctx->use_sigma_ovr = false;
  ctx->use_dq_ovr = ctx->use_clamp_scale = false;
  ctx->use_tape_in = ctx->tape_valid = false;
  int rc = Validate(ctx, p);
  if (rc != PIKGPU_OK) return rc;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  Geo& g = ctx->g;
  g.W = p->xsize;
  g.H = p->ysize;
  g.Bx = (g.W + 7) / 8;
  g.By = (g.H + 7) / 8;
  g.PW = 8 * g.Bx;
  g.PH = 8 * g.By;
  g.Tx = (g.W + 63) / 64;
  g.Ty = (g.H + 63) / 64;
  g.Gx = (g.W + 511) / 512;
  g.Gy = (g.H + 511) / 512;
  g.ac_stride = g.Bx * 64;
  ComputeScalars(p, &ctx->s);
  for (int c = 0; c < 3; ++c) {
    // AdaptiveDCReconstruction half step (pik/adaptive_reconstruction.cc:
    // 319-322): inv_quant_dc * DequantMatrix(0, DCT8, c)[0] * 0.5f.
    ctx->dc_half_step[c] = ctx->s.inv_quant_dc *
                           p->dequant_table[p->dequant_offsets[c]] * 0.5f;
  }
  const size_t nb = size_t(g.Bx) * g.By, nt = size_t(g.Tx) * g.Ty;
  const size_t npx = size_t(g.PW) * g.PH;
  const size_t nac = size_t(g.ac_stride) * g.By;
  const int ng = g.Gx * g.Gy;
  const int dpw = (g.Bx + 7) / 8 * 8, dph = (g.By + 7) / 8 * 8;
  struct {
    DevBuf* b;
    size_t bytes;
  } allocs[] = {
      {&ctx->acs, nb},
      {&ctx->qf, 4 * nb},
      {&ctx->lut, nb},
      {&ctx->dq_cf, nt},
      {&ctx->dq_map, 16 * 256},
      {&ctx->ytox, 4 * nt},
      {&ctx->ytob, 4 * nt},
      {&ctx->table, 4 * size_t(p->dequant_table_size)},
      {&ctx->offsets, 4 * size_t(p->num_dequant_tables) * 21},
      {&ctx->qdc, 2 * 3 * nb},
      {&ctx->qac, 2 * 3 * nac},
      {&ctx->dc, 4 * 3 * nb},
      {&ctx->dcpad, 4 * 3 * size_t(dpw) * dph},
      {&ctx->ac, 4 * 3 * nac},
      {&ctx->pred2x2_g, 4 * kG2GroupFloats * ng},
      {&ctx->idct, 4 * 3 * npx},
      {&ctx->filt, 4 * 3 * npx},
      {&ctx->mm, 64},
      {&ctx->sigma, 4 * nb},
      {&ctx->dc_sigma, 4 * size_t(dpw / 8) * (dph / 8)},
  };
  for (auto& a : allocs) {
    rc = Ensure(ctx, a.b, a.bytes);
    if (rc != PIKGPU_OK) return rc;
  }
  if (ctx->keep_stages) {
    if ((rc = Ensure(ctx, &ctx->dbg_dequant, 4 * 3 * nac)) ||
        (rc = Ensure(ctx, &ctx->dbg_epf, 4 * 3 * npx)) ||
        (rc = Ensure(ctx, &ctx->dbg_pre, 4 * 3 * size_t(g.W) * g.H)) ||
        (rc = Ensure(ctx, &ctx->adj_tape, nac))) {
      return rc;
    }
  }
  // Block lists per transform class (first blocks only).
  for (auto& l : ctx->lists) l.clear();
  for (int y = 0; y < g.By; ++y) {
    for (int x = 0; x < g.Bx; ++x) {
      const uint8_t a = p->ac_strategy[y * g.Bx + x];
      if (a & 0xF) continue;
      ctx->lists[ClassOf(a >> 4)].push_back(uint32_t(x) | (uint32_t(y) << 16));
    }
  }
  // The small-transform class in type order: its inverse runs one thread
  // per block, and warps of one type do not diverge.
  std::stable_sort(ctx->lists[kCSmall].begin(), ctx->lists[kCSmall].end(),
                   [&](uint32_t u, uint32_t v) {
                     const auto type = [&](uint32_t q) {
                       return p->ac_strategy[(q >> 16) * g.Bx + (q & 0xFFFF)];
                     };
                     return type(u) < type(v);
                   });
  cudaStream_t st = ctx->stream;
  if ((rc = Ensure(ctx, &ctx->counters, sizeof(int) * kNumCounters))) {
    return rc;
  }
  for (int k = 0; k < kNumClasses; ++k) {
    rc = Ensure(ctx, &ctx->list[k], 4 * ctx->lists[k].size());
    if (rc != PIKGPU_OK) return rc;
    rc = Ensure(ctx, &ctx->active[k], 4 * ctx->lists[k].size());
    if (rc != PIKGPU_OK) return rc;
    if (!ctx->lists[k].empty()) {
      CUDA_TRY(ctx, cudaMemcpyAsync(ctx->list[k].p, ctx->lists[k].data(),
                                    4 * ctx->lists[k].size(),
                                    cudaMemcpyHostToDevice, st));
    }
  }
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->acs.p, p->ac_strategy, nb,
                                cudaMemcpyHostToDevice, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->qf.p, p->raw_quant_field, 4 * nb,
                                cudaMemcpyHostToDevice, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->lut.p, p->ar_sigma_lut_ids, nb,
                                cudaMemcpyHostToDevice, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->dq_cf.p, p->dequant_control_field, nt,
                                cudaMemcpyHostToDevice, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->dq_map.p, p->dequant_map, 16 * 256,
                                cudaMemcpyHostToDevice, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->ytox.p, p->ytox_map, 4 * nt,
                                cudaMemcpyHostToDevice, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->ytob.p, p->ytob_map, 4 * nt,
                                cudaMemcpyHostToDevice, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->table.p, p->dequant_table,
                                4 * size_t(p->dequant_table_size),
                                cudaMemcpyHostToDevice, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->offsets.p, p->dequant_offsets,
                                4 * size_t(p->num_dequant_tables) * 21,
                                cudaMemcpyHostToDevice, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->qdc.p, p->quantized_dc, 2 * 3 * nb,
                                cudaMemcpyHostToDevice, st));
  ctx->have_frame = true;
  bool same = had_frame && !had_overrides && ctx->generation == gen0 &&
              memcmp(&old_g, &ctx->g, sizeof(Geo)) == 0 &&
              memcmp(&old_s, &ctx->s, sizeof(FrameScalars)) == 0 &&
              memcmp(old_half, ctx->dc_half_step, sizeof(old_half)) == 0;
  for (int k = 0; k < kNumClasses; ++k) {
    same = same && old_n[k] == ctx->lists[k].size();
  }
  if (same) ctx->generation = gen0 - 1;
  return PIKGPU_OK;
}

}  // extern "C"

namespace {
// Where the dequantisation reads the AC from: the context's copy (NULL) or
// the caller's device planes. A change makes captured graphs stale.
void SetAcSource(pikgpu_ctx* ctx, const int16_t* in_place) {
  if (ctx->qac_in != in_place) {
    ctx->qac_in = in_place;
    ++ctx->generation;
  }
}
}  // namespace

extern "C" {

int pikgpu_frame_set_ac(pikgpu_ctx* ctx, const int16_t* const planes[3],
                        size_t stride) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  PIKGPU_NOT_PENDING(ctx);
  if (!ctx->have_frame) return Fail(ctx, PIKGPU_ERR_STATE, "no frame");
  // The copies go to the context's stream from the caller's thread, whose
  // current device may be another one.
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (!planes || stride < size_t(ctx->g.ac_stride)) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "bad AC planes/stride");
  }
  const Geo& g = ctx->g;
  for (int c = 0; c < 3; ++c) {
    if (!planes[c]) return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "NULL AC plane");
    int16_t* dst = P<int16_t>(ctx->qac) + size_t(c) * g.ac_stride * g.By;
    CUDA_TRY(ctx, cudaMemcpy2DAsync(dst, 2 * size_t(g.ac_stride), planes[c],
                                    2 * stride, 2 * size_t(g.ac_stride), g.By,
                                    cudaMemcpyHostToDevice, ctx->stream));
  }
  SetAcSource(ctx, nullptr);
  ctx->have_ac = true;
  return PIKGPU_OK;
}

int pikgpu_frame_set_group_ac(pikgpu_ctx* ctx, uint32_t group_index,
                              const int16_t* const planes[3], size_t stride) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  PIKGPU_NOT_PENDING(ctx);
  if (!ctx->have_frame) return Fail(ctx, PIKGPU_ERR_STATE, "no frame");
  // The copies go to the context's stream from the caller's thread, whose
  // current device may be another one.
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const Geo& g = ctx->g;
  if (group_index >= uint32_t(g.Gx * g.Gy)) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "group %u of %d", group_index,
                g.Gx * g.Gy);
  }
  const int x0 = (group_index % g.Gx) * 64, y0 = (group_index / g.Gx) * 64;
  const int gxs = std::min(64, g.Bx - x0), gys = std::min(64, g.By - y0);
  if (!planes || stride < size_t(gxs) * 64) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "bad AC planes/stride");
  }
  for (int c = 0; c < 3; ++c) {
    if (!planes[c]) return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "NULL AC plane");
    int16_t* dst = P<int16_t>(ctx->qac) + size_t(c) * g.ac_stride * g.By +
                   size_t(y0) * g.ac_stride + size_t(x0) * 64;
    CUDA_TRY(ctx, cudaMemcpy2DAsync(dst, 2 * size_t(g.ac_stride), planes[c],
                                    2 * stride, 2 * size_t(gxs) * 64, gys,
                                    cudaMemcpyHostToDevice, ctx->stream));
  }
  SetAcSource(ctx, nullptr);
  ctx->have_ac = true;
  return PIKGPU_OK;
}

int pikgpu_frame_set_ac_device(pikgpu_ctx* ctx, const int16_t* const planes[3],
                               size_t stride) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  PIKGPU_NOT_PENDING(ctx);
  if (!ctx->have_frame) return Fail(ctx, PIKGPU_ERR_STATE, "no frame");
  // The copies go to the context's stream from the caller's thread, whose
  // current device may be another one.
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (!planes || stride < size_t(ctx->g.ac_stride)) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "bad AC planes/stride");
  }
  const Geo& g = ctx->g;
  for (int c = 0; c < 3; ++c) {
    if (!planes[c]) return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "NULL AC plane");
  }
  // Planes in the context's own layout (stride Bx * 64, consecutive, the
  // first 16-byte aligned) are read in place; others are copied.
  const size_t plane = size_t(g.ac_stride) * g.By;
  if (stride == size_t(g.ac_stride) && planes[1] == planes[0] + plane &&
      planes[2] == planes[1] + plane &&
      (reinterpret_cast<uintptr_t>(planes[0]) & 15) == 0) {
    SetAcSource(ctx, planes[0]);
    ctx->have_ac = true;
    return PIKGPU_OK;
  }
  SetAcSource(ctx, nullptr);
  for (int c = 0; c < 3; ++c) {
    int16_t* dst = P<int16_t>(ctx->qac) + size_t(c) * plane;
    CUDA_TRY(ctx, cudaMemcpy2DAsync(dst, 2 * size_t(g.ac_stride), planes[c],
                                    2 * stride, 2 * size_t(g.ac_stride), g.By,
                                    cudaMemcpyDeviceToDevice, ctx->stream));
  }
  ctx->have_ac = true;
  return PIKGPU_OK;
}

}  // extern "C"

namespace {

// Enqueues one reconstruction and its output copies on the context's
// stream (pikgpu_reconstruct without the final synchronisation).
int EnqueueReconstruct(pikgpu_ctx* ctx, float* const out_linear[3],
                       size_t linear_stride, uint8_t* out_srgb8,
                       size_t srgb8_stride, int outputs_on_device) {
  ctx->have_result = false;
  if (!ctx->have_frame || !(ctx->have_ac || ctx->use_dq_ovr)) {
    return Fail(ctx, PIKGPU_ERR_STATE, "frame or AC not supplied");
  }
  const Geo& g = ctx->g;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (out_linear) {
    for (int c = 0; c < 3; ++c) {
      if (!out_linear[c]) {
        return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "NULL output plane");
      }
    }
    if (linear_stride < size_t(g.W)) {
      return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "linear stride too small");
    }
  }
  if (out_srgb8 && srgb8_stride < 3 * size_t(g.W)) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "sRGB-8 stride too small");
  }
  float* lin = nullptr;
  size_t lin_stride = size_t(g.W);
  uint8_t* rgb8 = nullptr;
  size_t rgb8_stride = 3 * size_t(g.W);
  int rc;
  // The kernel writes three planes at lin + c * lin_stride * H; device
  // outputs must be laid out that way (checked below), host outputs go
  // through a dense device buffer.
  if (out_linear) {
    if (outputs_on_device) {
      const size_t plane = linear_stride * g.H;
      if (out_linear[1] != out_linear[0] + plane ||
          out_linear[2] != out_linear[0] + 2 * plane) {
        return Fail(ctx, PIKGPU_ERR_INVALID_ARG,
                    "device output planes must be consecutive (plane = "
                    "stride * ysize)");
      }
      lin = out_linear[0];
      lin_stride = linear_stride;
    } else {
      if ((rc = Ensure(ctx, &ctx->out_lin, 4 * 3 * size_t(g.W) * g.H))) {
        return rc;
      }
      lin = P<float>(ctx->out_lin);
    }
  }
  if (out_srgb8) {
    if (outputs_on_device) {
      rgb8 = out_srgb8;
      rgb8_stride = srgb8_stride;
    } else {
      if ((rc = Ensure(ctx, &ctx->out_rgb8, 3 * size_t(g.W) * g.H))) return rc;
      rgb8 = P<uint8_t>(ctx->out_rgb8);
    }
  }
  rc = RunFrame(ctx, lin, lin_stride, rgb8, rgb8_stride);
  if (rc != PIKGPU_OK) return rc;
  ctx->last_lin = lin;
  ctx->last_lin_stride = lin_stride;
  if (!outputs_on_device) {
    if (out_linear) {
      for (int c = 0; c < 3; ++c) {
        CUDA_TRY(ctx, cudaMemcpy2DAsync(
                          out_linear[c], 4 * linear_stride,
                          lin + size_t(c) * g.W * g.H, 4 * size_t(g.W),
                          4 * size_t(g.W), g.H, cudaMemcpyDeviceToHost,
                          ctx->stream));
      }
    }
    if (out_srgb8) {
      CUDA_TRY(ctx, cudaMemcpy2DAsync(out_srgb8, srgb8_stride, rgb8,
                                      3 * size_t(g.W), 3 * size_t(g.W), g.H,
                                      cudaMemcpyDeviceToHost, ctx->stream));
    }
  }
  // The wait-timeout flag comes back with the same synchronisation.
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->tc_err_host, ctx->tc_err.p, sizeof(int),
                                cudaMemcpyDeviceToHost, ctx->stream));
  ctx->pending = true;
  return PIKGPU_OK;
}

// Waits for the enqueued reconstruction and checks it.
int FinishReconstruct(pikgpu_ctx* ctx) {
  ctx->pending = false;
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (const int code = *ctx->tc_err_host) {
    *ctx->tc_err_host = 0;
    cudaMemset(ctx->tc_err.p, 0, sizeof(int));
    return Fail(ctx, PIKGPU_ERR_CUDA, "%s", WaitTimeoutMessage(code));
  }
  if (ctx->profile) {
    for (int i = 0; i < kNumTimed; ++i) {
      cudaEventElapsedTime(&ctx->times[i], ctx->ev[i], ctx->ev[i + 1]);
    }
  }
  ctx->have_result = true;
  return PIKGPU_OK;
}

}  // namespace

extern "C" {

int pikgpu_reconstruct(pikgpu_ctx* ctx, float* const out_linear[3],
                       size_t linear_stride, uint8_t* out_srgb8,
                       size_t srgb8_stride, int outputs_on_device) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  PIKGPU_NOT_PENDING(ctx);
  const int rc = EnqueueReconstruct(ctx, out_linear, linear_stride,
                                    out_srgb8, srgb8_stride,
                                    outputs_on_device);
  if (rc != PIKGPU_OK) return rc;
  return FinishReconstruct(ctx);
}

int pikgpu_reconstruct_async(pikgpu_ctx* ctx, float* const out_linear[3],
                             size_t linear_stride, uint8_t* out_srgb8,
                             size_t srgb8_stride, int outputs_on_device) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  PIKGPU_NOT_PENDING(ctx);
  return EnqueueReconstruct(ctx, out_linear, linear_stride, out_srgb8,
                            srgb8_stride, outputs_on_device);
}

int pikgpu_wait(pikgpu_ctx* ctx) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  if (!ctx->pending) return PIKGPU_OK;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  return FinishReconstruct(ctx);
}

int pikgpu_get_stage(pikgpu_ctx* ctx, int stage, float* const planes[3],
                     size_t stride, size_t xsize, size_t ysize) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  PIKGPU_NOT_PENDING(ctx);
  if (!ctx->have_result) return Fail(ctx, PIKGPU_ERR_STATE, "no result");
  const Geo& g = ctx->g;
  const float* src = nullptr;
  size_t w = 0, h = 0;
  switch (stage) {
    case PIKGPU_STAGE_DC:
      src = P<float>(ctx->dc), w = g.Bx, h = g.By;
      break;
    case PIKGPU_STAGE_IDCT:
      src = P<float>(ctx->idct), w = g.PW, h = g.PH;
      break;
    case PIKGPU_STAGE_SMOOTHED: {
      // Without gaborish the EPF guide source is the IDCT output itself
      // (DoAdaptiveReconstruction, pik/compressed_image.cc:1126-1132).
      const int rc = EnsureSmoothed(ctx);
      if (rc != PIKGPU_OK) return rc;
      src = P<float>(ctx->s.gaborish ? ctx->smoothed : ctx->idct);
      w = g.PW, h = g.PH;
      break;
    }
    case PIKGPU_STAGE_EPF:
      src = P<float>(ctx->dbg_epf), w = g.PW, h = g.PH;
      break;
    case PIKGPU_STAGE_AR:
      src = P<float>(ctx->filt), w = g.PW, h = g.PH;
      break;
    case PIKGPU_STAGE_PRE_OPSIN:
      src = P<float>(ctx->dbg_pre), w = g.W, h = g.H;
      break;
    case PIKGPU_STAGE_DEQUANT_AC:
      src = P<float>(ctx->dbg_dequant), w = g.ac_stride, h = g.By;
      break;
    default:
      return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "stage %d", stage);
  }
  const bool debug_stage = stage == PIKGPU_STAGE_EPF ||
                           stage == PIKGPU_STAGE_PRE_OPSIN ||
                           stage == PIKGPU_STAGE_DEQUANT_AC;
  if (debug_stage && !ctx->keep_stages) {
    return Fail(ctx, PIKGPU_ERR_STATE,
                "stage %d needs PIKGPU_OPT_KEEP_STAGES before frame_begin",
                stage);
  }
  if (!planes || xsize != w || ysize != h || stride < w) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG,
                "stage %d is %zux%zu (got %zux%zu, stride %zu)", stage, w, h,
                xsize, ysize, stride);
  }
  for (int c = 0; c < 3; ++c) {
    CUDA_TRY(ctx, cudaMemcpy2D(planes[c], 4 * stride, src + c * w * h, 4 * w,
                               4 * w, h, cudaMemcpyDeviceToHost));
  }
  return PIKGPU_OK;
}

int pikgpu_set_epf_decisions(pikgpu_ctx* ctx, const uint8_t* guide,
                             const int32_t* sigma) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  PIKGPU_NOT_PENDING(ctx);
  if (!ctx->have_frame) return Fail(ctx, PIKGPU_ERR_STATE, "no frame");
  ++ctx->generation;
  const Geo& g = ctx->g;
  int rc;
  ctx->use_guide_ovr = guide != nullptr;
  ctx->use_sigma_ovr = sigma != nullptr;
  if (guide) {
    const size_t n = 3 * size_t(g.PW + 12) * (g.PH + 12);
    if ((rc = Ensure(ctx, &ctx->guide_ovr, n))) return rc;
    CUDA_TRY(ctx, cudaMemcpy(ctx->guide_ovr.p, guide, n,
                             cudaMemcpyHostToDevice));
  }
  if (sigma) {
    // The EPF indexes its weight table by sigma (pik/epf.h:70-76).
    for (size_t i = 0; i < size_t(g.Bx) * g.By; ++i) {
      if (sigma[i] > kMaxSigma) {
        ctx->use_guide_ovr = ctx->use_sigma_ovr = false;
        return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "sigma %d > %d at block %zu",
                    sigma[i], kMaxSigma, i);
      }
    }
    const size_t n = 4 * size_t(g.Bx) * g.By;
    if ((rc = Ensure(ctx, &ctx->sigma_ovr, n))) return rc;
    CUDA_TRY(ctx, cudaMemcpy(ctx->sigma_ovr.p, sigma, n,
                             cudaMemcpyHostToDevice));
  }
  return PIKGPU_OK;
}

int pikgpu_get_epf_decisions(pikgpu_ctx* ctx, uint8_t* guide,
                             int32_t* sigma) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  PIKGPU_NOT_PENDING(ctx);
  if (!ctx->have_result || !ctx->s.have_ar) {
    return Fail(ctx, PIKGPU_ERR_STATE, "no EPF result");
  }
  const Geo& g = ctx->g;
  if (sigma) {
    CUDA_TRY(ctx, cudaMemcpy(sigma, ctx->sigma.p, 4 * size_t(g.Bx) * g.By,
                             cudaMemcpyDeviceToHost));
  }
  if (guide) {
    const size_t n = 3 * size_t(g.PW + 12) * (g.PH + 12);
    const bool smoothed = ctx->s.gaborish && !ctx->s.use_sharpened;
    int rc;
    if (smoothed && (rc = EnsureSmoothed(ctx)) != PIKGPU_OK) return rc;
    DevBuf tmp;
    if ((rc = Ensure(ctx, &tmp, n))) return rc;
    const float* src =
        smoothed ? P<float>(ctx->smoothed) : P<float>(ctx->idct);
    dim3 b(32, 8), gr(Blocks(g.PW + 12, 32), Blocks(g.PH + 12, 8), 3);
    k_export_guide<<<gr, b, 0, ctx->stream>>>(src, g.PW, g.PH,
                                              P<uint32_t>(ctx->mm),
                                              P<uint8_t>(tmp));
    cudaStreamSynchronize(ctx->stream);
    const cudaError_t e =
        cudaMemcpy(guide, tmp.p, n, cudaMemcpyDeviceToHost);
    FreeBuf(&tmp);
    if (e != cudaSuccess) {
      return Fail(ctx, PIKGPU_ERR_CUDA, "guide copy: %s",
                  cudaGetErrorString(e));
    }
  }
  return PIKGPU_OK;
}

int pikgpu_last_kernel_times(pikgpu_ctx* ctx, float* ms, int n) {
  if (!ctx || !ms) return PIKGPU_ERR_INVALID_ARG;
  if (!ctx->profile) return Fail(ctx, PIKGPU_ERR_STATE, "profiling is off");
  for (int i = 0; i < n && i < kNumTimed; ++i) ms[i] = ctx->times[i];
  return kNumTimed;
}

int pikgpu_encode_pnm(pikgpu_ctx* ctx, int bits_per_sample, int transfer,
                      uint8_t* out, size_t capacity, size_t* size,
                      int out_on_device) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  PIKGPU_NOT_PENDING(ctx);
  if (!ctx->have_result || !ctx->last_lin) {
    return Fail(ctx, PIKGPU_ERR_STATE,
                "no reconstruction with linear planes to encode");
  }
  if (bits_per_sample != 8 && bits_per_sample != 16 &&
      bits_per_sample != 32) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "bits per sample %d",
                bits_per_sample);
  }
  if (transfer != PIKGPU_TF_LINEAR && transfer != PIKGPU_TF_SRGB) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "transfer %d", transfer);
  }
  if (!size) return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "size is NULL");
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const Geo& g = ctx->g;
  // EncodeHeader (pik/codec_pnm.cc:179-196): PFM with the scale's sign
  // giving the byte order (little-endian: -1), PPM with the maximum value.
  char hdr[96];
  int hlen;
  if (bits_per_sample == 32) {
    hlen = snprintf(hdr, sizeof(hdr), "PF %zu %zu\n%f\n", size_t(g.W),
                    size_t(g.H), -1.0);
  } else {
    hlen = snprintf(hdr, sizeof(hdr), "P6\n%zu %zu\n%u\n", size_t(g.W),
                    size_t(g.H), (1u << bits_per_sample) - 1);
  }
  const size_t body = size_t(g.W) * g.H * 3 * (bits_per_sample / 8);
  *size = size_t(hlen) + body;
  if (!out) return PIKGPU_OK;
  if (capacity < *size) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG,
                "output of %zu bytes is smaller than the file (%zu)",
                capacity, *size);
  }
  uint8_t* dst = out + hlen;
  if (!out_on_device) {
    int rc = Ensure(ctx, &ctx->pnm, body);
    if (rc != PIKGPU_OK) return rc;
    dst = P<uint8_t>(ctx->pnm);
  }
  k_encode_pnm<<<dim3(Blocks(g.W, 128), g.H), 128, 0, ctx->stream>>>(
      ctx->last_lin, ctx->last_lin_stride, g.W, g.H, bits_per_sample,
      transfer == PIKGPU_TF_SRGB, dst);
  CUDA_TRY(ctx, cudaGetLastError());
  if (out_on_device) {
    CUDA_TRY(ctx, cudaMemcpyAsync(out, hdr, hlen, cudaMemcpyHostToDevice,
                                  ctx->stream));
  } else {
    memcpy(out, hdr, hlen);
    CUDA_TRY(ctx, cudaMemcpyAsync(out + hlen, dst, body,
                                  cudaMemcpyDeviceToHost, ctx->stream));
  }
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PIKGPU_OK;
}

int pikgpu_last_launch_count(const pikgpu_ctx* ctx) {
  return ctx ? ctx->launches : PIKGPU_ERR_INVALID_ARG;
}

int pikgpu_graph_stats(const pikgpu_ctx* ctx, int* captures,
                       int* last_replayed) {
  if (!ctx) return PIKGPU_ERR_INVALID_ARG;
  if (captures) *captures = ctx->graph_captures;
  if (last_replayed) *last_replayed = ctx->last_replayed ? 1 : 0;
  return PIKGPU_OK;
}

const char* pikgpu_kernel_name(int index) {
  return index >= 0 && index < kNumTimed ? kTimedNames[index] : "";
}

}  // extern "C"

#include "dc_noalloc.cu"
#include "batch.cu"
#include "adjoint.cu"
