// Batched reconstruction of many frames of uneven sizes
// (pikgpu_batch_* in include/pikgpu.h). The reference decodes one frame per
// call; here the launch sequences of all frames of a batch are captured
// once into one CUDA graph, one branch per frame (forked from and joined to
// the batch stream through events), and the graph is replayed. Frames that
// are too small to fill the GPU then run side by side, and the CPU cost of
// the frames' 17 or so launches each is paid once at capture instead of on every
// call. The graph depends on each frame's geometry, block lists, options and
// output pointers; any change re-captures it on the next call.
// Included by pikgpu.cu (uses the context internals and LaunchAll).

struct pikgpu_batch {
  int device = 0;
  std::vector<pikgpu_ctx*> frames;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> joins;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // State the captured graph was built for.
  std::vector<uint64_t> gens;
  std::vector<float*> outs;
  std::vector<size_t> strides;
  int captures = 0;
  // Launch shape: frames run in `chains` concurrent branches (frame i in
  // branch i % chains, in order within a branch), and the persistent
  // tensor-core kernels use `tc_ctas` CTAs per SM.
  int chains = 0;  // 0: one branch per frame
  int tc_ctas = kTcCtasPerSm;
  bool exec_valid_for_shape = false;  // the graph was captured with these
  // The frames' wait-timeout flags, gathered (and cleared) by one kernel
  // after each replay and read back with one copy.
  int** flag_ptrs = nullptr;  // device: each frame's flag
  int* flags = nullptr;       // device: the gathered values
  int* flags_host = nullptr;  // pinned
  std::string err;
};

// Copies and clears the frames' wait-timeout flags.
__global__ void k_gather_flags(int* const* src, int n, int* dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = atomicExch(src[i], 0);
}

namespace {

int BatchFail(pikgpu_batch* b, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  b->err = buf;
  return code;
}

#define CUDA_TRY_B(b, call)                                                \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) {                                                \
      return BatchFail(b, PIKGPU_ERR_CUDA, "%s: %s", #call,                 \
                       cudaGetErrorString(e_));                             \
    }                                                                       \
  } while (0)

void DropGraph(pikgpu_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

// Records every frame's launch sequence into a new graph.
int Capture(pikgpu_batch* b, float* const* out, const size_t* strides) {
  DropGraph(b);
  cudaError_t e = cudaStreamBeginCapture(b->stream,
                                         cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    return BatchFail(b, PIKGPU_ERR_CUDA, "begin capture: %s",
                     cudaGetErrorString(e));
  }
  int rc = PIKGPU_OK;
  e = cudaEventRecord(b->fork, b->stream);
  const size_t n = b->frames.size();
  const size_t k = b->chains > 0 ? std::min<size_t>(b->chains, n) : n;
  // Branch j runs on the stream of frame j, frames j, j + k, ... in order.
  for (size_t j = 0; j < k && e == cudaSuccess; ++j) {
    e = cudaStreamWaitEvent(b->frames[j]->own_stream, b->fork, 0);
  }
  for (size_t i = 0; i < n && e == cudaSuccess && rc == PIKGPU_OK; ++i) {
    pikgpu_ctx* ctx = b->frames[i];
    cudaStream_t user = ctx->stream;
    ctx->stream = b->frames[i % k]->own_stream;
    ctx->tc_ctas_per_sm = b->tc_ctas;
    rc = LaunchAll(ctx, out[i], strides[i], nullptr, 0,
                   /*single_stream=*/true);
    if (rc != PIKGPU_OK) BatchFail(b, rc, "frame %zu: %s", i, ctx->err.c_str());
    ctx->stream = user;
  }
  for (size_t j = 0; j < k && e == cudaSuccess; ++j) {
    e = cudaEventRecord(b->joins[j], b->frames[j]->own_stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->joins[j], 0);
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t end = cudaStreamEndCapture(b->stream, &graph);
  if (rc != PIKGPU_OK || e != cudaSuccess || end != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    if (rc != PIKGPU_OK) return rc;
    return BatchFail(b, PIKGPU_ERR_CUDA, "capture: %s",
                     cudaGetErrorString(e != cudaSuccess ? e : end));
  }
  b->graph = graph;
  e = cudaGraphInstantiate(&b->exec, graph, 0);
  if (e != cudaSuccess) {
    DropGraph(b);
    return BatchFail(b, PIKGPU_ERR_CUDA, "instantiate: %s",
                     cudaGetErrorString(e));
  }
  b->gens.resize(n);
  b->outs.assign(out, out + n);
  b->strides.assign(strides, strides + n);
  for (size_t i = 0; i < n; ++i) b->gens[i] = b->frames[i]->generation;
  b->exec_valid_for_shape = true;
  ++b->captures;
  return PIKGPU_OK;
}

}  // namespace

extern "C" {

int pikgpu_batch_create(int device, int num_frames, pikgpu_batch** out) {
  if (!out || num_frames < 1 || num_frames > 4096) {
    return PIKGPU_ERR_INVALID_ARG;
  }
  *out = nullptr;
  pikgpu_batch* b = new pikgpu_batch;
  b->device = device;
  for (int i = 0; i < num_frames; ++i) {
    pikgpu_ctx* ctx = nullptr;
    const int rc = pikgpu_ctx_create(device, &ctx);
    if (rc != PIKGPU_OK) {
      pikgpu_batch_destroy(b);
      return rc;
    }
    b->frames.push_back(ctx);
  }
  b->joins.assign(num_frames, nullptr);
  bool ok = cudaSetDevice(device) == cudaSuccess &&
            cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) ==
                cudaSuccess &&
            cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) ==
                cudaSuccess;
  for (auto& e : b->joins) {
    ok = ok && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) ==
                   cudaSuccess;
  }
  if (ok) {
    std::vector<int*> ptrs;
    for (auto* ctx : b->frames) ptrs.push_back(P<int>(ctx->tc_err));
    ok = cudaMalloc(&b->flag_ptrs, sizeof(int*) * num_frames) ==
             cudaSuccess &&
         cudaMalloc(&b->flags, sizeof(int) * num_frames) == cudaSuccess &&
         cudaMallocHost(&b->flags_host, sizeof(int) * num_frames) ==
             cudaSuccess &&
         cudaMemcpy(b->flag_ptrs, ptrs.data(), sizeof(int*) * num_frames,
                    cudaMemcpyHostToDevice) == cudaSuccess;
  }
  if (!ok) {
    pikgpu_batch_destroy(b);
    return PIKGPU_ERR_CUDA;
  }
  *out = b;
  return PIKGPU_OK;
}

int pikgpu_batch_destroy(pikgpu_batch* b) {
  if (!b) return PIKGPU_ERR_INVALID_ARG;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  DropGraph(b);
  for (auto e : b->joins) {
    if (e) cudaEventDestroy(e);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->flag_ptrs) cudaFree(b->flag_ptrs);
  if (b->flags) cudaFree(b->flags);
  if (b->flags_host) cudaFreeHost(b->flags_host);
  if (b->stream) cudaStreamDestroy(b->stream);
  for (auto* ctx : b->frames) pikgpu_ctx_destroy(ctx);
  delete b;
  return PIKGPU_OK;
}

pikgpu_ctx* pikgpu_batch_frame(pikgpu_batch* b, int index) {
  if (!b || index < 0 || index >= int(b->frames.size())) return nullptr;
  return b->frames[index];
}

const char* pikgpu_batch_last_error(const pikgpu_batch* b) {
  return b ? b->err.c_str() : "NULL batch";
}

int pikgpu_batch_reconstruct(pikgpu_batch* b, float* const* out_linear,
                             const size_t* linear_strides, void* stream) {
  if (!b) return PIKGPU_ERR_INVALID_ARG;
  if (!out_linear || !linear_strides) {
    return BatchFail(b, PIKGPU_ERR_INVALID_ARG, "NULL outputs");
  }
  const size_t n = b->frames.size();
  for (size_t i = 0; i < n; ++i) {
    const pikgpu_ctx* ctx = b->frames[i];
    if (!ctx->have_frame || !(ctx->have_ac || ctx->use_dq_ovr)) {
      return BatchFail(b, PIKGPU_ERR_STATE, "frame %zu: frame or AC not "
                       "supplied", i);
    }
    if (ctx->profile) {
      return BatchFail(b, PIKGPU_ERR_UNSUPPORTED,
                       "frame %zu: profiling is not available in a batch", i);
    }
    if (!out_linear[i] || linear_strides[i] < size_t(ctx->g.W)) {
      return BatchFail(b, PIKGPU_ERR_INVALID_ARG,
                       "frame %zu: NULL output or stride below xsize", i);
    }
  }
  CUDA_TRY_B(b, cudaSetDevice(b->device));
  bool stale = !b->exec || !b->exec_valid_for_shape;
  for (size_t i = 0; i < n && !stale; ++i) {
    stale = b->gens[i] != b->frames[i]->generation ||
            b->outs[i] != out_linear[i] ||
            b->strides[i] != linear_strides[i];
  }
  // The frames' uploads (set_ac on their streams) finish before the replay.
  for (auto* ctx : b->frames) {
    CUDA_TRY_B(b, cudaStreamSynchronize(ctx->stream));
  }
  if (stale) {
    const int rc = Capture(b, out_linear, linear_strides);
    if (rc != PIKGPU_OK) return rc;
  }
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->stream;
  CUDA_TRY_B(b, cudaGraphLaunch(b->exec, st));
  k_gather_flags<<<Blocks(n, 256), 256, 0, st>>>(b->flag_ptrs, int(n),
                                                  b->flags);
  CUDA_TRY_B(b, cudaMemcpyAsync(b->flags_host, b->flags, sizeof(int) * n,
                                cudaMemcpyDeviceToHost, st));
  CUDA_TRY_B(b, cudaStreamSynchronize(st));
  for (size_t i = 0; i < n; ++i) {
    if (const int code = b->flags_host[i]) {
      return BatchFail(b, PIKGPU_ERR_CUDA, "frame %zu: %s", i,
                       WaitTimeoutMessage(code));
    }
    b->frames[i]->have_result = true;
  }
  return PIKGPU_OK;
}

int pikgpu_batch_launch_count(const pikgpu_batch* b) {
  if (!b) return PIKGPU_ERR_INVALID_ARG;
  int n = 1;  // k_gather_flags
  for (const auto* ctx : b->frames) n += ctx->launches;
  return n;
}

int pikgpu_batch_capture_count(const pikgpu_batch* b) {
  return b ? b->captures : PIKGPU_ERR_INVALID_ARG;
}

int pikgpu_batch_autotune(pikgpu_batch* b, float* const* out_linear,
                          const size_t* linear_strides, void* stream,
                          int* chains, int* tc_ctas_per_sm) {
  if (!b) return PIKGPU_ERR_INVALID_ARG;
  const int n = int(b->frames.size());
  bool tensor = false;
  for (auto* ctx : b->frames) tensor |= ctx->form != PIKGPU_FORM_FP32;
  std::vector<int> chain_opts;
  for (int k : {1, 2, 4, 8, 16, 32, n}) {
    if (k <= n && (chain_opts.empty() || chain_opts.back() < k)) {
      chain_opts.push_back(k);
    }
  }
  std::vector<int> tc_opts = tensor ? std::vector<int>{1, 2, 4}
                                    : std::vector<int>{kTcCtasPerSm};
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->stream;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CUDA_TRY_B(b, cudaEventCreate(&e0));
  CUDA_TRY_B(b, cudaEventCreate(&e1));
  float best = 1e30f;
  int best_k = n, best_tc = kTcCtasPerSm, rc = PIKGPU_OK;
  for (int tc : tc_opts) {
    for (int k : chain_opts) {
      b->chains = k;
      b->tc_ctas = tc;
      b->exec_valid_for_shape = false;
      // Capture and one warm-up replay, then the median of 3 timed ones.
      rc = pikgpu_batch_reconstruct(b, out_linear, linear_strides, stream);
      if (rc != PIKGPU_OK) break;
      float t[3];
      for (float& ti : t) {
        cudaEventRecord(e0, st);
        cudaGraphLaunch(b->exec, st);
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
          rc = BatchFail(b, PIKGPU_ERR_CUDA, "autotune replay failed");
          break;
        }
        cudaEventElapsedTime(&ti, e0, e1);
      }
      if (rc != PIKGPU_OK) break;
      std::sort(t, t + 3);
      if (t[1] < best) {
        best = t[1];
        best_k = k;
        best_tc = tc;
      }
    }
    if (rc != PIKGPU_OK) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->chains = best_k;
  b->tc_ctas = best_tc;
  b->exec_valid_for_shape = false;
  if (rc != PIKGPU_OK) return rc;
  if (chains) *chains = best_k;
  if (tc_ctas_per_sm) *tc_ctas_per_sm = best_tc;
  return PIKGPU_OK;
}

}  // extern "C"
