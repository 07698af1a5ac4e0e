// Allocation-free DC reconstruction (pikgpu_dc_reconstruct_noalloc in
// include/pikgpu.h). It runs the kernels, with the arithmetic, of the DC
// stage of pikgpu_reconstruct in the plain FP32 form: DequantDC +
// AdaptiveDCReconstruction (pik/compressed_dc.cc:181-231,
// pik/adaptive_reconstruction.cc:300-332), with the same EPF tile shape
// choice. Its result is bit-identical to that form's DC stage. The
// tensor-core forms' DC EPF computes its weighted sums with fused
// multiply-adds, so their DC stage differs from this result by FP32
// rounding (within 2e-6). The context path keeps the intermediates in
// cudaMalloc'd buffers. Here they live in one fixed-size file-scope device
// array, and the caller passes its own input and output buffers.
//
// Who needs it: a caller that must not allocate device memory at the point
// where it reconstructs DC. Examples are a decoder driven from a real-time or
// callback thread, where cudaMalloc/cudaFree would stall on their implicit
// device synchronisation, and a process whose device memory is owned by
// another allocator (a caching allocator or a fixed arena) that this library
// must not go around. This entry point takes device pointers only. It calls
// no cudaMalloc, cudaFree or other allocating routine.
//
// Limits:
//  * The DC image (xsize_blocks x ysize_blocks, one value per 8x8 block) is
//    at most kNoAllocMaxBlocks x kNoAllocMaxBlocks, so images up to
//    4096 x 4096 pixels. Larger sizes are rejected with PIKGPU_ERR_INVALID_ARG
//    before any work is queued.
//  * The scratch holds the padded DC image (3 x 512 x 512 floats), 4096
//    per-block sigmas and the guide min/max words, about 3.02 MiB of static
//    device memory per device.
//  * No part of the scratch has to start at zero. Every call first resets
//    the min/max words with a kernel, then fully writes the padded image
//    and the sigmas before it reads them.
//  * The first call on a device does the set-up, with that device current:
//    it uploads the constant tables, sets the EPF kernel's shared-memory
//    limit, reads the SM count and looks up the scratch address. Make
//    that first call before any stream capture on the device.
//  * All calls on one device share the scratch. Calls that overlap in time
//    on the same device (other streams, or host threads without ordering)
//    race on it and give wrong results. Issue them on one stream, or
//    serialise them.
// Included by pikgpu.cu: the kernels, tables and helpers come from there.

namespace {

constexpr int kNoAllocMaxBlocks = 512;
constexpr size_t kNoAllocPlane = size_t(kNoAllocMaxBlocks) * kNoAllocMaxBlocks;
constexpr size_t kNoAllocSigmas = kNoAllocPlane / 64;  // 8x8-block EPF cells
constexpr size_t kNoAllocPadOff = 0;                  // 3 padded DC planes
constexpr size_t kNoAllocSigOff = 3 * kNoAllocPlane;  // int32 sigma / cell
constexpr size_t kNoAllocMmOff = kNoAllocSigOff + kNoAllocSigmas;  // 16 words
constexpr size_t kNoAllocWords = kNoAllocMmOff + 64;

struct NoAllocDevice {
  bool ready = false;
  uint32_t* scratch = nullptr;
  int num_sms = 148;
};
std::mutex g_noalloc_mutex;
NoAllocDevice g_noalloc[64];

}  // namespace

// 32-bit words; each region above starts on a 256-byte boundary.
static __device__ __align__(256) uint32_t g_dc_scratch[kNoAllocWords];

namespace {

// True for managed memory and for device memory of device `dev` (the
// kernels run there; another GPU's buffer is refused rather than read
// through the peer mapping or faulted on).
bool IsDevicePointer(const void* p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // leave no error behind for the caller's next call
    return false;
  }
  return a.type == cudaMemoryTypeManaged ||
         (a.type == cudaMemoryTypeDevice && a.device == dev);
}

bool Overlaps(const void* a, size_t na, const void* b, size_t nb) {
  const uintptr_t x = reinterpret_cast<uintptr_t>(a);
  const uintptr_t y = reinterpret_cast<uintptr_t>(b);
  return x < y + nb && y < x + na;
}

int DcNoAlloc(pikgpu_ctx* ctx, const int16_t* quantized_dc, uint32_t bx,
              uint32_t by, int32_t global_scale, int32_t quant_dc,
              const float dc_dequant[3], int32_t ytox_dc, int32_t ytob_dc,
              float* dc, cudaStream_t st) {
  if (!quantized_dc || !dc || !dc_dequant) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "NULL pointer argument");
  }
  if (bx == 0 || by == 0) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "empty DC image %ux%u", bx, by);
  }
  if (bx > uint32_t(kNoAllocMaxBlocks) || by > uint32_t(kNoAllocMaxBlocks)) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG,
                "DC image of %ux%u blocks exceeds the %dx%d-block limit of "
                "the allocation-free entry point (use pikgpu_reconstruct)",
                bx, by, kNoAllocMaxBlocks, kNoAllocMaxBlocks);
  }
  if (global_scale < 1 || global_scale > 32768) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "global_scale %d", global_scale);
  }
  if (quant_dc < 1 || quant_dc > 256) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "quant_dc %d", quant_dc);
  }
  const size_t n = size_t(bx) * by;
  int dev = 0;
  CUDA_TRY(ctx, cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    return Fail(ctx, PIKGPU_ERR_UNSUPPORTED, "device %d", dev);
  }
  if (!IsDevicePointer(quantized_dc, dev) || !IsDevicePointer(dc, dev)) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG,
                "quantized_dc and dc must be device pointers on the current "
                "device (%d)",
                dev);
  }
  if (Overlaps(quantized_dc, 3 * n * sizeof(int16_t), dc,
               3 * n * sizeof(float))) {
    return Fail(ctx, PIKGPU_ERR_INVALID_ARG, "quantized_dc and dc overlap");
  }
  ctx->device = dev;
  uint32_t* scratch = nullptr;
  int num_sms = 148;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoAllocDevice& d = g_noalloc[dev];
    if (!d.ready) {
      const int rc = UploadTables(ctx);
      if (rc != PIKGPU_OK) return rc;
      void* p = nullptr;
      CUDA_TRY(ctx, cudaGetSymbolAddress(&p, g_dc_scratch));
      CUDA_TRY(ctx, cudaDeviceGetAttribute(
                        &d.num_sms, cudaDevAttrMultiProcessorCount, dev));
      d.scratch = static_cast<uint32_t*>(p);
      d.ready = true;
    }
    scratch = d.scratch;
    num_sms = d.num_sms;
  }

  // Same scalars, in the same operation order, as pikgpu_frame_begin.
  pikgpu_frame_params p{};
  const uint32_t offsets[3] = {0, 1, 2};
  p.global_scale = global_scale;
  p.quant_dc = quant_dc;
  p.dequant_table = dc_dequant;
  p.dequant_offsets = offsets;
  p.ytox_dc = ytox_dc;
  p.ytob_dc = ytob_dc;
  FrameScalars s{};
  ComputeScalars(&p, &s);
  float half_step[3];
  for (int c = 0; c < 3; ++c) {
    half_step[c] = s.inv_quant_dc * dc_dequant[c] * 0.5f;
  }
  Geo g{};
  g.Bx = int(bx);
  g.By = int(by);
  DevFrame f{};
  f.qdc = quantized_dc;
  f.dc = dc;

  float* dcpad = reinterpret_cast<float*>(scratch + kNoAllocPadOff);
  int32_t* sig = reinterpret_cast<int32_t*>(scratch + kNoAllocSigOff);
  uint32_t* mm = scratch + kNoAllocMmOff;
  const int dpw = (g.Bx + 7) / 8 * 8, dph = (g.By + 7) / 8 * 8;

  // The FP32 form's DC stage of LaunchAll: min/max reset, dequantisation
  // with the padded copy and its min/max, then the EPF clamping into `dc`.
  k_frame_init<<<1, 32, 0, st>>>(mm, nullptr, 0);
  k_dc_prep<<<dim3(Blocks(dpw, 32), Blocks(dph, 8)), 256, 0, st>>>(
      g, f, s, dcpad, dpw, dph, mm + 8);
  EpfSigma sgs{};
  sgs.const_qf = s.quant_dc / 2;
  sgs.fixed = -1;
  sgs.out = sig;
  const EpfDc dco{dc, g.Bx, g.By, half_step[0], half_step[1], half_step[2]};
  EpfLaunch(st, num_sms, PIKGPU_FORM_FP32, dcpad, dcpad, 0, dpw, dph, mm + 8,
            sgs, nullptr, nullptr, dco, /*err=*/nullptr);
  CUDA_TRY(ctx, cudaGetLastError());
  return PIKGPU_OK;
}

}  // namespace

extern "C" int pikgpu_dc_reconstruct_noalloc(
    const int16_t* quantized_dc, uint32_t xsize_blocks, uint32_t ysize_blocks,
    int32_t global_scale, int32_t quant_dc, const float dc_dequant[3],
    int32_t ytox_dc, int32_t ytob_dc, float* dc, void* stream, char* msg,
    size_t msg_size) {
  pikgpu_ctx tmp;  // host-side error text only; owns no device resources
  const int rc = DcNoAlloc(&tmp, quantized_dc, xsize_blocks, ysize_blocks,
                           global_scale, quant_dc, dc_dequant, ytox_dc,
                           ytob_dc, dc, static_cast<cudaStream_t>(stream));
  if (msg && msg_size) {
    snprintf(msg, msg_size, "%s", rc == PIKGPU_OK ? "" : tmp.err.c_str());
  }
  return rc;
}
