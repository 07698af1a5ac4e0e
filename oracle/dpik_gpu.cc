// dpik_gpu: the reference decoder (PikToPixels, pik/pik.cc:92-131, built
// from its unmodified sources into oracle/_ref/libpikref_scalar.so) with its
// reconstruction swapped for libpikgpu at the reference's own function
// boundaries. Nothing of the reference is copied or patched: this
// executable defines five of the library's exported functions, and the
// dynamic linker binds the library's calls to these definitions (symbol
// interposition; the library is built with -fPIC and default visibility,
// so its cross-file calls go through the PLT / GOT). The overrides reach the
// library's own definitions through dlsym(RTLD_NEXT).
//
// The hook points are those of an `#ifdef PIKGPU` build of the decoder:
//  * AdaptiveDCReconstruction (called by DecodeDCGroups,
//    pik/compressed_dc.cc:549): keeps a copy of the frame's dequantised DC
//    (DequantDC's output, pik/compressed_dc.cc:181-225), then runs the
//    reference's own smoothing for the CPU caches.
//  * DecodeFromBitstream<true> (pik/compressed_image.cc:720-813, called per
//    group from the ThreadPool, pik/pik_frame.cc:906-916): runs the
//    reference's own, then -- the first call of the decode, under a mutex -- starts
//    the GPU frame from the decoder's frame state (pikgpu_frame_begin) and
//    hands the group's int16 coefficients to the GPU
//    (pikgpu_frame_set_group_ac), from the pool thread.
//  * DecodeAC (pik/entropy_coder.cc:1149, called per 64x64 tile by
//    DecodeFromBitstream, :775-779): the reference decodes the tile into a
//    tile-sized buffer that the next tile overwrites, so the hook copies
//    each decoded tile into the group's coefficient planes, applying the
//    reference's un-scatter step (:780-801, with its own
//    AcStrategy::GatherCoefficients) to the copy. The reference's DoAC still
//    runs on the CPU (it is inlined into DecodeFromBitstream, out of reach
//    of the dynamic linker); a patched build of the decoder drops it.
//  * ReconOpsinImage (pik/pik_frame.cc:925-928): skipped; the GPU
//    reconstructs the whole frame.
//  * FinalizeFrameDecoding (pik/pik_frame.cc:1149-1152): one
//    pikgpu_reconstruct into the decoder's opsin image, which the reference
//    then treats as linear sRGB, as after its own FinalizeFrameDecoding.
//
// The reference keeps only the dequantised DC (DequantDC runs inside
// compressed_dc.cc's anonymous namespace, out of reach), while the ABI takes
// the quantised DC. It is recovered by inverting DequantDC's two steps
// (q_Y = dc_Y / mul_Y; q_XB = (dc_XB - ytox_dc * dc_Y) / mul_XB, rounded to
// the nearest integer) and accepted only if recomputing DequantDC from the
// recovered integers reproduces every dequantised value bit for bit.
//
// Usage: dpik_gpu in.pik out.f32 [fp32|split_bf16|split_bf16x3|validate]
//                 [threads] [reps]
// out.f32: int32 xsize, int32 ysize, then 3 planes of ysize x xsize floats
// (linear RGB, 0..255 scale, as PikToPixels leaves io.color()). Prints the
// number of calls each override took, and with reps > 1 the wall time of
// each PikToPixels call (the output is the last one's). `validate` needs no GPU: it builds
// the frame parameters from the decoder state, recovers the quantised DC
// and checks them with pikgpu_validate, then stops before the
// reconstruction (printing "validated" and exiting 0 if they pass); its
// out.f32 holds int32 Bx, By, the quantised DC (3 x By x Bx int16) and the
// coefficients the groups would upload (3 x By x Bx * 64 int16).

#include <dlfcn.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "pik/ac_strategy.h"
#include "pik/adaptive_reconstruction.h"
#include "pik/ans_decode.h"
#include "pik/block_dictionary.h"
#include "pik/codec.h"
#include "pik/color_correlation.h"
#include "pik/compressed_image.h"
#include "pik/compressed_image_fwd.h"
#include "pik/data_parallel.h"
#include "pik/entropy_coder.h"
#include "pik/headers.h"
#include "pik/image.h"
#include "pik/noise.h"
#include "pik/pik.h"
#include "pik/pik_info.h"
#include "pik/pik_params.h"
#include "pik/quant_weights.h"
#include "pik/quantizer.h"

#include "pikgpu.h"

namespace {

pikgpu_ctx* g_ctx = nullptr;
// The image size from the file header (read in main before decoding):
// pikgpu_frame_begin needs it before the decoder reaches
// FinalizeFrameDecoding, which is the first hook that is given it.
uint32_t g_xsize = 0, g_ysize = 0;
std::mutex g_begin_mu;
bool g_begun = false;  // pikgpu_frame_begin done for the current decode
int g_begin_rc = 0;
std::string g_error;
pik::Image3F g_dc_dequant;  // frame DC after DequantDC

// The group a pool thread is decoding (set by the DecodeFromBitstream hook
// for the DecodeAC hooks it calls): its block rectangle in the frame, the
// frame's strategies, and its un-scattered coefficients (3 planes of
// ysize rows x xsize * 64 int16).
struct GroupCapture {
  size_t x0_blocks, y0_blocks, xsize_blocks, ysize_blocks;
  const pik::FrameDecCache* fdc;
  std::vector<int16_t> ac[3];
  pik::Image3S tile;  // scratch for the un-scatter
};
thread_local GroupCapture* t_cap = nullptr;

// Validation only: the frame's quantised DC and coefficients as the hooks
// pass them to the ABI (written to the output file for comparison).
bool g_validate_only = false;
std::vector<int16_t> g_qdc, g_frame_ac;
size_t g_bx = 0, g_by = 0;
std::atomic<int> g_calls_dc{0}, g_calls_groups{0}, g_calls_recon{0},
    g_calls_finalize{0};

void* Next(const char* symbol) {
  void* p = dlsym(RTLD_NEXT, symbol);
  if (!p) {
    fprintf(stderr, "dpik_gpu: %s not found in the reference library\n",
            symbol);
    abort();
  }
  return p;
}

template <typename T>
std::vector<T> Pack(const pik::Image<T>& img) {
  std::vector<T> v(img.xsize() * img.ysize());
  for (size_t y = 0; y < img.ysize(); ++y) {
    memcpy(v.data() + y * img.xsize(), img.ConstRow(y),
           img.xsize() * sizeof(T));
  }
  return v;
}

// The quantised DC from the dequantised one (see the file comment); false if
// any value does not round-trip.
bool RecoverQuantizedDC(const pik::Quantizer& quantizer,
                        const pik::ColorCorrelationMap& cmap,
                        std::vector<int16_t>* q) {
  const pik::Image3F& dc = g_dc_dequant;
  const size_t bx = dc.xsize(), by = dc.ysize();
  float mul_dc[3];
  for (int c = 0; c < 3; ++c) {
    mul_dc[c] = quantizer.DequantMatrix(0, pik::kQuantKindDCT8, c)[0] *
                quantizer.inv_quant_dc();
  }
  const float y_mul[3] = {
      pik::ColorCorrelationMap::YtoX(1.0f, cmap.ytox_dc), 0.f,
      pik::ColorCorrelationMap::YtoB(1.0f, cmap.ytob_dc)};
  q->assign(3 * bx * by, 0);
  for (size_t y = 0; y < by; ++y) {
    const float* row_y = dc.ConstPlaneRow(1, y);
    for (int c : {1, 0, 2}) {
      const float* row = dc.ConstPlaneRow(c, y);
      int16_t* out = q->data() + (c * by + y) * bx;
      for (size_t x = 0; x < bx; ++x) {
        const float rest = c == 1 ? row[x] : row[x] - y_mul[c] * row_y[x];
        const long v = lrintf(rest / mul_dc[c]);
        if (v < -32768 || v > 32767) return false;
        out[x] = int16_t(v);
        // DequantDC's arithmetic: q * mul (Y), y_mul * Y + q * mul (X, B).
        const float dq = float(out[x]) * mul_dc[c];
#if defined(__FMA__)  // the AVX2 flavour's mul_add is fused
        const float back = c == 1 ? dq : fmaf(y_mul[c], row_y[x], dq);
#else
        const float back = c == 1 ? dq : y_mul[c] * row_y[x] + dq;
#endif
        if (memcmp(&back, &row[x], sizeof(float)) != 0) return false;
      }
    }
  }
  return true;
}

int BeginFrame(const pik::FrameHeader& hd, const pik::Quantizer& quantizer,
               const pik::ColorCorrelationMap& cmap,
               const pik::FrameDecCache& fdc) {
  std::vector<int16_t> qdc;
  if (!RecoverQuantizedDC(quantizer, cmap, &qdc)) {
    g_error = "the quantised DC did not round-trip through DequantDC";
    return -1;
  }
  const pik::DequantMatrices& m = fdc.matrices;
  std::vector<uint32_t> offsets(pik::kNumPredefinedTables *
                                pik::kNumQuantKinds * 3);
  for (size_t t = 0; t < pik::kNumPredefinedTables; ++t) {
    for (size_t k = 0; k < pik::kNumQuantKinds; ++k) {
      for (int c = 0; c < 3; ++c) {
        offsets[(t * pik::kNumQuantKinds + k) * 3 + c] =
            m.MatrixOffset(t, k, c);
      }
    }
  }
  const auto cf = Pack(fdc.dequant_control_field);
  const auto ytox = Pack(cmap.ytox_map), ytob = Pack(cmap.ytob_map);
  const auto acs = Pack(fdc.ac_strategy.ConstRaw());
  const auto qf = Pack(fdc.raw_quant_field);
  const auto lut = Pack(fdc.ar_sigma_lut_ids);
  pikgpu_frame_params p = {};
  p.xsize = g_xsize;
  p.ysize = g_ysize;
  p.flags = hd.flags;
  p.gaborish = static_cast<uint32_t>(hd.gaborish);
  p.predict_lf = hd.predict_lf;
  p.predict_hf = hd.predict_hf;
  p.have_adaptive_reconstruction = hd.have_adaptive_reconstruction;
  p.epf_enable_adaptive = hd.epf_params.enable_adaptive;
  p.epf_sigma = hd.epf_params.sigma;
  p.epf_use_sharpened = hd.epf_params.use_sharpened;
  // Quantizer::global_scale_ from its inverse (pik/quantizer.h:131-139).
  p.global_scale = int(65536.0f / quantizer.InvGlobalScale() + 0.5f);
  p.quant_dc = quantizer.QuantDC();
  p.dequant_table = m.Matrix(0, pik::kQuantKindDCT8, 0) -
                    m.MatrixOffset(0, pik::kQuantKindDCT8, 0);
  p.dequant_table_size = uint32_t(m.Size());
  p.dequant_offsets = offsets.data();
  p.num_dequant_tables = pik::kNumPredefinedTables;
  p.dequant_control_field = cf.data();
  p.dequant_map = &fdc.dequant_map[0][0];
  p.ytox_map = ytox.data();
  p.ytob_map = ytob.data();
  p.ytox_dc = cmap.ytox_dc;
  p.ytob_dc = cmap.ytob_dc;
  p.ac_strategy = acs.data();
  p.raw_quant_field = qf.data();
  p.ar_sigma_lut_ids = lut.data();
  p.quantized_dc = qdc.data();
  char msg[256] = {0};
  if (pikgpu_validate(&p, msg, sizeof(msg)) != PIKGPU_OK) {
    g_error = std::string("pikgpu_validate: ") + msg;
    return -1;
  }
  if (g_validate_only) {
    g_qdc = qdc;
    g_bx = (g_xsize + 7) / 8, g_by = (g_ysize + 7) / 8;
    g_frame_ac.assign(3 * g_by * g_bx * 64, 0);
    return 0;
  }
  if (pikgpu_frame_begin(g_ctx, &p) != PIKGPU_OK) {
    g_error = pikgpu_last_error(g_ctx);
    return -1;
  }
  return 0;
}

}  // namespace

namespace pik {

void AdaptiveDCReconstruction(Image3F& dc, const Quantizer& quantizer,
                              ThreadPool* pool) {
  using Fn = void (*)(Image3F&, const Quantizer&, ThreadPool*);
  static const Fn next = reinterpret_cast<Fn>(
      Next("_ZN3pik24AdaptiveDCReconstructionERNS_6Image3IfEERKNS_9"
           "QuantizerEPNS_10ThreadPoolE"));
  g_dc_dequant = CopyImage(dc);
  ++g_calls_dc;
  next(dc, quantizer, pool);
}

template <>
bool DecodeFromBitstream<true>(
    const FrameHeader& frame_header, const GroupHeader& header,
    const PaddedBytes& compressed, BitReader* reader, const Rect& group_rect,
    MultipassHandler* handler, const size_t xsize_blocks,
    const size_t ysize_blocks, const ColorCorrelationMap& cmap,
    const Rect& cmap_rect, NoiseParams* noise_params,
    const Quantizer& quantizer, FrameDecCache* PIK_RESTRICT frame_dec_cache,
    GroupDecCache* PIK_RESTRICT group_dec_cache, PikInfo* aux_out) {
  using Fn = bool (*)(const FrameHeader&, const GroupHeader&,
                      const PaddedBytes&, BitReader*, const Rect&,
                      MultipassHandler*, size_t, size_t,
                      const ColorCorrelationMap&, const Rect&, NoiseParams*,
                      const Quantizer&, FrameDecCache*, GroupDecCache*,
                      PikInfo*);
  static const Fn next = reinterpret_cast<Fn>(Next(
      "_ZN3pik19DecodeFromBitstreamILb1EEEbRKNS_11FrameHeaderERKNS_11"
      "GroupHeaderERKNS_11PaddedBytesEPNS_9BitReaderERKNS_4RectEPNS_16"
      "MultipassHandlerEmmRKNS_19ColorCorrelationMapESE_PNS_11NoiseParamsE"
      "RKNS_9QuantizerEPNS_13FrameDecCacheEPNS_13GroupDecCacheEPNS_7"
      "PikInfoE"));
  thread_local GroupCapture cap;
  cap.x0_blocks = group_rect.x0() / kBlockDim;
  cap.y0_blocks = group_rect.y0() / kBlockDim;
  cap.fdc = frame_dec_cache;
  cap.xsize_blocks = xsize_blocks;
  cap.ysize_blocks = ysize_blocks;
  for (auto& plane : cap.ac) plane.assign(ysize_blocks * xsize_blocks * 64, 0);
  t_cap = &cap;
  const bool ok = next(frame_header, header, compressed, reader, group_rect,
                       handler, xsize_blocks, ysize_blocks, cmap, cmap_rect,
                       noise_params, quantizer, frame_dec_cache,
                       group_dec_cache, aux_out);
  t_cap = nullptr;
  if (!ok) return false;
  {
    std::lock_guard<std::mutex> lock(g_begin_mu);
    if (!g_begun) {
      g_begin_rc =
          BeginFrame(frame_header, quantizer, cmap, *frame_dec_cache);
      g_begun = true;
    }
    if (g_begin_rc != 0) return false;
  }
  // group_rect: the group's pixels (512x512 groups, row-major).
  const uint32_t groups_x = (g_xsize + 511) / 512;
  const uint32_t gi = uint32_t(group_rect.y0() / 512) * groups_x +
                      uint32_t(group_rect.x0() / 512);
  const int16_t* planes[3] = {cap.ac[0].data(), cap.ac[1].data(),
                              cap.ac[2].data()};
  ++g_calls_groups;
  if (g_validate_only) {
    for (int c = 0; c < 3; ++c) {
      for (size_t by = 0; by < ysize_blocks; ++by) {
        memcpy(g_frame_ac.data() +
                   ((c * g_by) + cap.y0_blocks + by) * g_bx * 64 +
                   cap.x0_blocks * 64,
               planes[c] + by * xsize_blocks * 64,
               xsize_blocks * 64 * sizeof(int16_t));
      }
    }
    return true;
  }
  if (pikgpu_frame_set_group_ac(g_ctx, gi, planes, xsize_blocks * 64) !=
      PIKGPU_OK) {
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    g_error = pikgpu_last_error(g_ctx);
    return false;
  }
  return true;
}

bool DecodeAC(const std::vector<uint8_t>& context_map,
              const int32_t* PIK_RESTRICT coeff_order,
              BitReader* PIK_RESTRICT br, ANSSymbolReader* decoder,
              Image3S* PIK_RESTRICT ac, const Rect& rect,
              Image3I* PIK_RESTRICT tmp_num_nzeroes) {
  using Fn = bool (*)(const std::vector<uint8_t>&, const int32_t*,
                      BitReader*, ANSSymbolReader*, Image3S*, const Rect&,
                      Image3I*);
  static const Fn next = reinterpret_cast<Fn>(
      Next("_ZN3pik8DecodeACERKSt6vectorIhSaIhEEPKiPNS_9BitReaderEPNS_15"
           "ANSSymbolReaderEPNS_6Image3IsEERKNS_4RectEPNSB_IiEE"));
  if (!next(context_map, coeff_order, br, decoder, ac, rect,
            tmp_num_nzeroes)) {
    return false;
  }
  GroupCapture* cap = t_cap;
  if (!cap) return true;
  // The tile (rect: block units within the group) sits at the top left of
  // `ac`. Copy it, un-scatter the copy as the reference does, and place it.
  const size_t row_len = rect.xsize() * kDCTBlockSize;
  if (cap->tile.xsize() < ac->xsize() || cap->tile.ysize() < ac->ysize()) {
    cap->tile = Image3S(ac->xsize(), ac->ysize());
  }
  for (int c = 0; c < 3; ++c) {
    for (size_t by = 0; by < rect.ysize(); ++by) {
      memcpy(cap->tile.PlaneRow(c, by), ac->ConstPlaneRow(c, by),
             row_len * sizeof(int16_t));
    }
  }
  const size_t stride = cap->tile.PixelsPerRow();
  const Rect acs_rect(cap->x0_blocks, cap->y0_blocks, cap->xsize_blocks,
                      cap->ysize_blocks);
  SIMD_ALIGN int16_t unscattered[AcStrategy::kMaxCoeffArea];
  for (int c = 0; c < 3; ++c) {
    for (size_t by = 0; by < rect.ysize(); ++by) {
      AcStrategyRow acs_row =
          cap->fdc->ac_strategy.ConstRow(acs_rect, by + rect.y0());
      int16_t* PIK_RESTRICT row = cap->tile.PlaneRow(c, by);
      for (size_t bx = 0; bx < rect.xsize(); ++bx) {
        AcStrategy acs = acs_row[bx + rect.x0()];
        if (!acs.IsFirstBlock()) continue;
        int16_t* block = row + bx * kDCTBlockSize;
        acs.GatherCoefficients(block, stride, unscattered,
                               acs.covered_blocks_x() * kDCTBlockSize);
        for (size_t i = 0; i < acs.covered_blocks_y(); i++) {
          memcpy(block + stride * i,
                 unscattered + acs.covered_blocks_x() * kDCTBlockSize * i,
                 sizeof(int16_t) * acs.covered_blocks_x() * kDCTBlockSize);
        }
      }
    }
    for (size_t by = 0; by < rect.ysize(); ++by) {
      memcpy(cap->ac[c].data() +
                 (rect.y0() + by) * cap->xsize_blocks * kDCTBlockSize +
                 rect.x0() * kDCTBlockSize,
             cap->tile.ConstPlaneRow(c, by), row_len * sizeof(int16_t));
    }
  }
  return true;
}

void ReconOpsinImage(const FrameHeader& frame_header,
                     const GroupHeader& header, const Quantizer& quantizer,
                     const Rect& block_group_rect,
                     FrameDecCache* PIK_RESTRICT frame_dec_cache,
                     GroupDecCache* PIK_RESTRICT group_dec_cache,
                     Image3F* PIK_RESTRICT idct, const Rect& idct_rect,
                     PikInfo* aux_out, size_t downsample) {
  ++g_calls_recon;  // the GPU reconstructs the frame at the end
}

Status FinalizeFrameDecoding(Image3F* PIK_RESTRICT idct, size_t xsize,
                             size_t ysize, const FrameHeader& frame_header,
                             const NoiseParams& noise_params,
                             const Quantizer& quantizer,
                             const BlockDictionary& dictionary,
                             ThreadPool* pool, FrameDecCache* frame_dec_cache,
                             PikInfo* aux_out, size_t downsample) {
  ++g_calls_finalize;
  if (downsample != 1) return PIK_FAILURE("dpik_gpu: downsampling");
  // A frame whose block dictionary places blocks (dots) is not on the GPU
  // path. The dictionary's members are private; its encoding equals the
  // empty dictionary's exactly when it has no entries and no positions.
  if (dictionary.Encode(nullptr) != BlockDictionary().Encode(nullptr)) {
    return PIK_FAILURE("dpik_gpu: block dictionary");
  }
  if (xsize != g_xsize || ysize != g_ysize) {
    return PIK_FAILURE("dpik_gpu: image size differs from the header's");
  }
  if (g_validate_only) {
    g_error = "validation only";
    return false;
  }
  float* rows[3] = {idct->PlaneRow(0, 0), idct->PlaneRow(1, 0),
                    idct->PlaneRow(2, 0)};
  if (pikgpu_reconstruct(g_ctx, rows, idct->PixelsPerRow(), nullptr, 0,
                         /*outputs_on_device=*/0) != PIKGPU_OK) {
    g_error = pikgpu_last_error(g_ctx);
    return PIK_FAILURE("dpik_gpu: pikgpu_reconstruct failed");
  }
  idct->ShrinkTo(xsize, ysize);
  return true;
}

}  // namespace pik

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr,
            "usage: dpik_gpu in.pik out.f32 "
            "[fp32|split_bf16|split_bf16x3|validate] [threads] [reps]\n");
    return 2;
  }
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 2;
  fseek(f, 0, SEEK_END);
  const long size = ftell(f);
  fseek(f, 0, SEEK_SET);
  pik::PaddedBytes compressed(size);
  if (fread(compressed.data(), 1, size, f) != size_t(size)) return 2;
  fclose(f);
  int form = PIKGPU_FORM_FP32;
  if (argc > 3 && !strcmp(argv[3], "split_bf16")) form = PIKGPU_FORM_SPLIT_BF16;
  if (argc > 3 && !strcmp(argv[3], "split_bf16x3")) {
    form = PIKGPU_FORM_SPLIT_BF16X3;
  }
  const bool validate_only = argc > 3 && !strcmp(argv[3], "validate");
  g_validate_only = validate_only;
  const int threads = argc > 4 ? atoi(argv[4]) : 8;

  // The image size (the file header's), which pikgpu_frame_begin needs
  // before the decoder reaches FinalizeFrameDecoding.
  {
    pik::BitReader reader(compressed.data(), compressed.size());
    pik::FileHeader container;
    if (!pik::ReadFileHeader(&reader, &container)) {
      fprintf(stderr, "dpik_gpu: cannot read the file header\n");
      return 1;
    }
    g_xsize = uint32_t(container.xsize());
    g_ysize = uint32_t(container.ysize());
  }
  if (!validate_only &&
      (pikgpu_ctx_create(0, &g_ctx) != PIKGPU_OK ||
       pikgpu_set_option(g_ctx, PIKGPU_OPT_FORM, form) != PIKGPU_OK)) {
    fprintf(stderr, "dpik_gpu: context: %s\n",
            g_ctx ? pikgpu_last_error(g_ctx) : "create failed");
    return 1;
  }

  pik::CodecContext context;
  pik::CodecInOut io(&context);
  pik::DecompressParams dparams;
  std::unique_ptr<pik::ThreadPool> pool;
  if (threads > 0) pool.reset(new pik::ThreadPool(threads));
  const int reps = argc > 5 ? std::max(1, atoi(argv[5])) : 1;
  bool ok = true;
  std::vector<double> ms;
  for (int r = 0; r < reps && ok; ++r) {
    g_begun = false;
    g_calls_dc = g_calls_groups = g_calls_recon = g_calls_finalize = 0;
    const auto t0 = std::chrono::steady_clock::now();
    ok = pik::PikToPixels(dparams, compressed, &io, nullptr, pool.get());
    const auto t1 = std::chrono::steady_clock::now();
    ms.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
  }
  if (reps > 1) {
    printf("PikToPixels ms:");
    for (double v : ms) printf(" %.3f", v);
    printf("\n");
  }
  printf("overrides: AdaptiveDCReconstruction %d, DecodeFromBitstream %d, "
         "ReconOpsinImage %d, FinalizeFrameDecoding %d\n",
         g_calls_dc.load(), g_calls_groups.load(), g_calls_recon.load(),
         g_calls_finalize.load());
  if (validate_only) {
    const bool passed = g_begin_rc == 0 && g_calls_finalize.load() == 1;
    printf("%s%s\n", passed ? "validated" : "not validated: ",
           passed ? "" : g_error.c_str());
    if (!passed) return 1;
    FILE* out = fopen(argv[2], "wb");
    if (!out) return 2;
    const int32_t dims[2] = {int32_t(g_bx), int32_t(g_by)};
    fwrite(dims, sizeof(dims), 1, out);
    fwrite(g_qdc.data(), sizeof(int16_t), g_qdc.size(), out);
    fwrite(g_frame_ac.data(), sizeof(int16_t), g_frame_ac.size(), out);
    fclose(out);
    return 0;
  }
  if (!ok) {
    fprintf(stderr, "dpik_gpu: PikToPixels failed: %s\n", g_error.c_str());
    pikgpu_ctx_destroy(g_ctx);
    return 1;
  }
  const pik::Image3F& color = io.color();
  FILE* out = fopen(argv[2], "wb");
  if (!out) return 2;
  const int32_t dims[2] = {int32_t(color.xsize()), int32_t(color.ysize())};
  fwrite(dims, sizeof(dims), 1, out);
  for (int c = 0; c < 3; ++c) {
    for (size_t y = 0; y < color.ysize(); ++y) {
      fwrite(color.ConstPlaneRow(c, y), sizeof(float), color.xsize(), out);
    }
  }
  fclose(out);
  pikgpu_ctx_destroy(g_ctx);
  return 0;
}
