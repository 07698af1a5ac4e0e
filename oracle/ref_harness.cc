// Test-infrastructure harness around the reference decoder built from the
// unmodified google/pik sources (see oracle/Makefile). It is linked only
// into oracle/_ref/libpikref_{avx2,scalar}.so and used only by tests/,
// __graft_entry__.smoke() and bench.py's reference/CPU-baseline leg.
//
// It provides:
//  * pikref_encode: the reference encoder (PixelsToPik, pik/pik.cc:56-86)
//    on linear-sRGB float planes, producing a bitstream;
//  * pikref_frozen_*: decodes a bitstream exactly like PikPassToPixels
//    (pik/pik_frame.cc:935-1065) and DecodeFromBitstream
//    (pik/compressed_image.cc:720-813) but stops at the boundary of the
//    reconstruction path, keeping the integer coefficients, side information
//    and decoder-side scalars ("frozen frame");
//  * pikref_run_stages: runs the reference's own reconstruction on a frozen
//    frame -- DequantImageAC + ReconOpsinImage per group, then the stages of
//    FinalizeFrameDecoding (pik/compressed_image.cc:1144-1181) called one by
//    one -- returning every stage's planes;
//  * pikref_reconstruct_timed: the same reconstruction on a ThreadPool, timed
//    (the CPU baseline);
//  * small probes of individual reference functions (transforms, EPF
//    weights, opsin inverse matrix) for pinning the C++ restatement.

#include <stdint.h>
#include <string.h>

#include <atomic>
#include <chrono>
#include <string>
#include <memory>
#include <mutex>
#include <vector>

#include "pik/ac_strategy.h"
#include "pik/adaptive_reconstruction.h"
#include "pik/ans_decode.h"
#include "pik/block_dictionary.h"
#include "pik/codec.h"
#include "pik/codec_pnm.h"
#include "pik/color_correlation.h"
#include "pik/common.h"
#include "pik/compressed_dc.h"
#include "pik/compressed_image.h"
#include "pik/compressed_image_fwd.h"
#include "pik/data_parallel.h"
#include "pik/entropy_coder.h"
#include "pik/epf.h"
#include "pik/gaborish.h"
#include "pik/headers.h"
#include "pik/image.h"
#include "pik/noise.h"
#include "pik/opsin_image.h"
#include "pik/opsin_inverse.h"
#include "pik/opsin_params.h"
#include "pik/pik.h"
#include "pik/pik_info.h"
#include "pik/pik_params.h"
#include "pik/quant_weights.h"
#include "pik/quantizer.h"
#include "pik/simd/simd.h"
#include "pik/single_image_handler.h"
#include "pik/size_coder.h"

using namespace pik;

namespace {

// Same size coder the reference uses for the DC-group and AC-group tables
// of contents (pik/compressed_dc.cc:348, pik/pik_frame.cc:416).
using TocCoder = SizeCoderT<0x150F0E0C>;

struct Frozen {
  size_t xsize = 0, ysize = 0, xsize_blocks = 0, ysize_blocks = 0;
  FrameHeader header;
  std::unique_ptr<FrameDecCache> fdc;
  std::unique_ptr<Quantizer> quantizer;  // decoder-side (Quantizer::Decode)
  ColorCorrelationMap cmap;
  BlockDictionary dictionary;
  Image3S quantized_dc;  // Bx x By (after ExpandDC)
  Image3S quantized_ac;  // Bx*64 x By, un-scattered (GroupDecCache::ac layout)
  Image3F dc_smoothed;   // FrameDecCache::dc after AdaptiveDCReconstruction
};

void CopyPlaneOut(const Image3F& img, float* dst) {
  const size_t xs = img.xsize(), ys = img.ysize();
  for (int c = 0; c < 3; ++c) {
    for (size_t y = 0; y < ys; ++y) {
      memcpy(dst + (c * ys + y) * xs, img.ConstPlaneRow(c, y),
             xs * sizeof(float));
    }
  }
}

Status DecodeToFrozen(const PaddedBytes& compressed, int override_ar,
                      int override_gaborish, Frozen* f) {
  BitReader reader(compressed.data(), compressed.size());
  FileHeader container;
  PIK_RETURN_IF_ERROR(ReadFileHeader(&reader, &container));
  if (container.preview.size_bits != 0) {
    reader.SkipBits(container.preview.size_bits);
  }
  f->xsize = container.xsize();
  f->ysize = container.ysize();
  const size_t padded_xsize = DivCeil(f->xsize, kBlockDim) * kBlockDim;
  const size_t padded_ysize = DivCeil(f->ysize, kBlockDim) * kBlockDim;
  f->xsize_blocks = padded_xsize / kBlockDim;
  f->ysize_blocks = padded_ysize / kBlockDim;

  FrameHeader& header = f->header;
  PIK_RETURN_IF_ERROR(ReadPassHeader(&reader, &header));
  PIK_RETURN_IF_ERROR(reader.JumpToByteBoundary());
  if (header.encoding != ImageEncoding::kPasses) {
    return PIK_FAILURE("only kPasses frames are on the reconstruction path");
  }
  if (header.num_passes != 1) return PIK_FAILURE("multipass unsupported");
  // Decoder-side overrides, as OverridePassFlags (pik/pik_frame.cc:100-121).
  if (override_ar == 0) header.have_adaptive_reconstruction = false;
  if (override_ar == 1) header.have_adaptive_reconstruction = true;
  if (override_gaborish >= 0) {
    header.gaborish = GaborishStrength(override_gaborish);
  }

  f->fdc.reset(new FrameDecCache);
  FrameDecCache& fdc = *f->fdc;
  fdc.use_new_dc = false;
  fdc.grayscale = header.flags & FrameHeader::kGrayscaleOpt;
  fdc.ac_strategy = AcStrategyImage(f->xsize_blocks, f->ysize_blocks);
  fdc.raw_quant_field = ImageI(f->xsize_blocks, f->ysize_blocks);
  fdc.ar_sigma_lut_ids = ImageB(f->xsize_blocks, f->ysize_blocks);
  fdc.dequant_control_field =
      ImageB(DivCeil(f->xsize, kTileDim), DivCeil(f->ysize, kTileDim));
  f->cmap = ColorCorrelationMap(f->xsize, f->ysize);
  f->quantizer.reset(new Quantizer(&fdc.matrices, 0, 0));

  PIK_RETURN_IF_ERROR(fdc.matrices.Decode(&reader));
  PIK_RETURN_IF_ERROR(f->quantizer->Decode(&reader));
  PIK_RETURN_IF_ERROR(reader.JumpToByteBoundary());
  DecodeColorMap(&reader, &f->cmap.ytob_map, &f->cmap.ytob_dc);
  DecodeColorMap(&reader, &f->cmap.ytox_map, &f->cmap.ytox_dc);

  // Quantized DC integers: replay the DC-group entropy decode
  // (DecodeDCGroups' TOC walk, pik/compressed_dc.cc:455-505, then the
  // DecodeImage + ExpandDC steps of DecodeDCGroup, :289-302) on a copy of
  // the reader. The real DecodeDCGroups below then decodes everything else.
  f->quantized_dc = Image3S(f->xsize_blocks, f->ysize_blocks);
  {
    BitReader dc_reader = reader;
    const size_t xg = DivCeil(f->xsize_blocks, kDcGroupDimInBlocks);
    const size_t yg = DivCeil(f->ysize_blocks, kDcGroupDimInBlocks);
    std::vector<size_t> offsets{0};
    for (size_t i = 0; i < xg * yg; ++i) {
      offsets.push_back(offsets.back() + TocCoder::Decode(&dc_reader));
    }
    PIK_RETURN_IF_ERROR(dc_reader.JumpToByteBoundary());
    const size_t begin = dc_reader.Position();
    for (size_t gi = 0; gi < xg * yg; ++gi) {
      BitReader gr(compressed.data(), begin + offsets[gi + 1]);
      gr.SkipBits((begin + offsets[gi]) * kBitsPerByte);
      const Rect rect((gi % xg) * kDcGroupDimInBlocks,
                      (gi / xg) * kDcGroupDimInBlocks, kDcGroupDimInBlocks,
                      kDcGroupDimInBlocks, f->xsize_blocks, f->ysize_blocks);
      Image3S q(rect.xsize(), rect.ysize());
      ImageS dc_y(rect.xsize(), rect.ysize());
      ImageS res(rect.xsize() * 2, rect.ysize());
      ImageS exp(rect.xsize() * 2, rect.ysize());
      if (!DecodeImage(&gr, Rect(q), &q)) {
        return PIK_FAILURE("DC image decode failed");
      }
      ExpandDC(Rect(q), &q, &dc_y, &res, &exp);
      for (int c = 0; c < 3; ++c) {
        for (size_t y = 0; y < rect.ysize(); ++y) {
          memcpy(rect.PlaneRow(&f->quantized_dc, c, y), q.ConstPlaneRow(c, y),
                 rect.xsize() * sizeof(int16_t));
        }
      }
    }
  }

  std::vector<GroupDecCache> group_dec_caches(1);
  SingleImageManager manager;
  manager.StartPass(header);
  PIK_RETURN_IF_ERROR(DecodeDCGroups(
      &reader, compressed, header, f->xsize_blocks, f->ysize_blocks,
      *f->quantizer, f->cmap, /*pool=*/nullptr, &manager, &fdc,
      &group_dec_caches, /*aux_out=*/nullptr));
  PIK_RETURN_IF_ERROR(f->dictionary.Decode(&reader, padded_xsize, padded_ysize));
  PIK_RETURN_IF_ERROR(
      DecodeDequantControlField(&reader, &fdc.dequant_control_field));
  PIK_RETURN_IF_ERROR(DecodeDequantControlFieldMap(
      &reader, fdc.raw_quant_field, fdc.dequant_control_field,
      fdc.dequant_map));
  f->dc_smoothed = CopyImage(fdc.dc);

  // AC groups (PikPassToPixels TOC :1070-1104, PikGroupToPixels :846-931,
  // DecodeFromBitstream :720-813), keeping the un-scattered integers.
  const size_t xsize_groups = DivCeil(f->xsize, kGroupDim);
  const size_t ysize_groups = DivCeil(f->ysize, kGroupDim);
  const size_t num_groups = xsize_groups * ysize_groups;
  std::vector<size_t> offsets{0};
  for (size_t i = 0; i < num_groups; ++i) {
    offsets.push_back(offsets.back() + TocCoder::Decode(&reader));
  }
  PIK_RETURN_IF_ERROR(reader.JumpToByteBoundary());
  const size_t codes_begin = reader.Position();
  f->quantized_ac = Image3S(f->xsize_blocks * kDCTBlockSize, f->ysize_blocks);
  ZeroFillImage(&f->quantized_ac);

  for (size_t gi = 0; gi < num_groups; ++gi) {
    BitReader gr(compressed.data(), codes_begin + offsets[gi + 1]);
    gr.SkipBits((codes_begin + offsets[gi]) * kBitsPerByte);
    GroupHeader gh;
    gh.nonserialized_have_alpha = header.has_alpha;
    PIK_RETURN_IF_ERROR(ReadGroupHeader(&gr, &gh));
    PIK_RETURN_IF_ERROR(gr.JumpToByteBoundary());
    const Rect group_rect((gi % xsize_groups) * kGroupDim,
                          (gi / xsize_groups) * kGroupDim, kGroupDim,
                          kGroupDim, f->xsize, f->ysize);
    const size_t gx0 = group_rect.x0() / kBlockDim;
    const size_t gy0 = group_rect.y0() / kBlockDim;
    const size_t gxs = DivCeil(group_rect.xsize(), kBlockDim);
    const size_t gys = DivCeil(group_rect.ysize(), kBlockDim);
    const Rect group_acs_qf_rect(gx0, gy0, gxs, gys);

    NoiseParams noise_params;
    PIK_RETURN_IF_ERROR(DecodeNoise(&gr, &noise_params));
    int coeff_order[kOrderContexts * kDCTBlockSize];
    for (size_t c = 0; c < kOrderContexts; ++c) {
      DecodeCoeffOrder(&coeff_order[c * kDCTBlockSize], &gr);
    }
    PIK_RETURN_IF_ERROR(gr.JumpToByteBoundary());
    ANSCode code;
    std::vector<uint8_t> context_map;
    PIK_RETURN_IF_ERROR(
        DecodeHistograms(&gr, kNumContexts, 256, &code, &context_map));
    PIK_RETURN_IF_ERROR(gr.JumpToByteBoundary());
    ANSSymbolReader ac_decoder(&code);

    Image3S tile_ac(kTileDimInBlocks * kDCTBlockSize, kTileDimInBlocks);
    Image3I num_nzeroes(kTileDimInBlocks, kTileDimInBlocks);
    SIMD_ALIGN int16_t unscattered[AcStrategy::kMaxCoeffArea];
    const size_t stride = tile_ac.PixelsPerRow();
    const size_t xt = DivCeil(gxs, kTileDimInBlocks);
    const size_t yt = DivCeil(gys, kTileDimInBlocks);
    for (size_t task = 0; task < xt * yt; ++task) {
      const Rect rect((task % xt) * kTileDimInBlocks,
                      (task / xt) * kTileDimInBlocks, kTileDimInBlocks,
                      kTileDimInBlocks, gxs, gys);
      if (!DecodeAC(context_map, coeff_order, &gr, &ac_decoder, &tile_ac, rect,
                    &num_nzeroes)) {
        return PIK_FAILURE("Failed to decode AC.");
      }
      for (int c = 0; c < 3; ++c) {
        for (size_t by = 0; by < rect.ysize(); by++) {
          AcStrategyRow acs_row =
              fdc.ac_strategy.ConstRow(group_acs_qf_rect, by + rect.y0());
          int16_t* PIK_RESTRICT row = tile_ac.PlaneRow(c, by);
          for (size_t bx = 0; bx < rect.xsize(); bx++) {
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
          // Copy the (un-scattered) tile row into the frame image. Multi-
          // block transforms that straddle the tile's right/bottom edge are
          // written by the tile holding their first block, as in the
          // reference, and the stride spans the whole tile row.
          const size_t fy = gy0 + rect.y0() + by;
          int16_t* out = f->quantized_ac.PlaneRow(c, fy) +
                         (gx0 + rect.x0()) * kDCTBlockSize;
          memcpy(out, row, rect.xsize() * kDCTBlockSize * sizeof(int16_t));
        }
      }
    }
    if (!ac_decoder.CheckANSFinalState()) {
      return PIK_FAILURE("ANS checksum failure.");
    }
  }
  return true;
}

thread_local std::string g_error;
thread_local bool g_dictionary_changed = false;

// The EPF weight table must be initialised before any filtering; the
// reference does this in CodecContext's constructor
// (pik/codec_impl.cc:185-189).
void InitEpf() {
  static std::once_flag once;
  std::call_once(once, [] { TargetBitfield().Foreach(InitEdgePreservingFilter()); });
}

// Reconstruction on a frozen frame using the reference functions, with each
// stage exported. stages[] (nullable entries):
//  0 dc (Bx x By) 1 dequant_ac (Bx*64 x By) 2 idct (padded) 3 smoothed
//  4 epf (pre-clamp) 5 ar 6 pre-opsin (after gaborish #2, unpadded)
//  7 linear (unpadded)
Status RunStages(const Frozen& f, ThreadPool* pool, float* const* stages,
                 double* seconds) {
  FrameDecCache fdc;
  fdc.use_new_dc = false;
  fdc.grayscale = false;
  fdc.dc = CopyImage(f.dc_smoothed);
  fdc.raw_quant_field = CopyImage(f.fdc->raw_quant_field);
  fdc.ac_strategy = f.fdc->ac_strategy.Copy();
  fdc.dequant_control_field = CopyImage(f.fdc->dequant_control_field);
  memcpy(fdc.dequant_map, f.fdc->dequant_map, sizeof(fdc.dequant_map));
  fdc.ar_sigma_lut_ids = CopyImage(f.fdc->ar_sigma_lut_ids);
  // Quantizer with the decoder's scalars and a raw quant field (needed by
  // DequantImageAC's size checks and Quantizer::Copy).
  Quantizer quantizer = f.quantizer->Copy(Rect(0, 0, 0, 0));
  quantizer.SetRawQuantField(CopyImage(f.fdc->raw_quant_field));

  const auto t0 = std::chrono::steady_clock::now();
  const size_t padded_x = f.xsize_blocks * kBlockDim;
  const size_t padded_y = f.ysize_blocks * kBlockDim;
  Image3F opsin(padded_x, padded_y);
  Image3F dequant_ac;
  if (stages && stages[1]) {
    dequant_ac = Image3F(f.xsize_blocks * kDCTBlockSize, f.ysize_blocks);
  }
  const size_t xsize_groups = DivCeil(f.xsize, kGroupDim);
  const size_t ysize_groups = DivCeil(f.ysize, kGroupDim);
  const size_t num_groups = xsize_groups * ysize_groups;
  std::vector<GroupDecCache> caches(NumThreads(pool));
  std::atomic<int> errors{0};
  GroupHeader gh;
  const auto process_group = [&](const int gi, const int thread) {
    const Rect group_rect((gi % xsize_groups) * kGroupDim,
                          (gi / xsize_groups) * kGroupDim, kGroupDim,
                          kGroupDim, f.xsize, f.ysize);
    const Rect padded_rect(group_rect.x0(), group_rect.y0(),
                           DivCeil(group_rect.xsize(), kBlockDim) * kBlockDim,
                           DivCeil(group_rect.ysize(), kBlockDim) * kBlockDim);
    const Rect block_rect(padded_rect.x0() / kBlockDim,
                          padded_rect.y0() / kBlockDim,
                          padded_rect.xsize() / kBlockDim,
                          padded_rect.ysize() / kBlockDim);
    const Rect cmap_rect(block_rect.x0() / kColorTileDimInBlocks,
                         block_rect.y0() / kColorTileDimInBlocks,
                         DivCeil(block_rect.xsize(), kColorTileDimInBlocks),
                         DivCeil(block_rect.ysize(), kColorTileDimInBlocks));
    GroupDecCache* gdc = &caches[thread];
    InitializeDecCache(fdc, padded_rect, gdc);
    Image3S q(block_rect.xsize() * kDCTBlockSize, block_rect.ysize());
    for (int c = 0; c < 3; ++c) {
      for (size_t y = 0; y < block_rect.ysize(); ++y) {
        memcpy(q.PlaneRow(c, y),
               f.quantized_ac.ConstPlaneRow(c, block_rect.y0() + y) +
                   block_rect.x0() * kDCTBlockSize,
               block_rect.xsize() * kDCTBlockSize * sizeof(int16_t));
      }
    }
    const Quantizer gq = quantizer.Copy(block_rect);
    // DequantImageAC reads frame-level fields through block_group_rect.
    DequantImageAC(gq, f.cmap, cmap_rect, q, &fdc, gdc, padded_rect, nullptr);
    if (dequant_ac.xsize() != 0) {
      for (int c = 0; c < 3; ++c) {
        for (size_t y = 0; y < block_rect.ysize(); ++y) {
          memcpy(dequant_ac.PlaneRow(c, block_rect.y0() + y) +
                     block_rect.x0() * kDCTBlockSize,
                 gdc->ac.ConstPlaneRow(c, y),
                 block_rect.xsize() * kDCTBlockSize * sizeof(float));
        }
      }
    }
    ReconOpsinImage(f.header, gh, quantizer, block_rect, &fdc, gdc, &opsin,
                    padded_rect, nullptr, 1);
  };
  RunOnPool(pool, 0, num_groups, process_group, "harness groups");
  if (errors.load() != 0) return PIK_FAILURE("group failed");

  if (stages && stages[0]) CopyPlaneOut(fdc.dc, stages[0]);
  if (stages && stages[1]) CopyPlaneOut(dequant_ac, stages[1]);
  if (stages && stages[2]) CopyPlaneOut(opsin, stages[2]);

  // FinalizeFrameDecoding, stage by stage (pik/compressed_image.cc:1144-1181
  // and DoAdaptiveReconstruction :1113-1141).
  if (f.header.have_adaptive_reconstruction) {
    Image3F smoothed;
    const Image3F* smoothed_ptr = &opsin;
    if (f.header.gaborish != GaborishStrength::kOff) {
      PIK_RETURN_IF_ERROR(
          ConvolveGaborish(opsin, f.header.gaborish, pool, &smoothed));
      smoothed_ptr = &smoothed;
    }
    if (stages && stages[3]) CopyPlaneOut(*smoothed_ptr, stages[3]);
    Image3F filtered;
    AdaptiveReconstructionAux aux;
    if (stages && stages[4]) aux.filtered = &filtered;
    Image3F ar = AdaptiveReconstruction(
        *smoothed_ptr, opsin, quantizer, fdc.raw_quant_field,
        fdc.dequant_control_field, fdc.dequant_map, fdc.ar_sigma_lut_ids,
        fdc.ac_strategy, f.header.epf_params, pool,
        (stages && stages[4]) ? &aux : nullptr);
    if (stages && stages[4]) CopyPlaneOut(filtered, stages[4]);
    opsin = std::move(ar);
  } else if (stages && stages[3]) {
    Image3F smoothed;
    if (f.header.gaborish != GaborishStrength::kOff) {
      PIK_RETURN_IF_ERROR(
          ConvolveGaborish(opsin, f.header.gaborish, pool, &smoothed));
      CopyPlaneOut(smoothed, stages[3]);
    } else {
      CopyPlaneOut(opsin, stages[3]);
    }
  }
  if (stages && stages[5]) CopyPlaneOut(opsin, stages[5]);
  // ApplyForwardBilinear is a no-op (kUseBilinearTransforms = false,
  // pik/bilinear_transform.cc:11); the block dictionary adds detected dots.
  {
    Image3F before = CopyImage(opsin);
    f.dictionary.AddTo(&opsin, 1);
    bool changed = false;
    for (int c = 0; c < 3 && !changed; ++c) {
      for (size_t y = 0; y < opsin.ysize() && !changed; ++y) {
        changed = memcmp(before.ConstPlaneRow(c, y), opsin.ConstPlaneRow(c, y),
                         opsin.xsize() * sizeof(float)) != 0;
      }
    }
    g_dictionary_changed = changed;
  }
  if (f.header.gaborish != GaborishStrength::kOff) {
    Image3F g;
    PIK_RETURN_IF_ERROR(ConvolveGaborish(opsin, f.header.gaborish, pool, &g));
    opsin = std::move(g);
  }
  opsin.ShrinkTo(f.xsize, f.ysize);
  if (stages && stages[6]) CopyPlaneOut(opsin, stages[6]);
  OpsinToLinear(&opsin, pool);
  const auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  if (stages && stages[7]) CopyPlaneOut(opsin, stages[7]);
  return true;
}

}  // namespace

extern "C" {

const char* pikref_last_error() { return g_error.c_str(); }

// 1 if the last pikref_run_stages call's block dictionary changed pixels.
int pikref_dictionary_changed() { return g_dictionary_changed ? 1 : 0; }

const char* pikref_flavour() {
#if SIMD_ENABLE == 0
  return "scalar";
#else
  return "avx2";
#endif
}

// Encodes 3 planes (R, G, B; each ysize*xsize floats, linear sRGB on the
// reference's 0..255 scale). ar: -1 default (on), 0 off, 1 on.
// Returns the bitstream in a malloc'd buffer.
int pikref_encode(const float* planes, int xsize, int ysize, float distance,
                  int ar, int gaborish, int fast_mode, int num_threads,
                  uint8_t** out, size_t* out_size) {
  CodecContext context;
  CodecInOut io(&context);
  Image3F img(xsize, ysize);
  for (int c = 0; c < 3; ++c) {
    for (int y = 0; y < ysize; ++y) {
      memcpy(img.PlaneRow(c, y), planes + (size_t(c) * ysize + y) * xsize,
             xsize * sizeof(float));
    }
  }
  io.SetFromImage(std::move(img), context.c_linear_srgb[0]);
  io.SetOriginalBitsPerSample(32);
  CompressParams params;
  params.butteraugli_distance = distance;
  params.fast_mode = fast_mode != 0;
  if (ar == 0) params.adaptive_reconstruction = Override::kOff;
  if (ar == 1) params.adaptive_reconstruction = Override::kOn;
  if (gaborish >= 0) params.gaborish = gaborish;
  PaddedBytes compressed;
  std::unique_ptr<ThreadPool> pool;
  if (num_threads > 0) pool.reset(new ThreadPool(num_threads));
  if (!PixelsToPik(params, &io, &compressed, nullptr, pool.get())) {
    g_error = "PixelsToPik failed";
    return -1;
  }
  *out = static_cast<uint8_t*>(malloc(compressed.size()));
  memcpy(*out, compressed.data(), compressed.size());
  *out_size = compressed.size();
  return 0;
}

void pikref_free(void* p) { free(p); }

// LinearToXyb (pik/opsin_image.cc:34-47), the encoder's opsin transform, on
// n pixels of planar linear sRGB (0..255): planar XYB out.
int pikref_linear_to_xyb(const float* lin, size_t n, float* xyb) {
  for (size_t i = 0; i < n; ++i) {
    LinearToXyb(lin[i], lin[n + i], lin[2 * n + i], &xyb[i], &xyb[n + i],
                &xyb[2 * n + i]);
  }
  return 0;
}

// Full reference decode (PikToPixels, pik/pik.cc:92-131) to linear planes
// (3 * ysize * xsize floats).
int pikref_decode(const uint8_t* data, size_t size, int num_threads,
                  float* out_linear, size_t capacity_floats) {
  CodecContext context;
  CodecInOut io(&context);
  PaddedBytes compressed(size);
  memcpy(compressed.data(), data, size);
  DecompressParams dparams;
  std::unique_ptr<ThreadPool> pool;
  if (num_threads > 0) pool.reset(new ThreadPool(num_threads));
  if (!PikToPixels(dparams, compressed, &io, nullptr, pool.get())) {
    g_error = "PikToPixels failed";
    return -1;
  }
  const Image3F& color = io.color();
  if (3 * color.xsize() * color.ysize() > capacity_floats) {
    g_error = "output too small";
    return -1;
  }
  CopyPlaneOut(color, out_linear);
  return 0;
}

void* pikref_frozen_from_bitstream(const uint8_t* data, size_t size,
                                   int override_ar, int override_gaborish) {
  InitEpf();
  PaddedBytes compressed(size);
  memcpy(compressed.data(), data, size);
  std::unique_ptr<Frozen> f(new Frozen);
  if (!DecodeToFrozen(compressed, override_ar, override_gaborish, f.get())) {
    g_error = "frozen decode failed";
    return nullptr;
  }
  return f.release();
}

void pikref_frozen_free(void* h) { delete static_cast<Frozen*>(h); }

// The reference's PNM writer (EncodeImagePNM, pik/codec_pnm.cc:260-294) on
// linear planes (0..255 scale, as PikToPixels leaves io.color()), written
// in sRGB (to_srgb) or linear light with bits_per_sample 8, 16 or 32. The
// sRGB transfer runs through oracle/ref_shim.cc's colour management (the
// reference's skip-lcms route); the container, casts and rounding are the
// reference's own. Returns 0 and the file's size in *size.
int pikref_encode_pnm(const float* planes, int xsize, int ysize, int bits,
                      int to_srgb, uint8_t* out, size_t capacity,
                      size_t* size) {
  CodecContext context;
  CodecInOut io(&context);
  Image3F img(xsize, ysize);
  for (int c = 0; c < 3; ++c) {
    for (int y = 0; y < ysize; ++y) {
      memcpy(img.PlaneRow(c, y), planes + (size_t(c) * ysize + y) * xsize,
             xsize * sizeof(float));
    }
  }
  io.SetFromImage(std::move(img), context.c_linear_srgb[0]);
  PaddedBytes bytes;
  const ColorEncoding& c_out =
      to_srgb ? context.c_srgb[0] : context.c_linear_srgb[0];
  if (!EncodeImagePNM(&io, c_out, bits, nullptr, &bytes)) {
    g_error = "EncodeImagePNM failed";
    return -1;
  }
  *size = bytes.size();
  if (bytes.size() > capacity) {
    g_error = "output too small";
    return -1;
  }
  memcpy(out, bytes.data(), bytes.size());
  return 0;
}

// The decoder's fixed-sigma override (DecompressParams::epf_sigma > 0,
// OverridePassFlags, pik/pik_frame.cc:112-115): the EPF runs with one sigma
// for every block (Filter, pik/epf_target.cc:1342-1386).
int pikref_frozen_set_fixed_sigma(void* h, int sigma) {
  Frozen* f = static_cast<Frozen*>(h);
  if (!f || sigma <= 0) return -1;
  f->header.epf_params.enable_adaptive = false;
  f->header.epf_params.sigma = uint32_t(sigma);
  return 0;
}

// PikToPixels with DecompressParams::epf_sigma set (0: the bitstream's own
// EPF parameters), to linear planes (3 * ysize * xsize floats).
int pikref_decode_epf_sigma(const uint8_t* data, size_t size, int num_threads,
                            int epf_sigma, float* out_linear,
                            size_t capacity_floats) {
  CodecContext context;
  CodecInOut io(&context);
  PaddedBytes compressed(size);
  memcpy(compressed.data(), data, size);
  DecompressParams dparams;
  dparams.epf_sigma = epf_sigma;
  std::unique_ptr<ThreadPool> pool;
  if (num_threads > 0) pool.reset(new ThreadPool(num_threads));
  if (!PikToPixels(dparams, compressed, &io, nullptr, pool.get())) {
    g_error = "PikToPixels failed";
    return -1;
  }
  const Image3F& color = io.color();
  if (3 * color.xsize() * color.ysize() > capacity_floats) {
    g_error = "output too small";
    return -1;
  }
  CopyPlaneOut(color, out_linear);
  return 0;
}

// Scalars: [0] xsize [1] ysize [2] Bx [3] By [4] flags [5] gaborish
// [6] predict_lf [7] predict_hf [8] have_ar [9] epf_enable_adaptive
// [10] epf_sigma [11] epf_use_sharpened [12] global_scale [13] quant_dc
// [14] ytox_dc [15] ytob_dc [16] dequant_table_size [17] num_tables
// [18] dictionary empty (1) [19] Tx [20] Ty
// floats: [0] inv_global_scale [1] inv_quant_dc [2] global_scale_float
int pikref_frozen_scalars(void* h, int64_t* ints, float* floats) {
  const Frozen& f = *static_cast<Frozen*>(h);
  const FrameHeader& hd = f.header;
  ints[0] = f.xsize;
  ints[1] = f.ysize;
  ints[2] = f.xsize_blocks;
  ints[3] = f.ysize_blocks;
  ints[4] = hd.flags;
  ints[5] = static_cast<int>(hd.gaborish);
  ints[6] = hd.predict_lf;
  ints[7] = hd.predict_hf;
  ints[8] = hd.have_adaptive_reconstruction;
  ints[9] = hd.epf_params.enable_adaptive;
  ints[10] = hd.epf_params.sigma;
  ints[11] = hd.epf_params.use_sharpened;
  ints[12] = int(65536.0f / f.quantizer->InvGlobalScale() + 0.5f);
  ints[13] = f.quantizer->QuantDC();
  ints[14] = f.cmap.ytox_dc;
  ints[15] = f.cmap.ytob_dc;
  ints[16] = f.fdc->matrices.Size();
  ints[17] = kNumPredefinedTables;
  ints[18] = 1;
  ints[19] = f.cmap.ytox_map.xsize();
  ints[20] = f.cmap.ytox_map.ysize();
  floats[0] = f.quantizer->InvGlobalScale();
  floats[1] = f.quantizer->inv_quant_dc();
  floats[2] = f.quantizer->Scale();
  return 0;
}

// Copies a named array out (plane-major, densely packed).
int pikref_frozen_copy(void* h, const char* name, void* dst, size_t nbytes) {
  const Frozen& f = *static_cast<Frozen*>(h);
  const FrameDecCache& fdc = *f.fdc;
  uint8_t* out = static_cast<uint8_t*>(dst);
  auto copy_img = [&](const auto& img, size_t elem) -> int {
    const size_t row = img.xsize() * elem;
    if (row * img.ysize() > nbytes) return -1;
    for (size_t y = 0; y < img.ysize(); ++y) {
      memcpy(out + y * row, img.ConstRow(y), row);
    }
    return 0;
  };
  auto copy_img3 = [&](const auto& img, size_t elem) -> int {
    const size_t row = img.xsize() * elem;
    if (3 * row * img.ysize() > nbytes) return -1;
    for (int c = 0; c < 3; ++c) {
      for (size_t y = 0; y < img.ysize(); ++y) {
        memcpy(out + (c * img.ysize() + y) * row, img.ConstPlaneRow(c, y),
               row);
      }
    }
    return 0;
  };
  const std::string n(name);
  if (n == "ac_strategy") return copy_img(fdc.ac_strategy.ConstRaw(), 1);
  if (n == "raw_quant_field") return copy_img(fdc.raw_quant_field, 4);
  if (n == "ar_sigma_lut_ids") return copy_img(fdc.ar_sigma_lut_ids, 1);
  if (n == "dequant_control_field") {
    return copy_img(fdc.dequant_control_field, 1);
  }
  if (n == "ytox_map") return copy_img(f.cmap.ytox_map, 4);
  if (n == "ytob_map") return copy_img(f.cmap.ytob_map, 4);
  if (n == "quantized_dc") return copy_img3(f.quantized_dc, 2);
  if (n == "quantized_ac") return copy_img3(f.quantized_ac, 2);
  if (n == "dc_smoothed") return copy_img3(f.dc_smoothed, 4);
  if (n == "dequant_map") {
    if (nbytes < sizeof(fdc.dequant_map)) return -1;
    memcpy(out, fdc.dequant_map, sizeof(fdc.dequant_map));
    return 0;
  }
  if (n == "dequant_table") {
    const size_t sz = fdc.matrices.Size() * sizeof(float);
    if (sz > nbytes) return -1;
    if (fdc.matrices.MatrixOffset(0, kQuantKindDCT8, 0) != 0) return -2;
    memcpy(out, fdc.matrices.Matrix(0, kQuantKindDCT8, 0), sz);
    return 0;
  }
  if (n == "dequant_offsets") {
    const size_t cnt = kNumPredefinedTables * kNumQuantKinds * 3;
    if (cnt * 4 > nbytes) return -1;
    uint32_t* o = reinterpret_cast<uint32_t*>(out);
    for (size_t t = 0; t < kNumPredefinedTables; ++t) {
      for (size_t k = 0; k < kNumQuantKinds; ++k) {
        for (int c = 0; c < 3; ++c) {
          o[(t * kNumQuantKinds + k) * 3 + c] =
              fdc.matrices.MatrixOffset(t, k, c);
        }
      }
    }
    return 0;
  }
  g_error = "unknown array " + n;
  return -3;
}

// Runs the reference reconstruction on a frozen frame. `stages` has 8
// (nullable) output pointers, see RunStages.
int pikref_run_stages(void* h, int num_threads, float* const* stages,
                      double* seconds) {
  const Frozen& f = *static_cast<Frozen*>(h);
  InitEpf();
  std::unique_ptr<ThreadPool> pool;
  if (num_threads > 0) pool.reset(new ThreadPool(num_threads));
  if (!RunStages(f, pool.get(), stages, seconds)) {
    g_error = "reconstruction failed";
    return -1;
  }
  return 0;
}

// Replaces the frozen frame's integer inputs (for synthetic workloads that
// reuse a decoded frame's side information layout). Sizes must match.
int pikref_frozen_set_ac(void* h, const int16_t* planes, size_t nelems) {
  Frozen& f = *static_cast<Frozen*>(h);
  const size_t row = f.quantized_ac.xsize();
  if (nelems != 3 * row * f.quantized_ac.ysize()) return -1;
  for (int c = 0; c < 3; ++c) {
    for (size_t y = 0; y < f.quantized_ac.ysize(); ++y) {
      memcpy(f.quantized_ac.PlaneRow(c, y),
             planes + (c * f.quantized_ac.ysize() + y) * row,
             row * sizeof(int16_t));
    }
  }
  return 0;
}

// Encoder route of pik/compressed_image_test.cc:31-95 for an all-DCT8
// frame with a uniform quant field: OpsinDynamicsImage + GaborishInverse,
// InitializeFrameEncCache / InitializeEncCache / ComputeCoefficients with an
// all-DCT AcStrategyImage. Returns a frozen frame holding the encoder's
// integers and the decoder-side quantizer (Quantizer::Decode of its encoded
// bytes), with EPF off; `gaborish` is the GaborishStrength in the header.
void* pikref_frozen_encode_dct8(const float* planes, int xsize, int ysize,
                                float quant, int gaborish) {
  InitEpf();
  CodecContext context;
  CodecInOut io(&context);
  Image3F img(xsize, ysize);
  for (int c = 0; c < 3; ++c) {
    for (int y = 0; y < ysize; ++y) {
      memcpy(img.PlaneRow(c, y), planes + (size_t(c) * ysize + y) * xsize,
             xsize * sizeof(float));
    }
  }
  io.SetFromImage(std::move(img), context.c_linear_srgb[0]);
  Image3F opsin =
      PadImageToMultiple(OpsinDynamicsImage(&io, Rect(io.color())), kBlockDim);
  FrameHeader header;
  header.gaborish = GaborishStrength(gaborish);
  header.have_adaptive_reconstruction = false;
  if (header.gaborish != GaborishStrength::kOff) {
    // Same pre-sharpening as PixelsToPikPass (pik/pik_frame.cc:529-532).
    opsin = GaborishInverse(opsin, 0.92718927264540152);
  }
  const size_t xb = opsin.xsize() / kBlockDim, yb = opsin.ysize() / kBlockDim;
  std::unique_ptr<Frozen> f(new Frozen);
  f->xsize = xsize;
  f->ysize = ysize;
  f->xsize_blocks = xb;
  f->ysize_blocks = yb;
  f->header = header;
  f->cmap = ColorCorrelationMap(opsin.xsize(), opsin.ysize());
  f->fdc.reset(new FrameDecCache);
  FrameDecCache& fdc = *f->fdc;
  DequantMatrices dequant(/*need_inv_matrices=*/true);
  Quantizer enc_q(&dequant, xb, yb);
  enc_q.SetQuant(quant);
  AcStrategyImage ac_strategy(xb, yb);
  FrameEncCache fec;
  fec.dequant_control_field =
      ImageB(DivCeil(opsin.xsize(), kTileDim), DivCeil(opsin.ysize(), kTileDim));
  ZeroFillImage(&fec.dequant_control_field);
  BlockDictionary dictionary;
  InitializeFrameEncCache(header, opsin, ac_strategy, enc_q, f->cmap,
                          dictionary, nullptr, &fec, nullptr);
  EncCache ec;
  GroupHeader gh;
  InitializeEncCache(header, gh, fec, Rect(opsin), &ec);
  ec.ac_strategy = ac_strategy.Copy();
  ComputeCoefficients(enc_q, f->cmap, Rect(f->cmap.ytob_map), nullptr, fec,
                      &ec);
  // Decoder-side state.
  const std::string qbytes = enc_q.Encode(nullptr);
  PaddedBytes qb(qbytes.size());
  memcpy(qb.data(), qbytes.data(), qbytes.size());
  BitReader br(qb.data(), qb.size());
  f->quantizer.reset(new Quantizer(&fdc.matrices, 0, 0));
  if (!f->quantizer->Decode(&br)) {
    g_error = "quantizer decode failed";
    return nullptr;
  }
  fdc.ac_strategy = ac_strategy.Copy();
  fdc.raw_quant_field = CopyImage(ec.quant_field);
  fdc.ar_sigma_lut_ids = ImageB(xb, yb);
  ZeroFillImage(&fdc.ar_sigma_lut_ids);
  fdc.dequant_control_field = CopyImage(fec.dequant_control_field);
  f->quantized_dc = CopyImage(fec.dc);
  f->quantized_ac = CopyImage(ec.ac);
  // DequantDC (pik/compressed_dc.cc:181-231; not exported by the
  // reference, restated here) + AdaptiveDCReconstruction.
  float mul_dc[3];
  for (int c = 0; c < 3; ++c) {
    mul_dc[c] = f->quantizer->DequantMatrix(0, kQuantKindDCT8, c)[0] *
                f->quantizer->inv_quant_dc();
  }
  const float ytox_dc = ColorCorrelationMap::YtoX(1.0f, f->cmap.ytox_dc);
  const float ytob_dc = ColorCorrelationMap::YtoB(1.0f, f->cmap.ytob_dc);
  Image3F dc(xb, yb);
  for (size_t y = 0; y < yb; ++y) {
    for (size_t x = 0; x < xb; ++x) {
      const float vy = f->quantized_dc.ConstPlaneRow(1, y)[x] * mul_dc[1];
      dc.PlaneRow(1, y)[x] = vy;
      const float dx = f->quantized_dc.ConstPlaneRow(0, y)[x] * mul_dc[0];
      dc.PlaneRow(0, y)[x] = ytox_dc * vy + dx;
      const float db = f->quantized_dc.ConstPlaneRow(2, y)[x] * mul_dc[2];
      dc.PlaneRow(2, y)[x] = ytob_dc * vy + db;
    }
  }
  AdaptiveDCReconstruction(dc, *f->quantizer, nullptr);
  f->dc_smoothed = std::move(dc);
  return f.release();
}

// ---- Probes of single reference functions (for pinning the restatement).

// AcStrategy::TransformToPixels / TransformFromPixels
// (pik/ac_strategy.cc:531-848) for one block of `type`. Coefficients use the
// frame layout with row stride `cstride` floats; pixels row stride `pstride`.
int pikref_transform(int type, int inverse, const float* in, size_t in_stride,
                     float* out, size_t out_stride) {
  if (type < 0 || type > 8) return -1;
  AcStrategy acs(static_cast<AcStrategy::Type>(type), 0);
  if (inverse) {
    acs.TransformToPixels(in, in_stride, out, out_stride);
  } else {
    acs.TransformFromPixels(in, in_stride, out, out_stride);
  }
  return 0;
}

// LLF / LF helpers (pik/ac_strategy.cc:850-1056). which: 0
// LowestFrequenciesFromDC 1 DC2x2FromLowestFrequencies 2
// DC2x2FromLowFrequencies 3 LowFrequenciesFromDC2x2.
int pikref_lf_helper(int type, int which, const float* in, size_t in_stride,
                     float* out, size_t out_stride) {
  if (type < 0 || type > 8) return -1;
  AcStrategy acs(static_cast<AcStrategy::Type>(type), 0);
  switch (which) {
    case 0:
      acs.LowestFrequenciesFromDC(in, in_stride, out, out_stride);
      break;
    case 1:
      acs.DC2x2FromLowestFrequencies(in, in_stride, out, out_stride);
      break;
    case 2:
      acs.DC2x2FromLowFrequencies(in, in_stride, out, out_stride);
      break;
    case 3:
      acs.LowFrequenciesFromDC2x2(in, in_stride, out, out_stride);
      break;
    default:
      return -1;
  }
  return 0;
}

// EPF WeightFast value for (sigma, sad) (pik/epf_target.cc:1405-1412).
float pikref_epf_weight(int sigma, int sad) {
  InitEpf();
  return Dispatch(TargetBitfield().Best(), EdgePreservingFilterTest(), sigma,
                  sad);
}

// The 3x3 inverse opsin absorbance matrix (pik/opsin_params.cc:22-25).
void pikref_opsin_inverse_matrix(float* out9) {
  memcpy(out9, GetOpsinAbsorbanceInverseMatrix(), 9 * sizeof(float));
}

// ConvolveGaborish on a planar 3-channel image (pik/gaborish.cc:137-159).
int pikref_gaborish(int strength, const float* in, int xsize, int ysize,
                    float* out) {
  Image3F img(xsize, ysize);
  for (int c = 0; c < 3; ++c) {
    for (int y = 0; y < ysize; ++y) {
      memcpy(img.PlaneRow(c, y), in + (size_t(c) * ysize + y) * xsize,
             xsize * sizeof(float));
    }
  }
  Image3F res;
  if (!ConvolveGaborish(img, GaborishStrength(strength), nullptr, &res)) {
    return -1;
  }
  CopyPlaneOut(res, out);
  return 0;
}

}  // extern "C"
