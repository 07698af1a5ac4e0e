/*
 * pikgpu: B200 (sm_100a) implementation of the google/pik decoder's
 * reconstruction path, exposed as a plain C ABI.
 *
 * The path is the one the reference runs after entropy decoding:
 *   dequantisation of AC/DC integers (Quantizer, quant field, quant_weights
 *   per AcStrategy) + chroma-from-luma -> DC smoothing -> LF/HF prediction ->
 *   variable-size IDCT (2x2 .. 32x32, IDENTITY, LINES) -> gaborish ->
 *   edge-preserving filter (EPF) + DCT-domain clamp -> gaborish ->
 *   XYB -> linear RGB (and optionally 8-bit sRGB).
 *
 * Reference interfaces this ABI replaces (reference paths are relative to the
 * google/pik checkout):
 *   Dequant<first>::DoAC            pik/compressed_image.cc:586-707
 *   ReconOpsinImage                 pik/compressed_image.h:93-98
 *   FinalizeFrameDecoding           pik/compressed_image.h:104-110
 *   DequantDC + AdaptiveDCReconstruction
 *                                   pik/compressed_dc.cc:181-231,
 *                                   pik/adaptive_reconstruction.cc:300-332
 * Their callers are PikGroupToPixels (pik/pik_frame.cc:925-928) and
 * PikPassToPixels (pik/pik_frame.cc:1149-1152).
 *
 * Conventions
 *  - Every entry point returns an int status: 0 = OK, negative = error
 *    (PIKGPU_ERR_*). Nothing aborts; the reason is in pikgpu_last_error().
 *  - Images are planar. "blocks" are 8x8 pixel cells; Bx = ceil(xsize/8),
 *    By = ceil(ysize/8). "colour tiles" are 64x64 pixels:
 *    Tx = ceil(xsize/64), Ty = ceil(ysize/64).
 *  - Host buffers stay owned by the caller. A context owns its device memory
 *    and one CUDA stream; contexts are independent.
 */
#ifndef PIKGPU_H_
#define PIKGPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PIKGPU_OK 0
#define PIKGPU_ERR_INVALID_ARG (-1) /* bad pointer, size or field value */
#define PIKGPU_ERR_UNSUPPORTED (-2) /* feature the reference path has but
                                       this build rejects (see below) */
#define PIKGPU_ERR_CUDA (-3)        /* a CUDA call failed */
#define PIKGPU_ERR_STATE (-4)       /* call out of order */
#define PIKGPU_ERR_NO_MEMORY (-5)   /* device allocation failed */

/* GaborishStrength (pik/pik_params.h:39-49). */
#define PIKGPU_GABORISH_OFF 0
#define PIKGPU_GABORISH_500 1
#define PIKGPU_GABORISH_750 2
#define PIKGPU_GABORISH_875 3
#define PIKGPU_GABORISH_1000 4

/* Number of QuantKind values (pik/quant_weights.h:25-34). */
#define PIKGPU_NUM_QUANT_KINDS 7
/* kMaxQuantControlFieldValue (pik/quant_weights.h:268). */
#define PIKGPU_MAX_QUANT_CONTROL_FIELD 16

/*
 * Frame-level side information. Mirrors what PikPassToPixels holds after
 * decoding the frame header and DC groups (pik/pik_frame.cc:1028-1065):
 * FrameHeader subset, Quantizer scalars, DequantMatrices, dequant control
 * field + map, ColorCorrelationMap, AcStrategyImage, raw quant field,
 * EPF LUT ids and the quantized DC.
 */
typedef struct pikgpu_frame_params {
  uint32_t xsize, ysize; /* pixels */

  /* FrameHeader (pik/headers.h:202-232). */
  uint32_t flags;    /* FrameHeader::flags; any set bit is UNSUPPORTED */
  uint32_t gaborish; /* PIKGPU_GABORISH_* */
  uint32_t predict_lf, predict_hf;
  uint32_t have_adaptive_reconstruction;
  /* EpfParams (pik/epf.h:19-40); used iff have_adaptive_reconstruction. */
  /* 0: the fixed-sigma EPF (Filter, pik/epf_target.cc:1342-1386) with
   * epf_sigma for every block (0: a copy; else within [16, 672]). */
  uint32_t epf_enable_adaptive;
  uint32_t epf_sigma;
  uint32_t epf_use_sharpened;

  /* Quantizer (pik/quantizer.h:111-389; Decode pik/quantizer.cc:63-71). */
  int32_t global_scale; /* [1, 32768] */
  int32_t quant_dc;     /* [1, 256] */

  /* DequantMatrices (pik/quant_weights.h:202-266): the flat table and
   * offsets[(table * 7 + kind) * 3 + c] into it. */
  const float* dequant_table;
  uint32_t dequant_table_size; /* floats */
  const uint32_t* dequant_offsets;
  uint32_t num_dequant_tables;
  const uint8_t* dequant_control_field; /* Tx * Ty */
  const uint8_t* dequant_map;           /* 16 * 256: [cf][qf - 1] -> table */

  /* ColorCorrelationMap (pik/color_correlation.h:44-89). */
  const int32_t* ytox_map; /* Tx * Ty */
  const int32_t* ytob_map; /* Tx * Ty */
  int32_t ytox_dc, ytob_dc;

  /* Per-block fields, Bx * By each. */
  const uint8_t* ac_strategy;     /* raw byte: type << 4 | sub-block index */
  const int32_t* raw_quant_field; /* [1, 256] */
  const uint8_t* ar_sigma_lut_ids;

  /* Quantized DC after DC-prediction expansion (ExpandDC), 3 planes of
   * Bx * By int16, plane-major (X, Y, B). */
  const int16_t* quantized_dc;
} pikgpu_frame_params;

typedef struct pikgpu_ctx pikgpu_ctx;

/* Creates a context on CUDA device `device`. */
int pikgpu_ctx_create(int device, pikgpu_ctx** out);
int pikgpu_ctx_destroy(pikgpu_ctx* ctx);
/* Message of the last failed call on this context (never NULL). */
const char* pikgpu_last_error(const pikgpu_ctx* ctx);

/* Starts a frame: validates `params` (see "Errors"), sizes device buffers
 * and uploads the side information. Replaces the frame-level state that
 * PikPassToPixels builds before its group loop (pik/pik_frame.cc:1040-1065).
 * Errors: INVALID_ARG for strategy > 8 (pik/ac_strategy.h:95-97), sub-block
 * indices inconsistent with the strategy, qf outside [1,256]
 * (pik/quantizer.h:125-128), LUT id > 1, dequant_map entries >= the number
 * of tables, offsets past the table, a fixed sigma outside {0} U [16, 672];
 * UNSUPPORTED for any FrameHeader flag (noise, gradient map, grayscale,
 * ...) and for multi-block transforms not aligned to their size. */
int pikgpu_frame_begin(pikgpu_ctx* ctx, const pikgpu_frame_params* params);

/* Supplies the whole frame's quantized AC after entropy decoding and
 * coefficient un-scattering (pik/compressed_image.cc:780-801): per plane,
 * By rows of Bx * 64 int16 in the GroupDecCache::ac layout
 * (pik/compressed_image_fwd.h:206). `stride` is in elements. Host memory. */
int pikgpu_frame_set_ac(pikgpu_ctx* ctx, const int16_t* const planes[3],
                        size_t stride);

/* Same for one 512x512 group (group_index = gy * ceil(xsize/512) + gx),
 * i.e. what DecodeFromBitstream decodes for that group
 * (pik/compressed_image.cc:720-813), as pik's group threads do
 * (pik/pik_frame.cc:1108-1135). Groups may be supplied from different host
 * threads concurrently: each call copies into its own region of the
 * context's device AC buffer, on the context's stream, from the calling
 * thread (with the context's device made current there). No other call on
 * the context may run while such uploads are in progress. */
int pikgpu_frame_set_group_ac(pikgpu_ctx* ctx, uint32_t group_index,
                              const int16_t* const planes[3], size_t stride);

/* Device-resident variant of pikgpu_frame_set_ac: `planes` are device
 * pointers on the context's device; no host copy is made. Planes in the
 * context's own layout -- stride Bx * 64, the three planes consecutive
 * (planes[c] = planes[0] + c * By * Bx * 64), planes[0] 16-byte aligned --
 * are read in place by every later pikgpu_reconstruct of this frame (no
 * device copy either): they must stay valid until the last reconstruction
 * that uses them has completed, and changing their contents between calls
 * changes the next result. Other layouts are copied into the context. */
int pikgpu_frame_set_ac_device(pikgpu_ctx* ctx, const int16_t* const planes[3],
                               size_t stride);

/* Runs the whole reconstruction: the per-group Dequant::DoAC +
 * ReconOpsinImage work and then FinalizeFrameDecoding
 * (pik/compressed_image.cc:1144-1181). Outputs (either may be NULL):
 *  out_linear: 3 planes of ysize rows x xsize floats, linear RGB on the
 *     reference's 0..255 scale, row stride `linear_stride` floats.
 *  out_srgb8: interleaved RGB bytes, row stride `srgb8_stride` bytes,
 *     sRGB-encoded (TF_SRGB, pik/color_management.cc:323-345) and rounded
 *     like ExternalImage::CopyTo (pik/external_image.cc:1205).
 * If `outputs_on_device` is nonzero both pointers are device pointers and no
 * host copy is made; otherwise they are host pointers. Blocks until done. */
int pikgpu_reconstruct(pikgpu_ctx* ctx, float* const out_linear[3],
                       size_t linear_stride, uint8_t* out_srgb8,
                       size_t srgb8_stride, int outputs_on_device);

/* Non-blocking form of pikgpu_reconstruct, for streaming decoders: enqueues
 * the reconstruction and the copies into the outputs on the context's
 * stream and returns. The outputs are complete, and errors of the GPU work
 * are reported, when pikgpu_wait returns. Host inputs given to
 * pikgpu_frame_set_ac and host outputs should be page-locked (pinned) for
 * the copies to run asynchronously, and must stay valid and unchanged until
 * pikgpu_wait. Until then every other call on the context fails with
 * PIKGPU_ERR_STATE: to overlap one frame's copies with another frame's
 * computation, alternate two or more contexts (each has its own stream).
 * No counterpart in the reference, which reconstructs synchronously. */
int pikgpu_reconstruct_async(pikgpu_ctx* ctx, float* const out_linear[3],
                             size_t linear_stride, uint8_t* out_srgb8,
                             size_t srgb8_stride, int outputs_on_device);
/* Waits for the context's pikgpu_reconstruct_async (returns at once if
 * there is none) and returns its status. */
int pikgpu_wait(pikgpu_ctx* ctx);

/* Output-format step of dpik's writer (WriteOutput, pik/dpik.cc:196-223;
 * EncodeImagePNM and EncodeHeader, pik/codec_pnm.cc:179-196,260-294;
 * ExternalImage's casts, pik/external_image.cc), run on the device for the
 * frame of the last pikgpu_reconstruct that wrote linear planes: the image
 * of a PPM file ("P6", 8 or 16 bits per sample, big-endian samples) or a
 * PFM file ("PF", 32-bit little-endian floats, scale -1: sample values
 * x 255), header included, rows top to bottom, RGB interleaved.
 *  transfer: PIKGPU_TF_SRGB encodes with TF_SRGB (what dpik writes for an
 *            sRGB original), PIKGPU_TF_LINEAR keeps linear light;
 *  8 / 16 bits clamp to [0, 1] and round like ExternalImage::CopyTo.
 * `out`: `capacity` bytes of host memory (device memory if out_on_device).
 * The file's size is written to *size; with out NULL only the size is
 * computed. Blocks until the bytes are written. */
#define PIKGPU_TF_LINEAR 0
#define PIKGPU_TF_SRGB 1
int pikgpu_encode_pnm(pikgpu_ctx* ctx, int bits_per_sample, int transfer,
                      uint8_t* out, size_t capacity, size_t* size,
                      int out_on_device);

/* Intermediate planes for stage-by-stage parity checks, valid after
 * pikgpu_reconstruct. Each is 3 planes in host memory. */
#define PIKGPU_STAGE_DC 0          /* Bx x By: DC after AdaptiveDCRecon. */
#define PIKGPU_STAGE_IDCT 1        /* padded frame: ReconOpsinImage output */
#define PIKGPU_STAGE_SMOOTHED 2    /* gaborish #1 (EPF guide source) */
#define PIKGPU_STAGE_EPF 3         /* EPF output before the DCT clamp */
#define PIKGPU_STAGE_AR 4          /* after AdaptiveReconstruction clamp */
#define PIKGPU_STAGE_PRE_OPSIN 5   /* after gaborish #2, before opsin */
#define PIKGPU_STAGE_DEQUANT_AC 6  /* Bx*64 x By: DoAC output */
int pikgpu_get_stage(pikgpu_ctx* ctx, int stage, float* const planes[3],
                     size_t stride, size_t xsize, size_t ysize);

/* Average device time in milliseconds of each kernel of the last
 * pikgpu_reconstruct call, written to `ms` (up to `n` entries); returns the
 * number of kernels or an error. Names via pikgpu_kernel_name. */
int pikgpu_last_kernel_times(pikgpu_ctx* ctx, float* ms, int n);
const char* pikgpu_kernel_name(int index);
/* Number of kernels the last pikgpu_reconstruct launched. */
int pikgpu_last_launch_count(const pikgpu_ctx* ctx);

/* Checks `params` exactly as pikgpu_frame_begin does, without a device.
 * Writes the reason for a failure into `msg` (may be NULL). */
int pikgpu_validate(const pikgpu_frame_params* params, char* msg,
                    size_t msg_size);

/* Options (set before pikgpu_frame_begin):
 *  KEEP_STAGES: keep the dequantised AC, EPF and pre-opsin planes for
 *               pikgpu_get_stage (costs extra device memory and copies);
 *  PROFILE:     time each kernel group with CUDA events
 *               (pikgpu_last_kernel_times); every kernel then runs on one
 *               stream after the one before it (no concurrent branches, no
 *               programmatic dependent launches, no graph replay);
 *  FORM:        PIKGPU_FORM_FP32 (default): every stage in FP32 on the CUDA
 *               cores in the reference's operation order;
 *               PIKGPU_FORM_SPLIT_BF16: the 16x16 and 32x32 transforms
 *               (the IDCT with HF prediction and the clamp's DCT pair) on
 *               the tensor cores as split-BF16 GEMMs with FP32
 *               accumulation; 16-point operands split in two BF16 terms
 *               (hi + lo, three products; about 16 significant bits) --
 *               in three for the IDCT of frames without HF prediction --
 *               and 32-point operands in three (hi + mid + lo, six
 *               products);
 *               PIKGPU_FORM_SPLIT_BF16X3: three terms for both sizes
 *               (FP32-level error).
 *               The tensor-core forms are not bit-identical to the FP32
 *               form;
 *  GRAPHS:      1 (default): when pikgpu_reconstruct is called again with
 *               the launch state of the previous call (frame geometry,
 *               header scalars, blocks per transform class, options,
 *               device buffers, outputs and stream all unchanged -- the
 *               coefficients and side information may differ), the launch
 *               sequence is captured once into a CUDA graph and replayed
 *               as one launch; 0: every call launches its 17 or so kernels.
 *               Either way some kernels are programmatic dependent launches
 *               of the kernel before them on their stream: they may start
 *               while it finishes, ordered by griddepcontrol in the kernels. */
#define PIKGPU_OPT_KEEP_STAGES 1
#define PIKGPU_OPT_PROFILE 2
#define PIKGPU_OPT_FORM 3
#define PIKGPU_OPT_GRAPHS 4
/* TC_WAIT_POLLS: the device's bounded waits on an mbarrier -- the
 *               tensor-core kernels' wait for each batch of MMAs, and the
 *               EPF's wait for each tile copied by the Tensor Memory
 *               Accelerator. If a first wait runs out of polls, the kernel
 *               drains what is in flight (a second bounded wait), stops,
 *               and pikgpu_reconstruct fails with PIKGPU_ERR_CUDA ("MMA
 *               completion wait timed out" / "EPF: TMA tile copy wait
 *               timed out"); the context stays usable. The value is the
 *               first wait's number of polls: -1 (default) 4194304; 0
 *               makes every first wait run out at once, which exercises
 *               that error path. No counterpart in the reference. */
#define PIKGPU_OPT_TC_WAIT_POLLS 5
#define PIKGPU_FORM_FP32 0
#define PIKGPU_FORM_SPLIT_BF16 1
#define PIKGPU_FORM_SPLIT_BF16X3 2
int pikgpu_set_option(pikgpu_ctx* ctx, int option, int value);
/* Graphs captured by this context so far (PIKGPU_OPT_GRAPHS), and whether
 * the last pikgpu_reconstruct ran as a graph replay (either may be NULL). */
int pikgpu_graph_stats(const pikgpu_ctx* ctx, int* captures,
                       int* last_replayed);

/* Verification hooks for the EPF's discrete decisions, which make two
 * implementations comparable on arithmetic alone: the u8 guide (3 planes of
 * (8By + 12) x (8Bx + 12), the padded frame with the filter's 6-pixel
 * mirrored border) and the per-block sigma (By x Bx int32), as computed by
 * MakeGuide / SigmaFromQuant (pik/epf_target.cc:1009-1111). `set` replaces
 * the computed values for the current frame (NULL restores computing them);
 * `get` exports the values of the last pikgpu_reconstruct. Host memory. */
int pikgpu_set_epf_decisions(pikgpu_ctx* ctx, const uint8_t* guide,
                             const int32_t* sigma);
int pikgpu_get_epf_decisions(pikgpu_ctx* ctx, uint8_t* guide, int32_t* sigma);

/* Sets the CUDA stream (a cudaStream_t passed as void*) the context launches
 * on; NULL restores the context's own stream. */
int pikgpu_set_stream(pikgpu_ctx* ctx, void* stream);

/* Batched reconstruction of many frames of uneven sizes. No counterpart in
 * the reference, which reconstructs one frame per FinalizeFrameDecoding
 * call. A batch owns one context per frame: fill each with
 * pikgpu_frame_begin / pikgpu_frame_set_ac(_device) / pikgpu_set_option on
 * the context that pikgpu_batch_frame returns. pikgpu_batch_reconstruct
 * then runs all frames at once: on its first call (and after any frame's
 * frame_begin, set_option or set_epf_decisions, or a change of outputs) it
 * captures every frame's launch sequence into one CUDA graph, one branch
 * per frame, and it replays that graph. Outputs are device pointers: frame
 * i writes 3 consecutive planes of linear_strides[i] x ysize floats at
 * out_linear[i]. `stream` (a cudaStream_t, NULL = the batch's own stream)
 * is where the graph runs; the call blocks until it is done. Profiling
 * (PIKGPU_OPT_PROFILE) is UNSUPPORTED in a batch. */
typedef struct pikgpu_batch pikgpu_batch;
int pikgpu_batch_create(int device, int num_frames, pikgpu_batch** out);
int pikgpu_batch_destroy(pikgpu_batch* batch);
pikgpu_ctx* pikgpu_batch_frame(pikgpu_batch* batch, int index);
int pikgpu_batch_reconstruct(pikgpu_batch* batch, float* const* out_linear,
                             const size_t* linear_strides, void* stream);
const char* pikgpu_batch_last_error(const pikgpu_batch* batch);
/* Kernels launched per replay, and graphs captured so far. */
int pikgpu_batch_launch_count(const pikgpu_batch* batch);
int pikgpu_batch_capture_count(const pikgpu_batch* batch);
/* Autotuner of the batch's launch shape: captures and times (median of 3
 * replays) every combination of the number of concurrent graph branches
 * (1, 2, 4, ... up to one per frame; frame i runs in branch i % chains) and,
 * when a tensor-core form is in use, of the persistent 16x16 transform
 * kernels' CTAs per SM (1, 2, 4), and keeps the fastest for later calls.
 * The chosen values are written to `chains` and `tc_ctas_per_sm` (either
 * may be NULL). Same outputs as pikgpu_batch_reconstruct. */
int pikgpu_batch_autotune(pikgpu_batch* batch, float* const* out_linear,
                          const size_t* linear_strides, void* stream,
                          int* chains, int* tc_ctas_per_sm);

/* Allocation-free DC reconstruction. No counterpart in the reference: its
 * DequantDC + AdaptiveDCReconstruction (pik/compressed_dc.cc:181-231,
 * pik/adaptive_reconstruction.cc:300-332) allocate their images as they go.
 * This call gives the result of the DC stage of pikgpu_reconstruct
 * (PIKGPU_STAGE_DC) in the plain FP32 form, bit for bit (the tensor-core
 * forms' DC EPF uses fused multiply-adds: within 2e-6 of it), for callers
 * that must not allocate device memory when they reconstruct: it calls no
 * allocating routine and keeps its intermediates in a static device array
 * of about 3 MiB per device.
 *  quantized_dc: device memory of the current device (or managed), 3
 *                planes (X, Y, B) of ysize_blocks x xsize_blocks int16,
 *                contiguous;
 *  dc:           same kind of memory, 3 planes of ysize_blocks x
 *                xsize_blocks floats, contiguous (output; must not overlap
 *                quantized_dc);
 *  dc_dequant:   host, DequantMatrix(0, DCT, c)[0] for c = 0..2;
 *  global_scale, quant_dc, ytox_dc, ytob_dc: as in pikgpu_frame_params.
 * Limit: xsize_blocks, ysize_blocks <= 512 (images up to 4096 x 4096);
 * larger sizes fail with PIKGPU_ERR_INVALID_ARG. Runs on the current device,
 * asynchronously on `stream` (a cudaStream_t; NULL = default stream). The
 * first call on a device does a one-time set-up (table upload, scratch
 * address lookup) and should come before any stream capture on it. All
 * calls on a device share the scratch: calls that overlap in time on one
 * device race and must be ordered on one stream or serialised. Writes the
 * reason for a failure into `msg` (may be NULL). */
int pikgpu_dc_reconstruct_noalloc(const int16_t* quantized_dc,
                                  uint32_t xsize_blocks, uint32_t ysize_blocks,
                                  int32_t global_scale, int32_t quant_dc,
                                  const float dc_dequant[3], int32_t ytox_dc,
                                  int32_t ytob_dc, float* dc, void* stream,
                                  char* msg, size_t msg_size);

/* Adjoint of the reconstruction. No counterpart in the reference (a
 * decoder). The variables are the dequantised AC coefficients -- the output
 * of Dequant::DoAC (pik/compressed_image.cc:586-707), 3 planes of
 * ysize_blocks x (64 xsize_blocks) floats in the frame layout of
 * pikgpu_frame_set_ac -- and the per-cell quant field taken as a real
 * number (ysize_blocks x xsize_blocks). The loss is
 *   L = sum over the xsize x ysize pixels and X, Y, B of
 *       (pre_opsin - target)^2,
 * pre_opsin being the frame after gaborish #2 and before OpsinToLinear
 * (PIKGPU_STAGE_PRE_OPSIN). The EPF's discrete decisions (u8 guide,
 * per-block sigma) are held at their values in the forward pass, which this
 * call runs first in the context's form.
 *  target:  3 planes of ysize x xsize floats (XYB), contiguous;
 *  loss:    1 double (may be NULL);
 *  grad_ac: 3 planes of ysize_blocks x 64 xsize_blocks floats (may be NULL;
 *           LLF entries, overwritten from DC, get 0);
 *  grad_qf: ysize_blocks x xsize_blocks floats (may be NULL).
 * All four in device memory if buffers_on_device, else host memory. */
int pikgpu_adjoint(pikgpu_ctx* ctx, const float* target, double* loss,
                   float* grad_ac, float* grad_qf, int buffers_on_device);

/* Move the forward pass off the integer lattice (finite differences of
 * pikgpu_adjoint, or a caller optimising coefficients). For the current
 * frame only (pikgpu_frame_begin clears both); NULL clears.
 * set_dequantized_ac: the dequantised AC coefficients used instead of
 *   Dequant::DoAC's (layout of pikgpu_adjoint's grad_ac); the int16 AC is
 *   then not needed.
 * set_clamp_scale: a per-cell multiplier (ysize_blocks x xsize_blocks
 *   floats) of the clamp's non-LLF intervals, which are half a quantisation
 *   step (pik/adaptive_reconstruction.cc:160-171). A quant field qf' of
 *   cell i in place of qf is modelled by scaling that cell's dequantised AC
 *   and its clamp scale by qf / qf'; pikgpu_adjoint's grad_qf is then taken
 *   at qf' = qf / scale. */
/* Verification hooks for the clamp's discrete decisions, the counterpart of
 * pikgpu_set_epf_decisions for AdaptiveReconstruction's clamp
 * (pik/adaptive_reconstruction.cc:128-244). Per coefficient, the minimum of
 * the three channels' ratios is taken by one of five branches, recorded as
 * a code: 0 no ratio below 1 (correction kept), 1..3 the ratio of channel
 * code - 1 (clamped), 4 a +0.0 correction (SymmetricClamp's ratio 0). Where
 * a correction cancels to zero, rounding decides between code 4 and a
 * neighbouring branch, so two precisions can take different branches on
 * identical inputs; sharing the codes makes their gradients comparable.
 * Layout: By x 64 Bx bytes (frame coefficient layout, first blocks'
 * entries). `get` exports the codes of the last forward pass that recorded
 * them (pikgpu_adjoint, or a reconstruction with PIKGPU_OPT_KEEP_STAGES set
 * before frame_begin; frames with the EPF only); `set` makes later passes
 * follow the given codes (NULL: computed). Host memory. */
int pikgpu_set_clamp_decisions(pikgpu_ctx* ctx, const uint8_t* tape);
int pikgpu_get_clamp_decisions(pikgpu_ctx* ctx, uint8_t* tape);

int pikgpu_frame_set_dequantized_ac(pikgpu_ctx* ctx, const float* ac,
                                    int on_device);
int pikgpu_frame_set_clamp_scale(pikgpu_ctx* ctx, const float* scale,
                                 int on_device);

#ifdef __cplusplus
}
#endif

#endif /* PIKGPU_H_ */
