/*
 * CPU restatement of google/pik's decoder reconstruction path (test
 * infrastructure: the parity oracle for the CUDA implementation).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
 * it. Built into oracle/_ref/libpikoracle.so by oracle/Makefile.
 *
 * Two precisions of one templated implementation:
 *   - FP32: float arithmetic in the reference's operation order wherever the
 *     reference is written as scalar expressions (dequant, CfL, prediction
 *     helpers, gaborish, EPF, clamp, opsin); transforms are evaluated as
 *     separable matrix products (the reference uses butterflies), so FP32
 *     results agree with the reference to rounding, not bit for bit.
 *   - FP64: the same algorithm in double precision: the accuracy oracle.
 *     Discrete EPF decisions (u8 guide, per-block sigma) can be supplied from
 *     another run so that only arithmetic error is measured.
 *
 * Parity is pinned against the reference compiled from its own sources
 * (oracle/_ref/libpikref_*.so; tests/test_oracle_golden.py) and
 * against golden fixtures generated from it (tests/golden/).
 */
#ifndef PIK_ORACLE_H_
#define PIK_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#include "../include/pikgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Stage outputs (any entry may be NULL); shapes as in PIKGPU_STAGE_*:
 *  [0] dc (3 x By x Bx)         [1] dequant_ac (3 x By x Bx*64)
 *  [2] idct (3 x 8By x 8Bx)     [3] smoothed   [4] epf   [5] ar
 *  [6] pre_opsin (3 x ysize x xsize)          [7] linear (3 x ysize x xsize)
 *  [8] srgb8 (ysize x xsize x 3 bytes, interleaved; uint8_t*)
 * Planes are dense, plane-major. */
#define PIKORACLE_NUM_STAGES 9

/* Optional EPF decisions: u8 guide planes of the padded frame with the
 * 6-pixel border (3 x (8By+12) x (8Bx+12)), per-block sigma (By x Bx), and
 * the same for the DC image's EPF (guide over the 8-padded DC image). NULL
 * fields are computed. */
typedef struct pikoracle_decisions {
  const uint8_t* guide;
  const int32_t* sigma;
  const uint8_t* dc_guide;
  const int32_t* dc_sigma;
  /* The clamp's branch per coefficient (By x 64 Bx bytes, frame coefficient
   * layout; the codes of pikgpu_get_clamp_decisions): 0 ratio 1, 1..3 the
   * ratio of channel code - 1, 4 ratio 0. NULL: computed. */
  const uint8_t* clamp_tape;
} pikoracle_decisions;

/* Runs the path in FP32. `ac` is 3 planes of By x Bx*64 int16. `stages`
 * entries are float* (entry 8: uint8_t*). Exported decisions (guide, sigma)
 * are written to `decisions_out` buffers if non-NULL. Returns 0 or <0. */
int pikoracle_run_f32(const pikgpu_frame_params* p, const int16_t* ac,
                      void* const* stages,
                      const pikoracle_decisions* decisions_in,
                      uint8_t* guide_out, int32_t* sigma_out);
/* Same in FP64; float stage entries are double*. */
int pikoracle_run_f64(const pikgpu_frame_params* p, const int16_t* ac,
                      void* const* stages,
                      const pikoracle_decisions* decisions_in,
                      uint8_t* guide_out, int32_t* sigma_out);

/* FP64 adjoint: loss L = sum over xsize x ysize x 3 of (XYB
 * reconstruction before OpsinToLinear - target)^2 and its gradient with
 * respect to the dequantised AC coefficients (`grad_ac`, 3 planes of
 * By x Bx*64, frame layout) and the per-cell quant field as a real number
 * (`grad_qf`, By x Bx). EPF decisions are held fixed (pass the base point's
 * in `decisions_in`). For finite differences the forward can be evaluated
 * off the integer lattice: `ac_dequant` (may be NULL) replaces DoAC's
 * output, `ar_scale` (may be NULL) multiplies 1/qf of each cell in the
 * clamp intervals. `target`: 3 x ysize x xsize doubles. Gradient outputs
 * may be NULL (loss only). */
int pikoracle_adjoint_f64(const pikgpu_frame_params* p, const int16_t* ac,
                          const pikoracle_decisions* decisions_in,
                          const double* ac_dequant, const double* ar_scale,
                          const double* target, double* loss,
                          double* grad_ac, double* grad_qf);

/* Single-function probes (FP64 unless noted), for unit tests:
 * transform one block of AcStrategy `type` (frame coefficient layout with
 * row stride `cstride`; pixels row stride `pstride`). */
int pikoracle_transform_f64(int type, int inverse, const double* in,
                            size_t in_stride, double* out, size_t out_stride);
int pikoracle_transform_f32(int type, int inverse, const float* in,
                            size_t in_stride, float* out, size_t out_stride);
int pikoracle_lf_helper_f32(int type, int which, const float* in,
                            size_t in_stride, float* out, size_t out_stride);
float pikoracle_epf_weight(int sigma, int sad);
void pikoracle_opsin_inverse_matrix(float* out9);
/* DCTScales/IDCTScales/L1Norm/L1NormInv for N (which 0..3). */
int pikoracle_dct_table(int n, int which, float* out);

#ifdef __cplusplus
}
#endif

#endif /* PIK_ORACLE_H_ */
