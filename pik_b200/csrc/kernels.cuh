// Device kernels of the reconstruction path (sm_100a).
//
// Arithmetic is IEEE single precision with every multiply and add rounded
// separately (this translation unit is compiled with -fmad=false) and sums
// taken in a fixed order; transforms are separable matrix products with the
// matrices of tables.h. This makes the plain FP32 form deterministic and
// reproducible run to run.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "tables.h"

namespace pikgpu {


// AcStrategy types (pik/ac_strategy.h:51-70).
enum : int {
  kDCT = 0, kIDENTITY = 1, kDCT2X2 = 2, kDCT4X4 = 3, kDCT16X16 = 4,
  kDCT32X32 = 5, kLINES = 6, kDCT_NOHF = 7, kDCT4X4_NOHF = 8
};

__host__ __device__ inline int Covered(int type) {
  return type == kDCT32X32 ? 4 : type == kDCT16X16 ? 2 : 1;
}
__host__ __device__ inline int QuantKindOf(int type) {
  return type == kDCT_NOHF ? 0 : type == kDCT4X4_NOHF ? 3 : type;
}
__host__ __device__ inline bool PredictHFOf(int type) {
  return type != kDCT2X2 && type != kIDENTITY && type != kDCT_NOHF &&
         type != kDCT4X4_NOHF && type != kLINES;
}
__device__ inline float ARQuantScaleOf(int type) {
  if (type == kDCT32X32) return 1.2282996852328099f;
  if (type == kDCT16X16) return 1.1423171621463439f;
  if (type == kDCT4X4 || type == kDCT4X4_NOHF) return 1.2f;
  if (type == kDCT2X2) return 1.0098134203870499f;
  return 1.0f;
}

// Mirror with the edge sample repeated once (pik/image_ops.h:217-227),
// reflecting repeatedly for overshoots larger than the size.
__host__ __device__ inline int MirrorIdx(int x, int size) {
  while (x < 0 || x >= size) {
    x = x < 0 ? -x - 1 : 2 * size - 1 - x;
  }
  return x;
}

// Programmatic dependent launch (PTX griddepcontrol, sm_90 and later). The
// transform classes, and the clamp classes, run as a chain of kernels on
// one stream, each launched as a programmatic dependent of the one before
// it: a dependent may start once every CTA of its predecessor has executed
// PdlLaunchDependents (or exited), which the chain kernels do first thing.
// The classes write disjoint blocks, so the one order kept is completion:
// PdlTail, declared at the top of a chain kernel, waits for the
// predecessor's completion (and the visibility of its writes) on every
// return path, so the chain's last kernel completes after all of them.
// Both instructions do nothing in a launch without such a dependency.
__device__ __forceinline__ void PdlLaunchDependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
struct PdlTail {
  __device__ __forceinline__ ~PdlTail() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
  }
};
// On the main stream, kernels that read their predecessor's output (the
// EPF reads the guide range of the min/max pass, the active-block pass the
// EPF's sigma) may also be launched that way: they call PdlWait before the
// first such read, and what comes before it (staging the frame's tile, say)
// overlaps the predecessor's last CTAs.
__device__ __forceinline__ void PdlWait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Frame geometry.
struct Geo {
  int W, H;       // pixels
  int Bx, By;     // blocks
  int PW, PH;     // padded pixels (8 Bx, 8 By)
  int Tx, Ty;     // 64-pixel tiles
  int Gx, Gy;     // 512-pixel groups
  int ac_stride;  // Bx * 64
};

// Per-group bordered arrays: llf (66 x 66) and 2x2 images (132 x 132).
constexpr int kGB = 66;
constexpr int kG2 = 132;
constexpr size_t kG2GroupFloats = size_t(3) * kG2 * kG2;

struct FrameScalars {
  float inv_global_scale;  // Quantizer::InvGlobalScale
  float inv_quant_dc;      // Quantizer::inv_quant_dc (decoder form)
  float mul_dc[3];         // DequantMatrix(0, DCT8, c)[0] * inv_quant_dc
  float ytox_dc, ytob_dc;  // YtoX(1, ytox_dc), YtoB(1, ytob_dc)
  int gaborish;
  int predict_lf, predict_hf;
  int have_ar;
  int use_sharpened;
  int quant_dc;
  // EpfParams::sigma when enable_adaptive is false, else -1.
  int epf_fixed_sigma;
};

// The first blocks of each transform class (x | y << 16), their count, and
// where the clamp's active blocks of the class go.
constexpr int kMaxClasses = 5;
struct ClassLists {
  const uint32_t* list[kMaxClasses];
  int n[kMaxClasses];
  uint32_t* active[kMaxClasses];
};

// Device pointers of one frame.
struct DevFrame {
  const uint8_t* acs;
  const int32_t* qf;
  const uint8_t* lut;
  const uint8_t* dq_cf;
  const uint8_t* dq_map;
  const int32_t* ytox;
  const int32_t* ytob;
  const float* table;
  const uint32_t* offsets;
  const int16_t* qdc;
  const int16_t* qac;
  float* dc;          // 3 x By x Bx
  float* ac;          // 3 x By x ac_stride
  float* pred2x2_g;   // groups x 3 x 132 x 132
  float* idct;        // 3 x PH x PW
  float* smoothed;    // 3 x PH x PW
  float* filt;        // 3 x PH x PW
  // Optional per-cell multiplier of the clamp's half-step interval (NULL:
  // none), By x Bx.
  const float* clamp_scale;
  // Optional clamp tape (By x ac_stride bytes, frame coefficient layout;
  // NULL: not written): the clamp's branch per coefficient, for the adjoint.
  uint8_t* clamp_tape;
  // Optional clamp tape to follow instead of the computed minimum (same
  // layout; NULL: computed), pikgpu_set_clamp_decisions.
  const uint8_t* clamp_tape_in;
  // Polls of the tensor-core kernels' first wait on each MMA completion
  // (tc::WaitMma).
  uint32_t tc_polls;
};

}  // namespace pikgpu
