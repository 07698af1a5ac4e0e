// Test infrastructure: the reference's own sRGB encoding of linear planes,
// the checker of the device's 8-bit (and 16-bit) sRGB output.
//
// TF_SRGB is compiled from the reference's own text: oracle/extract_tf_srgb.py
// copies `class TF_SRGB` out of pik/color_management.cc:291-356 into
// oracle/_ref/tf_srgb.inc (color_management.cc as a whole needs lcms2, which
// is absent), and this file compiles it against the reference's
// pik/simd/simd.h and pik/rational_polynomial.h, in the flavour of the build
// (scalar: SIMD_ENABLE=0; avx2). The steps around it restate
// ExternalImage::CopyTo's path for a linear image written as sRGB with
// bits_per_sample 8 or 16 (the ExtraTF postprocess of the skip-lcms route):
//   Image3ToTemp01      pik/external_image.cc:79-90    (x * (1.0f / 255))
//   TF_SRGB::EncodedFromDisplay, row in SIMD chunks
//                       pik/color_management.cc:929-934
//   CastClip01::FromTemp  pik/external_image.cc:666-696 (clamp to [0, 1],
//                       x width + min, GetInterval :578-586)
//   Sample::ToExternal  pik/external_image.cc:192-205  (int(sample + 0.5f))
// Built by oracle/Makefile (target `srgb`) only where the reference checkout
// is present; the .so files travel with oracle/_ref/.

#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>

#include "pik/rational_polynomial.h"
#include "pik/simd/simd.h"

namespace pik {
#include "tf_srgb.inc"

namespace {

SIMD_ATTR void EncodeRow(float* row, size_t n) {
  SIMD_FULL(float) df;
  for (size_t i = 0; i < n; i += df.N) {
    const auto val = load(df, row + i);
    const auto result = TF_SRGB().EncodedFromDisplay(val);
    store(result, df, row + i);
  }
}

}  // namespace
}  // namespace pik

extern "C" {

// linear: 3 planes (R, G, B) of ysize x xsize floats, 0..255 scale.
// out:    interleaved RGB, ysize x xsize x 3 samples; uint8_t for bits 8,
//         uint16_t (host order) for bits 16. Returns 0, or -1 on bad args.
int srgbprobe_encode(const float* linear, size_t xsize, size_t ysize,
                     int bits, void* out) {
  if (!linear || !out || (bits != 8 && bits != 16)) return -1;
  const size_t n = 3 * xsize;
  const size_t padded = (n + 63) / 64 * 64;
  float* row = static_cast<float*>(aligned_alloc(64, padded * sizeof(float)));
  if (!row) return -1;
  const float width = float((1u << bits) - 1);  // GetInterval: min 0
  const size_t plane = xsize * ysize;
  for (size_t y = 0; y < ysize; ++y) {
    memset(row, 0, padded * sizeof(float));
    for (size_t x = 0; x < xsize; ++x) {
      for (int c = 0; c < 3; ++c) {
        row[3 * x + c] = linear[c * plane + y * xsize + x] * (1.0f / 255);
      }
    }
    pik::EncodeRow(row, n);
    for (size_t i = 0; i < n; ++i) {
      const float clamped = std::min(std::max(0.0f, row[i]), 1.0f);
      const float sample = clamped * width + 0.0f;
      const int v = static_cast<int>(sample + 0.5f);
      if (bits == 8) {
        static_cast<uint8_t*>(out)[y * n + i] = static_cast<uint8_t>(v);
      } else {
        static_cast<uint16_t*>(out)[y * n + i] = static_cast<uint16_t>(v);
      }
    }
  }
  free(row);
  return 0;
}

}  // extern "C"
