// Link-time stand-ins for the four reference translation units whose
// third-party submodules (lcms2, brotli, lodepng, FiniteStateEntropy) are
// absent, so that the remaining unmodified reference sources link into a
// reference decoder/encoder used ONLY as test infrastructure (parity oracle
// and CPU baseline). Nothing here is shipped or measured as the product.
//
// What is restated and why:
//  * ColorManagement / ColorSpaceTransform (reference pik/color_management.h,
//    implementation pik/color_management.cc): only the sRGB <-> linear-sRGB
//    and identity transforms are supported, i.e. the reference's own
//    "skip lcms" route (pik/color_management.cc:745-790) with the TF_SRGB
//    rational polynomials (pik/color_management.cc:291-345). ICC profiles are
//    replaced by a non-empty placeholder, so SetProfileFromFields succeeds.
//  * Brotli, PNG and the FSE lossless entropy coder return failure: they are
//    not on the reconstruction path (metadata/ICC, file I/O, lossless mode).

#include <string.h>

#include <cmath>
#include <mutex>
#include <vector>

#include "pik/brotli.h"
#include "pik/codec_png.h"
#include "pik/color_encoding.h"
#include "pik/color_management.h"
#include "pik/lossless_entropy.h"
#include "pik/status.h"

namespace pik {

namespace {

// TF_SRGB, restated from pik/color_management.cc:291-345 (same rational
// polynomial coefficients; Horner evaluation in the order of
// pik/rational_polynomial.h:103-134 with an exact division).
float SrgbPoly(float x, const float* p, const float* q) {
  float yp = p[4], yq = q[4];
  for (int i = 3; i >= 0; --i) {
    yp = yp * x + p[i];
    yq = yq * x + q[i];
  }
  return yp / yq;
}

float DisplayFromEncodedSrgb(float x) {
  static const float p[5] = {2.200248328e-04f, 1.043637593e-02f,
                             1.624820318e-01f, 7.961564959e-01f,
                             8.210152774e-01f};
  static const float q[5] = {2.631846970e-01f, 1.076976492e+00f,
                             4.987528350e-01f, -5.512498495e-02f,
                             6.521209011e-03f};
  const float a = std::fabs(x);
  const float m = a > 0.04045f ? SrgbPoly(a, p, q) : a * (1.0f / 12.92f);
  return std::copysign(m, x);
}

float EncodedFromDisplaySrgb(float x) {
  static const float p[5] = {-5.135152395e-04f, 5.287254571e-03f,
                             3.903842876e-01f, 1.474205315e+00f,
                             7.352629620e-01f};
  static const float q[5] = {1.004519624e-02f, 3.036675394e-01f,
                             1.340816930e+00f, 9.258482155e-01f,
                             2.424867759e-02f};
  const float a = std::fabs(x);
  const float m = a > 0.0031308f ? SrgbPoly(std::sqrt(a), p, q) : a * 12.92f;
  return std::copysign(m, x);
}

// Per-instance mode, keyed by object address (the class layout is fixed by
// the reference header, so the shim keeps its own side table).
enum Mode { kCopy = 0, kToLinear = 1, kToSrgb = 2 };
struct Entry {
  const void* obj;
  int mode;
  size_t n;
};
std::vector<Entry>& Table() {
  static std::vector<Entry> t;
  return t;
}
std::mutex& TableMutex() {
  static std::mutex m;
  return m;
}

}  // namespace

Status ColorManagement::SetFromParams(const ProfileParams& pp,
                                      ColorEncoding* c) {
  return PIK_FAILURE("color management shim: SetFromParams unsupported");
}

Status ColorManagement::SetFromProfile(PaddedBytes&& icc, ColorEncoding* c) {
  return PIK_FAILURE("color management shim: SetFromProfile unsupported");
}

Status ColorManagement::MaybeRemoveProfile(ColorEncoding* c) {
  c->icc.clear();
  return true;
}

Status ColorManagement::SetProfileFromFields(ColorEncoding* c) {
  // Placeholder: the reconstruction path never reads profile bytes.
  static const char kTag[] = "pik-shim-icc";
  c->icc.resize(sizeof(kTag));
  memcpy(c->icc.data(), kTag, sizeof(kTag));
  return true;
}

ColorSpaceTransform::~ColorSpaceTransform() {
  std::lock_guard<std::mutex> lock(TableMutex());
  auto& t = Table();
  for (size_t i = 0; i < t.size(); ++i) {
    if (t[i].obj == this) {
      t.erase(t.begin() + i);
      break;
    }
  }
}

Status ColorSpaceTransform::Init(const ColorEncoding& c_src,
                                 const ColorEncoding& c_dst, size_t xsize,
                                 size_t num_threads) {
  if (!c_src.SameColorSpace(c_dst)) {
    return PIK_FAILURE("color management shim: gamut change unsupported");
  }
  int mode;
  if (c_src.transfer_function == c_dst.transfer_function) {
    mode = kCopy;
  } else if (IsSRGB(c_src.transfer_function) &&
             IsLinear(c_dst.transfer_function)) {
    mode = kToLinear;
  } else if (IsLinear(c_src.transfer_function) &&
             IsSRGB(c_dst.transfer_function)) {
    mode = kToSrgb;
  } else {
    return PIK_FAILURE("color management shim: transfer unsupported");
  }
  const size_t channels = c_src.Channels();
  buf_src_ = ImageF(xsize * channels, num_threads);
  buf_dst_ = ImageF(xsize * channels, num_threads);
  xsize_ = xsize;
  skip_lcms_ = true;
  std::lock_guard<std::mutex> lock(TableMutex());
  auto& t = Table();
  for (auto& e : t) {
    if (e.obj == this) {
      e.mode = mode;
      e.n = xsize * channels;
      return true;
    }
  }
  t.push_back(Entry{this, mode, xsize * channels});
  return true;
}

void ColorSpaceTransform::Run(const size_t thread, const float* buf_src,
                              float* buf_dst) {
  int mode = kCopy;
  size_t n = 0;
  {
    std::lock_guard<std::mutex> lock(TableMutex());
    for (const auto& e : Table()) {
      if (e.obj == this) {
        mode = e.mode;
        n = e.n;
        break;
      }
    }
  }
  for (size_t i = 0; i < n; ++i) {
    const float v = buf_src[i];
    buf_dst[i] = mode == kToLinear  ? DisplayFromEncodedSrgb(v)
                 : mode == kToSrgb ? EncodedFromDisplaySrgb(v)
                                   : v;
  }
}

Status BrotliCompress(int quality, const PaddedBytes& in,
                      PaddedBytes* PIK_RESTRICT out) {
  return PIK_FAILURE("brotli absent");
}
Status BrotliCompress(int quality, const uint8_t* in, const size_t in_size,
                      uint8_t* PIK_RESTRICT out,
                      size_t* PIK_RESTRICT total_out_size) {
  return PIK_FAILURE("brotli absent");
}
Status BrotliDecompress(const uint8_t* in, size_t max_input_size,
                        size_t max_output_size, size_t* PIK_RESTRICT bytes_read,
                        PaddedBytes* PIK_RESTRICT out) {
  return PIK_FAILURE("brotli absent");
}
Status BrotliDecompress(const PaddedBytes& in, size_t max_output_size,
                        size_t* PIK_RESTRICT bytes_read,
                        PaddedBytes* PIK_RESTRICT out) {
  return PIK_FAILURE("brotli absent");
}

Status DecodeImagePNG(const PaddedBytes& bytes, ThreadPool* pool,
                      CodecInOut* io) {
  return PIK_FAILURE("lodepng absent");
}
Status EncodeImagePNG(const CodecInOut* io, const ColorEncoding& c_desired,
                      size_t bits_per_sample, ThreadPool* pool,
                      PaddedBytes* bytes) {
  return PIK_FAILURE("lodepng absent");
}

size_t encodeVarInt(size_t value, uint8_t* output) { return 0; }
size_t decodeVarInt(const uint8_t* input, size_t inputSize, size_t* pos) {
  return 0;
}
bool MaybeEntropyEncode(const uint8_t* data, size_t size, size_t out_capacity,
                        uint8_t* out, size_t* out_size) {
  return false;
}
bool MaybeEntropyDecode(const uint8_t* data, size_t size, size_t out_capacity,
                        uint8_t* out, size_t* out_size) {
  return false;
}

}  // namespace pik
