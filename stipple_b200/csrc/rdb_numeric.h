// rdb_numeric.h -- the ImageMagick 7 Q16-HDRI numeric contract, shared by the
// host code and the sm_100a kernels.
//
// Reference: include/rd_types.h (rdither).  Every function below produces the
// same bits as its reference counterpart; the sources compile with
// -fmad=false (device) and -ffp-contract=off (host) so that no multiply-add
// is contracted.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define RDB_HD __host__ __device__ __forceinline__
#else
#define RDB_HD inline
#endif

namespace rdb {

constexpr double kQuantumRange = 65535.0;          // rd_types.h:24
constexpr double kQuantumScale = 1.0 / 65535.0;    // rd_types.h:25
constexpr double kOpaqueAlpha = 65535.0;           // rd_types.h:26
constexpr double kEpsilon = 1.0e-12;               // rd_types.h:27
constexpr int kQueue = 16;                         // rd_types.h:100
constexpr int kMaxTreeDepth = 8;                   // rd_types.h:106
constexpr int kMaxColormap = 65536;                // rd_types.h:109
// Initial ClosestColor distance, src/rd_riemersma_cpu.cpp:90.
constexpr double kSearchStart = 4.0 * ((kQuantumRange + 1.0) * (kQuantumRange + 1.0)) + 1.0;

// rd_types.h:30-33 (MagickSafeReciprocal).
RDB_HD double safe_reciprocal(double x) {
  const double sign = (x < 0.0) ? -1.0 : 1.0;
  return ((sign * x) >= kEpsilon) ? 1.0 / x : sign * (1.0 / kEpsilon);
}

// rd_types.h:39-43 (ClampPixel narrows through float).  NaN passes through as
// a float NaN, like the reference.
RDB_HD float clamp_pixel(double v) {
  if (v < 0.0) return 0.0f;
  if (v >= kQuantumRange) return 65535.0f;
  return static_cast<float>(v);
}

// rd_types.h:133-138 (ScaleQuantumToChar: q / 257.0f + 0.5f, truncated) for
// q = clamp_pixel(v), i.e. q in [0, 65535] or NaN.
//
// The float quotient and sum round to exactly the thresholds 257k - 128.5, so
// the byte is the count of those thresholds at or below q:
//     byte = min(255, (trunc(2q) + 257) / 514)
// Checked exhaustively against the division form over every float in
// [0, 65535] (tests/test_numeric.py).  This takes the IEEE divide off the
// dependent chain of the sequential walk.
RDB_HD unsigned scale_char(float q) {
  if (!(q > 0.0f)) return 0u;  // zero, -0 and NaN
  const unsigned twice = static_cast<unsigned>(static_cast<int>(2.0f * q));
  const unsigned v = (twice + 257u) / 514u;
  return v > 255u ? 255u : v;
}

// The top 6 bits of scale_char (rd_types.h:142, `>> kCacheShift`), directly.
RDB_HD unsigned key6(float q) {
  if (!(q > 0.0f)) return 0u;
  const unsigned twice = static_cast<unsigned>(static_cast<int>(2.0f * q));
  const unsigned v = (twice + 257u) / 2056u;
  return v > 63u ? 63u : v;
}

// rd_types.h:141-153 (CacheOffset) from already-clamped floats.
RDB_HD unsigned cache_key(bool assoc, float r, float g, float b, float a) {
  unsigned k = key6(r) | (key6(g) << 6) | (key6(b) << 12);
  if (assoc) k |= key6(a) << 18;
  return k;
}

// rd_types.h:169-176 (the error weights 16^(-i/15), by IM's own recurrence).
// Host functions (std::exp/std::log), defined in rdb_octree.cpp.
void error_weights(double w[kQueue]);
// scaled_w[k] = (kErrorRelativeWeight * diffusion) * weights[k],
// src/rd_riemersma_cpu.cpp:370-373.
void scaled_weights(double diffusion, double out[kQueue]);

}  // namespace rdb
