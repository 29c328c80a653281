// rdb_uniform_alpha.cuh -- uniform keys of alpha-associated palettes.
//
// The 24-bit memo key of an alpha-associated palette keeps the top 6 bits of
// the r, g, b and a bytes of the clamped pixel (rd_types.h:141-153).  The
// lookup descends by byte bits 7..1 of all four channels and runs
// ClosestColor over the stopping node's parent with the target associated
// once more: (b * r, b * g, b * b, a) with b = QuantumScale * a, each product
// rounded (src/rd_octree.cpp:190-208, src/rd_riemersma_cpu.cpp:82-92).
//
// The argument of rdb_uniform.h carries over: inside a key only byte bit 1 of
// each channel varies among the bits the descent reads (16 combinations), and
// the distance difference of two candidates is affine in the associated
// target, whose coordinates lie in a box fixed by the key -- rounding is
// monotone, so (QS * a_lo) * c_lo and (QS * a_hi) * c_hi bound every product
// the walk can form.  One candidate nearer than every other by a margin of 1.0
// over that box is the search result, and so the memo value, of every target
// with the key.  Colours 254 and 255 are never marked: 0xFE means "not yet
// classified" in the walk's lazily filled table, 0xFF "not uniform".
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "rdb_device.cuh"
#include "rdb_uniform.h"
#include "rdb_walk_thread.cuh"

namespace rdb {

__device__ __forceinline__ uint8_t uniform_alpha_key(const tw::Plan& P, unsigned key) {
  const unsigned kc[4] = {key & 63u, (key >> 6) & 63u, (key >> 12) & 63u, (key >> 18) & 63u};
  int node = -1;
#pragma unroll 1
  for (int c = 0; c < 16; ++c) {
    const int nd = tw::descend<true>(P, 4u * kc[0] + ((c & 1) ? 2u : 0u), 4u * kc[1] + ((c & 2) ? 2u : 0u),
                                     4u * kc[2] + ((c & 4) ? 2u : 0u), 4u * kc[3] + ((c & 8) ? 2u : 0u));
    if (node < 0) {
      node = nd;
    } else if (nd != node) {
      return kNotUniform;
    }
  }
  // Clamped targets with byte(q) in [4k, 4k + 3]: q in [1028k - 128.5, 1028k + 899.5).
  double lo[4], hi[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    lo[c] = fmax(0.0, 1028.0 * kc[c] - 128.5);
    hi[c] = fmin(65535.0, 1028.0 * kc[c] + 899.5);
  }
  // The search target's box: r, g, b associated by the alpha factor, alpha as is.
  const double blo = __dmul_rn(kQuantumScale, lo[3]);
  const double bhi = __dmul_rn(kQuantumScale, hi[3]);
  double tl[4], th[4], mid[4];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    tl[c] = __dmul_rn(blo, lo[c]);
    th[c] = __dmul_rn(bhi, hi[c]);
  }
  tl[3] = lo[3];
  th[3] = hi[3];
#pragma unroll
  for (int c = 0; c < 4; ++c) mid[c] = 0.5 * (tl[c] + th[c]);
  const int start = P.range[2 * node];
  const int len = P.range[2 * node + 1];
  const double* row[4] = {P.slotpal, P.slotpal + P.slot_stride, P.slotpal + 2 * P.slot_stride,
                          P.slotpal + 3 * P.slot_stride};
  double best = kSearchStart;
  int win = -1;
#pragma unroll 1
  for (int s = start; s < start + len; ++s) {
    double d = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const double x = row[c][s] - mid[c];
      d += x * x;
    }
    if (d <= best) {
      best = d;
      win = s;
    }
  }
  if (win < 0) return kNotUniform;
#pragma unroll 1
  for (int s = start; s < start + len; ++s) {
    if (s == win) continue;
    // max over the box of d(win) - d(s): each coordinate at the end that
    // favours s.
    double f = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const double w = row[c][win], j = row[c][s];
      const double x = (w - j) > 0.0 ? tl[c] : th[c];
      f += (w * w - j * j) - 2.0 * x * (w - j);
    }
    if (f > -1.0) return kNotUniform;
  }
  const unsigned col = P.seq[win];
  return col >= kUniformUnknown ? kNotUniform : static_cast<uint8_t>(col);
}

}  // namespace rdb
