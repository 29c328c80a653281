// rdb_cand.cu -- the candidate table (see rdb_cand.h).
#include <cuda_runtime.h>

#include "rdb_cand.h"
#include "rdb_device.cuh"
#include "rdb_walk_thread.cuh"

namespace rdb {
namespace {

// max over the box of d(x, w) - d(x, j): affine in x once the squares cancel,
// so each channel takes the corner that maximises it.
__device__ __forceinline__ double MaxGap(const double* const (&row)[3], int w, int j,
                                         const double (&lo)[3], const double (&hi)[3]) {
  double f = 0.0;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double a = row[c][w], b = row[c][j];
    const double x = (a - b) > 0.0 ? lo[c] : hi[c];
    f += (a * a - b * b) - 2.0 * x * (a - b);
  }
  return f;
}

__global__ void CandidateKernel(const unsigned char* plan, uint32_t* out) {
  const int key = blockIdx.x * blockDim.x + threadIdx.x;
  if (key >= kCandKeys) return;
  tw::Plan P;
  P.bind(plan);
  const unsigned kc[3] = {static_cast<unsigned>(key) & 63u, (static_cast<unsigned>(key) >> 6) & 63u,
                          static_cast<unsigned>(key) >> 12};
  // Inside a key only byte bit 1 varies among the bits the descent reads.
  int node = -1;
#pragma unroll 1
  for (int c = 0; c < 8; ++c) {
    const int nd = tw::descend<false>(P, 4u * kc[0] + ((c & 1) ? 2u : 0u), 4u * kc[1] + ((c & 2) ? 2u : 0u),
                                      4u * kc[2] + ((c & 4) ? 2u : 0u), 0u);
    if (node < 0) {
      node = nd;
    } else if (nd != node) {
      out[key] = kCandFallback;
      return;
    }
  }
  // Targets q with byte(q) in [4k, 4k + 3]: q in [1028k - 128.5, 1028k + 899.5),
  // within the clamp range [0, 65535].
  double lo[3], hi[3], mid[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    lo[c] = fmax(0.0, 1028.0 * kc[c] - 128.5);
    hi[c] = fmin(65535.0, 1028.0 * kc[c] + 899.5);
    mid[c] = 0.5 * (lo[c] + hi[c]);
  }
  const int start = P.range[2 * node];
  const int len = P.range[2 * node + 1];
  const double* const row[3] = {P.slotpal, P.slotpal + P.slot_stride, P.slotpal + 2 * P.slot_stride};
  // A first dominator to try: the nearest slot at the box centre.
  int near = start;
  double best = 1e300;
#pragma unroll 1
  for (int s = start; s < start + len; ++s) {
    double d = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double x = row[c][s] - mid[c];
      d += x * x;
    }
    if (d < best) {
      best = d;
      near = s;
    }
  }
  // Survivors: slots no other slot beats by the margin everywhere in the box.
  unsigned packed = 0;
  int n = 0;
#pragma unroll 1
  for (int j = start; j < start + len; ++j) {
    bool dominated = j != near && MaxGap(row, near, j, lo, hi) < -kCandMargin;
#pragma unroll 1
    for (int w = start; w < start + len && !dominated; ++w) {
      if (w != j && MaxGap(row, w, j, lo, hi) < -kCandMargin) dominated = true;
    }
    if (dominated) continue;
    if (n == 4) {
      out[key] = kCandFallback;
      return;
    }
    packed |= static_cast<unsigned>(j) << (8 * n);
    ++n;
  }
  if (n == 0) {
    out[key] = kCandFallback;  // cannot happen: the overall minimum is never beaten
    return;
  }
  // Repeat the last survivor into the unused bytes.
  const unsigned last = (packed >> (8 * (n - 1))) & 0xFFu;
  for (int i = n; i < 4; ++i) packed |= last << (8 * i);
  out[key] = packed;
}

}  // namespace

cudaError_t LaunchCandidateTable(const unsigned char* plan, uint32_t* out, cudaStream_t s) {
  CandidateKernel<<<kCandKeys / 128, 128, 0, s>>>(plan, out);
  return cudaGetLastError();
}

}  // namespace rdb
