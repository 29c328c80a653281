// rdb_uniform.cu -- the uniform-key table (see rdb_uniform.h).
#include <cuda_runtime.h>

#include "rdb_device.cuh"
#include "rdb_uniform.h"
#include "rdb_uniform_alpha.cuh"
#include "rdb_walk_thread.cuh"

namespace rdb {
namespace {

__global__ void UniformKernel(const unsigned char* plan, uint8_t* out) {
  const int key = blockIdx.x * blockDim.x + threadIdx.x;
  if (key >= kUniformKeys) return;
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
      out[key] = kNotUniform;
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
    mid[c] = static_cast<double>(static_cast<float>(0.5 * (lo[c] + hi[c])));
  }
  const int start = P.range[2 * node];
  const int len = P.range[2 * node + 1];
  const double* row[3] = {P.slotpal, P.slotpal + P.slot_stride, P.slotpal + 2 * P.slot_stride};
  double best = kSearchStart;
  int win = -1;
#pragma unroll 1
  for (int s = start; s < start + len; ++s) {
    double d = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double x = row[c][s] - mid[c];
      d += x * x;
    }
    if (d <= best) {
      best = d;
      win = s;
    }
  }
  if (win < 0) {
    out[key] = kNotUniform;
    return;
  }
#pragma unroll 1
  for (int s = start; s < start + len; ++s) {
    if (s == win) continue;
    double f = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double w = row[c][win], j = row[c][s];
      const double x = (w - j) > 0.0 ? lo[c] : hi[c];
      f += (w * w - j * j) - 2.0 * x * (w - j);
    }
    if (f > -1.0) {
      out[key] = kNotUniform;
      return;
    }
  }
  out[key] = P.seq[win];
}

// Every key of an alpha-associated palette's table still marked unknown.
__global__ void UniformAlphaKernel(const unsigned char* plan, uint8_t* out) {
  const unsigned key = blockIdx.x * blockDim.x + threadIdx.x;
  if (key >= static_cast<unsigned>(kUniformKeysAlpha) || out[key] != kUniformUnknown) return;
  tw::Plan P;
  P.bind(plan);
  out[key] = uniform_alpha_key(P, key);
}

}  // namespace

cudaError_t LaunchUniformTableAlpha(const unsigned char* plan, uint8_t* out, cudaStream_t s) {
  UniformAlphaKernel<<<kUniformKeysAlpha / 256, 256, 0, s>>>(plan, out);
  return cudaGetLastError();
}

cudaError_t LaunchUniformTable(const unsigned char* plan, uint8_t* out, cudaStream_t s) {
  UniformKernel<<<kUniformKeys / 256, 256, 0, s>>>(plan, out);
  return cudaGetLastError();
}

}  // namespace rdb
