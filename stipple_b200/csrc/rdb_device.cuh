// rdb_device.cuh -- device helpers shared by the sm_100a engines.
//
// Compiled with -fmad=false: every double multiply and add rounds on its own,
// in source order, as in the reference CPU walk (src/rd_riemersma_cpu.cpp).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "rdb_numeric.h"
#include "rdb_plan.h"

namespace rdb {

// Raises a kernel's dynamic shared-memory cap to all the device allows.  The
// cap is process-wide per kernel: setting it to one launch's own size would
// race with another host thread launching the same kernel with a larger size
// in between (that launch then fails with an invalid argument).  The maximum
// is the same value for every caller.
template <typename Kernel>
inline cudaError_t AllowMaxSmem(Kernel kernel) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa{};
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kernel);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              optin - static_cast<int>(fa.sharedSizeBytes));
}

// Error codes a kernel can leave in its status word.
enum DeviceStatus : int {
  kDevOk = 0,
  kDevBadPlan = 1,
  kDevBadItem = 2,
  kDevTimeout = 3,
};

// ----------------------------------------------------------------- Hilbert
// src/rd_riemersma_cpu.cpp:167-189 (HilbertPoint), the closed form of the
// curve quantize.c's recursion walks.
__device__ __forceinline__ void hilbert_point(uint64_t n, int level, int& ox, int& oy) {
  int x = 0, y = 0;
  for (int s = 0; s < level; ++s) {
    const int side = 1 << s;
    const int rx = static_cast<int>((n >> 1) & 1u);
    const int ry = static_cast<int>((n ^ static_cast<uint64_t>(rx)) & 1u);
    if (ry == 0) {
      if (rx == 1) {
        x = side - 1 - x;
        y = side - 1 - y;
      }
      const int t = x;
      x = y;
      y = t;
    }
    x += side * rx;
    y += side * ry;
    n >>= 2;
  }
  ox = x;
  oy = y;
}

// ------------------------------------------------------------------ plan view
struct PlanView {
  const PlanHeader* h;
  const unsigned char* pal;
  const int16_t* child;
  const uint16_t* range;
  const uint8_t* seq;
  int fan;
  int assoc;
  int stride;

  __device__ __forceinline__ void bind(const unsigned char* base) {
    h = reinterpret_cast<const PlanHeader*>(base);
    pal = base + h->off_pal;
    child = reinterpret_cast<const int16_t*>(base + h->off_child);
    range = reinterpret_cast<const uint16_t*>(base + h->off_range);
    seq = base + h->off_seq;
    fan = h->fan;
    assoc = h->assoc;
    stride = h->pal_stride;
  }
  // Distance-side colour (d*) of palette entry i.
  __device__ __forceinline__ const double* dcol(int i) const {
    return reinterpret_cast<const double*>(pal + i * stride);
  }
  // Residual-side colour (AssociateAlphaPixelInfo) of palette entry i.
  __device__ __forceinline__ const double* rcol(int i) const {
    return reinterpret_cast<const double*>(pal + i * stride) + (assoc ? 4 : 0);
  }
};

// Descent (src/rd_riemersma_cpu.cpp:82-89): bit `i` (7..1) of each channel's
// byte picks the child; stop at the first missing one.  Returns the live node.
__device__ __forceinline__ int plan_descend(const PlanView& p, unsigned br, unsigned bg,
                                            unsigned bb, unsigned ba) {
  int node = 0;
#pragma unroll 1
  for (int i = kMaxTreeDepth - 1; i > 0; --i) {
    int id = static_cast<int>(((br >> i) & 1u) | (((bg >> i) & 1u) << 1) | (((bb >> i) & 1u) << 2));
    if (p.assoc) id |= static_cast<int>(((ba >> i) & 1u) << 3);
    const int c = p.child[node * p.fan + id];
    if (c < 0) break;
    node = c;
  }
  return node;
}

// The per-pixel target as ClosestColor sees it (src/rd_octree.cpp:190-208):
// t* = beta * t with beta = QS * t.a when alpha is associated.
struct Target {
  double r, g, b, a;
};

__device__ __forceinline__ Target make_target(int assoc, double r, double g, double b, double a) {
  Target t;
  if (assoc) {
    const double beta = __dmul_rn(kQuantumScale, a);
    t.r = __dmul_rn(beta, r);
    t.g = __dmul_rn(beta, g);
    t.b = __dmul_rn(beta, b);
  } else {
    t.r = r;
    t.g = g;
    t.b = b;
  }
  t.a = a;
  return t;
}

// Full ClosestColor distance in the reference's order
// (((x^2 + y^2) + z^2) + w^2).  Early exits in the reference never change
// which candidate wins: partial sums of non-negative rounded terms are
// monotone, so a candidate reaches the final `<=` exactly when its full
// distance is at most the incumbent's.
__device__ __forceinline__ double plan_distance(const PlanView& p, int c, const Target& t) {
  const double* e = p.dcol(c);
  const double x = __dadd_rn(e[0], -t.r);
  const double y = __dadd_rn(e[1], -t.g);
  const double z = __dadd_rn(e[2], -t.b);
  double d = __dmul_rn(x, x);
  d = __dadd_rn(d, __dmul_rn(y, y));
  d = __dadd_rn(d, __dmul_rn(z, z));
  if (p.assoc) {
    const double w = __dadd_rn(e[3], -t.a);
    d = __dadd_rn(d, __dmul_rn(w, w));
  }
  return d;
}

// Thread-serial search over the run of slots: post-order, `<=` keeps the
// last equal minimum (rd_octree.cpp:198-213).  Returns the colour number.
__device__ __forceinline__ int plan_search_serial(const PlanView& p, int node, const Target& t) {
  const int start = p.range[2 * node];
  const int len = p.range[2 * node + 1];
  double best = kSearchStart;
  int index = 0;
#pragma unroll 1
  for (int s = start; s < start + len; ++s) {
    const int c = p.seq[s];
    const double d = plan_distance(p, c, t);
    if (d <= best) {
      best = d;
      index = c;
    }
  }
  return index;
}

// Warp-parallel form: lane l takes slots start+l, start+l+32, ...; then a
// butterfly keeps the minimum distance and, among equals, the highest slot.
// Every lane returns the same colour number.
__device__ __forceinline__ int plan_search_warp(const PlanView& p, int node, const Target& t,
                                                int lane) {
  const int start = p.range[2 * node];
  const int len = p.range[2 * node + 1];
  double best = kSearchStart;
  int slot = -1;
#pragma unroll 1
  for (int s = start + lane; s < start + len; s += 32) {
    const double d = plan_distance(p, p.seq[s], t);
    if (d <= best) {
      best = d;
      slot = s;
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double od = __shfl_xor_sync(0xffffffffu, best, off);
    const int os = __shfl_xor_sync(0xffffffffu, slot, off);
    if (od < best || (od == best && os > slot)) {
      best = od;
      slot = os;
    }
  }
  return slot < 0 ? 0 : static_cast<int>(p.seq[slot]);
}

// AssociateAlphaPixel (rd_types.h:179-192) of a Q16 float sample.
__device__ __forceinline__ void associate_sample(int assoc, float4 s, double& r, double& g,
                                                 double& b, double& a) {
  a = static_cast<double>(s.w);
  if (!assoc || s.w == 65535.0f) {
    r = static_cast<double>(s.x);
    g = static_cast<double>(s.y);
    b = static_cast<double>(s.z);
    return;
  }
  const double alpha = __dmul_rn(kQuantumScale, static_cast<double>(s.w));
  r = __dmul_rn(alpha, static_cast<double>(s.x));
  g = __dmul_rn(alpha, static_cast<double>(s.y));
  b = __dmul_rn(alpha, static_cast<double>(s.z));
}

// Device form of key6 for q = clamp_pixel(v): q is in [0, 65535] or NaN, and
// cvt.rzi maps NaN to 0, so no guard is needed.
__device__ __forceinline__ unsigned key6_dev(float q) {
  const unsigned twice = static_cast<unsigned>(__float2int_rz(2.0f * q));
  const unsigned v = (twice + 257u) / 2056u;
  return v > 63u ? 63u : v;
}
__device__ __forceinline__ unsigned byte_dev(float q) {
  const unsigned twice = static_cast<unsigned>(__float2int_rz(2.0f * q));
  const unsigned v = (twice + 257u) / 514u;
  return v > 255u ? 255u : v;
}

// Reads one pixel of an image as a Q16 float4 (8-bit samples widen as v*257,
// opaque alpha when there is none).
__device__ __forceinline__ float4 load_sample(const unsigned char* img, int layout,
                                              int64_t row_stride, int width, int pix) {
  const int y = pix / width;
  const int x = pix - y * width;
  const unsigned char* row = img + static_cast<int64_t>(y) * row_stride;
  if (layout == 16) return reinterpret_cast<const float4*>(row)[x];
  if (layout == 4) {
    const uchar4 v = reinterpret_cast<const uchar4*>(row)[x];
    return make_float4(v.x * 257.0f, v.y * 257.0f, v.z * 257.0f, v.w * 257.0f);
  }
  const unsigned char* q = row + 3 * x;
  return make_float4(q[0] * 257.0f, q[1] * 257.0f, q[2] * 257.0f, 65535.0f);
}

}  // namespace rdb
