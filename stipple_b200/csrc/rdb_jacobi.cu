// rdb_jacobi.cu -- the order-free (Jacobi) approximation of the walk.
//
// Reference: src/rd_approx_cuda.cu.  Along the block-mode list the walk's
// residual obeys x - q = (I - H) e, so the diffused target collapses to
//     t = q + F (x - q),   F = (I - H)^-1 truncated to `taps` taps,
// and q <- Q(t) is iterated to a fixed point, every sweep a convolution along
// the curve followed by a cache-free octree lookup.  It converges toward the
// cache-free walk, not the memoised one, and is held to a tolerance (index
// mismatch fraction and mean CIE dE76 against the sequential walk), not to
// equality.
//
// The convolution is tiled: a CTA stages the residuals r = x - pal[q] of its
// 256 positions plus the `taps` before them in shared memory once, so each
// residual is read from HBM once per sweep.  The FP32 path uses FMA (it is an
// approximation; the exact engines never contract).
#include <cuda_runtime.h>

#include "rdb_device.cuh"
#include "rdb_walk.h"

namespace rdb {
namespace {

constexpr int kTile = 256;

template <typename T>
__global__ void JacobiGather(JacobiLaunch L) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L.n) return;
  const int pix = (i == L.n - 1) ? 0 : L.order[i];
  const float4 s = load_sample(L.pixels, L.layout, L.row_stride, L.width, pix);
  T* cx = static_cast<T*>(L.cx) + 4 * static_cast<int64_t>(i);
  cx[0] = static_cast<T>(s.x);
  cx[1] = static_cast<T>(s.y);
  cx[2] = static_cast<T>(s.z);
  cx[3] = static_cast<T>(s.w);
}

// rd_cuda_common.cuh:57-72 (d_associate_from_double) then the cache-free
// selection (:449-476 with a null cache).
__device__ __forceinline__ int jacobi_select(const PlanView& P, double vr, double vg, double vb,
                                             double va) {
  const float fr = clamp_pixel(vr), fg = clamp_pixel(vg), fb = clamp_pixel(vb);
  const float fa = clamp_pixel(va);
  double tr = fr, tg = fg, tb = fb;
  const double ta = fa;
  if (P.assoc && va != kQuantumRange) {
    const double alpha = __dmul_rn(kQuantumScale, ta);
    tr = __dmul_rn(alpha, tr);
    tg = __dmul_rn(alpha, tg);
    tb = __dmul_rn(alpha, tb);
  }
  const unsigned br = byte_dev(clamp_pixel(tr)), bg = byte_dev(clamp_pixel(tg));
  const unsigned bb = byte_dev(clamp_pixel(tb)), ba = byte_dev(clamp_pixel(ta));
  const int node = plan_descend(P, br, bg, bb, ba);
  Target t;
  if (P.assoc) {
    t = make_target(1, tr, tg, tb, ta);
  } else {
    t.r = tr;
    t.g = tg;
    t.b = tb;
    t.a = ta;
  }
  return plan_search_serial(P, node, t);
}

template <typename T>
__global__ void JacobiInit(JacobiLaunch L) {
  extern __shared__ __align__(16) unsigned char smem[];
  for (int i = threadIdx.x; i < L.plan_smem / 16; i += blockDim.x) {
    reinterpret_cast<int4*>(smem)[i] = reinterpret_cast<const int4*>(L.plan)[i];
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L.n) return;
  PlanView P;
  P.bind(smem);
  const T* cx = static_cast<const T*>(L.cx) + 4 * static_cast<int64_t>(i);
  float4 s = make_float4(static_cast<float>(cx[0]), static_cast<float>(cx[1]),
                         static_cast<float>(cx[2]), static_cast<float>(cx[3]));
  double r, g, b, a;
  associate_sample(P.assoc, s, r, g, b, a);
  const float fr = clamp_pixel(r), fg = clamp_pixel(g), fb = clamp_pixel(b), fa = clamp_pixel(a);
  const int node = plan_descend(P, byte_dev(fr), byte_dev(fg), byte_dev(fb), byte_dev(fa));
  const Target t = make_target(P.assoc, r, g, b, a);
  L.q0[i] = static_cast<uint8_t>(plan_search_serial(P, node, t));
}

template <typename T>
__device__ __forceinline__ T mul_add(T a, T b, T c);
template <>
__device__ __forceinline__ float mul_add<float>(float a, float b, float c) {
  return __fmaf_rn(a, b, c);
}
template <>
__device__ __forceinline__ double mul_add<double>(double a, double b, double c) {
  return __fma_rn(a, b, c);
}

template <typename T>
__global__ void __launch_bounds__(kTile) JacobiSweep(JacobiLaunch L, const uint8_t* q_in,
                                                     uint8_t* q_out) {
  extern __shared__ __align__(16) unsigned char smem[];
  for (int i = threadIdx.x; i < L.plan_smem / 16; i += blockDim.x) {
    reinterpret_cast<int4*>(smem)[i] = reinterpret_cast<const int4*>(L.plan)[i];
  }
  __syncthreads();
  PlanView P;
  P.bind(smem);
  T* win = reinterpret_cast<T*>(smem + L.plan_smem);  // (kTile + taps) x 4 residuals
  T* gs = win + 4 * (kTile + L.taps);                    // taps + 1 coefficients
  const int taps = L.taps;
  const int tile0 = blockIdx.x * kTile;
  const int origin = tile0 - taps;
  const T* cx = static_cast<const T*>(L.cx);
  for (int k = threadIdx.x; k < kTile + taps; k += blockDim.x) {
    const int m = origin + k;
    T r0 = T(0), r1 = T(0), r2 = T(0), r3 = T(0);
    if (m >= 0 && m < L.n) {
      // Palette entries are floats widened to double (ClampToQuantum), so
      // the float copy in the plan's output table is exact.
      const float4 o = reinterpret_cast<const float4*>(L.plan + P.h->off_out)[q_in[m]];
      r0 = cx[4 * static_cast<int64_t>(m) + 0] - static_cast<T>(o.x);
      r1 = cx[4 * static_cast<int64_t>(m) + 1] - static_cast<T>(o.y);
      r2 = cx[4 * static_cast<int64_t>(m) + 2] - static_cast<T>(o.z);
      r3 = cx[4 * static_cast<int64_t>(m) + 3] - static_cast<T>(o.w);
    }
    win[4 * k + 0] = r0;
    win[4 * k + 1] = r1;
    win[4 * k + 2] = r2;
    win[4 * k + 3] = r3;
  }
  for (int d = threadIdx.x; d <= taps; d += blockDim.x) gs[d] = static_cast<T>(L.g[d]);
  __syncthreads();
  const int i = tile0 + threadIdx.x;
  if (i >= L.n) return;
  const int here = threadIdx.x + taps;
  const int dmax = taps < i ? taps : i;
  T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
#pragma unroll 4
  for (int d = 0; d <= dmax; ++d) {
    const T gk = gs[d];
    const T* w = win + 4 * (here - d);
    a0 = mul_add(gk, w[0], a0);
    a1 = mul_add(gk, w[1], a1);
    a2 = mul_add(gk, w[2], a2);
    a3 = mul_add(gk, w[3], a3);
  }
  const float4 p0 = reinterpret_cast<const float4*>(L.plan + P.h->off_out)[q_in[i]];
  const double vr = static_cast<double>(p0.x) + static_cast<double>(a0);
  const double vg = static_cast<double>(p0.y) + static_cast<double>(a1);
  const double vb = static_cast<double>(p0.z) + static_cast<double>(a2);
  const double va = P.assoc ? (static_cast<double>(p0.w) + static_cast<double>(a3)) : kQuantumRange;
  q_out[i] = static_cast<uint8_t>(jacobi_select(P, vr, vg, vb, va));
}

__global__ void JacobiScatter(JacobiLaunch L, const uint8_t* q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L.n) return;
  const int64_t npix = static_cast<int64_t>(L.width) * L.height;
  if (i == 0 && L.n > 1) {
    if (L.n == npix && L.rgba_out) {
      const int gap = L.width - 1;
      L.rgba_out[gap] = load_sample(L.pixels, L.layout, L.row_stride, L.width, gap);
    }
    return;
  }
  const int pix = (i == L.n - 1) ? 0 : L.order[i];
  const uint8_t index = q[i];
  L.indices[pix] = index;
  if (L.rgba_out) {
    const PlanHeader* h = reinterpret_cast<const PlanHeader*>(L.plan);
    const float4 pc = reinterpret_cast<const float4*>(L.plan + h->off_out)[index];
    const float a = h->assoc ? pc.w : load_sample(L.pixels, L.layout, L.row_stride, L.width, pix).w;
    L.rgba_out[pix] = make_float4(pc.x, pc.y, pc.z, a);
  }
}

template <typename T>
cudaError_t Run(const JacobiLaunch& L, cudaStream_t stream) {
  const unsigned g = static_cast<unsigned>((L.n + 255) / 256);
  JacobiGather<T><<<g, 256, 0, stream>>>(L);
  cudaError_t e = AllowMaxSmem(JacobiInit<T>);
  if (e != cudaSuccess) return e;
  JacobiInit<T><<<g, 256, L.plan_smem, stream>>>(L);
  const std::size_t smem = static_cast<std::size_t>(L.plan_smem) +
                           sizeof(T) * 4 * static_cast<std::size_t>(kTile + L.taps) +
                           sizeof(T) * static_cast<std::size_t>(L.taps + 1);
  e = AllowMaxSmem(JacobiSweep<T>);
  if (e != cudaSuccess) return e;
  const unsigned tiles = static_cast<unsigned>((L.n + kTile - 1) / kTile);
  uint8_t* a = L.q0;
  uint8_t* b = L.q1;
  for (int it = 0; it < L.iterations; ++it) {
    JacobiSweep<T><<<tiles, kTile, smem, stream>>>(L, a, b);
    uint8_t* t = a;
    a = b;
    b = t;
  }
  JacobiScatter<<<g, 256, 0, stream>>>(L, a);
  return cudaGetLastError();
}

}  // namespace

cudaError_t LaunchJacobi(const JacobiLaunch& L, cudaStream_t stream) {
  if (L.n <= 0) return cudaSuccess;
  return L.fp64 ? Run<double>(L, stream) : Run<float>(L, stream);
}

}  // namespace rdb
