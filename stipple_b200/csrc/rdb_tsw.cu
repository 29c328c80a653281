// rdb_tsw.cu -- kernels of the thread-walker segmented walk (see rdb_tsw.h).
//
// The per-position arithmetic is the block engine's thread walker
// (rdb_walk_thread.cuh): running sums of the 16 upcoming pixels in
// registers, rotated by a 16-way switch, the weights as constant operands,
// FP64 in the reference's operation order (src/rd_riemersma_cpu.cpp:39-113).
// What differs from a block is the start state (a carried or warmed-up
// queue instead of zeros) and the memo (rdb_tsw.h).
#include <cuda_runtime.h>

#include "rdb_device.cuh"
#include "rdb_tsw.h"
#include "rdb_uniform.h"
#include "rdb_walk_thread.cuh"

namespace rdb {
namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr uint32_t kNoUser = 0x7FFFFFFFu;
constexpr int kKeys = 1 << 18;

__device__ __forceinline__ int front_of(const TswLaunch& L, int image, int nsegs) {
  const int b = L.bad[(L.pass & 1) ^ 1][image];
  return b < nsegs ? b : nsegs;
}

__device__ __forceinline__ int find_image(const TswImage* imgs, int n, int64_t pos) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (imgs[mid].cx_offset <= pos) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ uint32_t pack_rgb8(const unsigned char* img, int layout, int64_t stride,
                                              int width, int pix) {
  const int y = pix / width;
  const int x = pix - y * width;
  const unsigned char* row = img + static_cast<int64_t>(y) * stride;
  if (layout == 4) return reinterpret_cast<const uint32_t*>(row)[x];
  const unsigned char* q = row + 3 * x;
  return static_cast<uint32_t>(q[0]) | (static_cast<uint32_t>(q[1]) << 8) |
         (static_cast<uint32_t>(q[2]) << 16) | 0xFF000000u;
}

__global__ void TswGather(TswLaunch L, int64_t total) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int m = find_image(L.images, L.n_images, i);
  const TswImage& im = L.images[m];
  const int64_t pos = i - im.cx_offset;
  if (pos >= im.n) return;  // alignment padding
  int pix = im.order[pos];
  if (static_cast<unsigned>(pix) >= static_cast<unsigned>(im.n)) {
    atomicExch(L.status, kDevBadItem);
    pix = 0;
  }
  if (L.is_float) {
    reinterpret_cast<float4*>(const_cast<void*>(L.cx))[i] =
        load_sample(im.pixels, im.layout, im.row_stride, im.width, pix);
  } else {
    reinterpret_cast<uint32_t*>(const_cast<void*>(L.cx))[i] =
        pack_rgb8(im.pixels, im.layout, im.row_stride, im.width, pix);
  }
}

template <bool kFloat>
__device__ __forceinline__ void sample(const TswLaunch& L, int64_t at, double (&p)[3]) {
  if (kFloat) {
    const float4 s = reinterpret_cast<const float4*>(L.cx)[at];
    p[0] = static_cast<double>(s.x);
    p[1] = static_cast<double>(s.y);
    p[2] = static_cast<double>(s.z);
  } else {
    const uint32_t w = reinterpret_cast<const uint32_t*>(L.cx)[at];
    p[0] = static_cast<double>((w & 0xFFu) * 257u);
    p[1] = static_cast<double>(((w >> 8) & 0xFFu) * 257u);
    p[2] = static_cast<double>(((w >> 16) & 0xFFu) * 257u);
  }
}

// Pixel t (slot U) takes its last term w15 * e_{t-1}; the 15 pixels after it
// take e_{t-1} with their weights; slot U is refilled with pixel t + 16.
template <int U>
__device__ __forceinline__ void Rotate(const double (&sw)[16], double (&R)[16][3],
                                       const double (&e)[3], double (&v)[3], const double (&p)[3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) v[c] = __dadd_rn(R[U][c], __dmul_rn(sw[15], e[c]));
#pragma unroll
  for (int jj = 1; jj < 16; ++jj) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      R[(U + jj) & 15][c] = __dadd_rn(R[(U + jj) & 15][c], __dmul_rn(sw[15 - jj], e[c]));
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) R[U][c] = p[c];
}

__device__ __forceinline__ unsigned own_hash(unsigned key) { return (key * 0x9E3779B1u) >> 8; }

// Fire-and-forget minimum (no value comes back, so nothing waits on it).
__device__ __forceinline__ void red_min(uint32_t* p, uint32_t v) {
  asm volatile("red.relaxed.gpu.global.min.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Segment k of one image, one thread per segment.  The step loop is
// warp-uniform (every lane runs the warp's longest segment's step count,
// idle past its own), so lanes that need a colour search hand it to the
// whole warp: each search is spread over the 32 lanes instead of running
// serially in one lane while the other 31 wait.
template <bool kFloat>
__device__ __forceinline__ void WalkSegment(const TswLaunch& L, const TswImage& im,
                                            const tw::Plan& P, const double* errp, int k,
                                            bool active, int lane) {
  const int sid = im.first_seg + k;
  const int begin = k * L.seg_len;
  const int end = active ? min(begin + L.seg_len, im.n) : begin;
  const bool warmup = L.pass == 0 && k > 0;
  const int ws = (active && warmup) ? begin - min(begin, L.warm_len) : begin;
  const int steps = end - ws;
  const int64_t base = im.cx_offset;
  const bool memo = L.use_cache != 0;

  double R[16][3];
  double e[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int u = 0; u < 16; ++u) {
    double p[3] = {0.0, 0.0, 0.0};
    if (ws + u < end) sample<kFloat>(L, base + ws + u, p);
#pragma unroll
    for (int c = 0; c < 3; ++c) R[u][c] = p[c];
  }
  if (active && !warmup && k > 0) {
    // Start from the predecessor's end queue q[0..15] (oldest first): pixel
    // begin + j holds p + sum_{m=j}^{14} w_{m-j} q[m] in ascending m, and
    // q[15] is the pending residual.
    const double* q = L.q_end[(L.pass & 1) ^ 1] + static_cast<int64_t>(sid - 1) * 64;
#pragma unroll
    for (int m = 0; m < 15; ++m) {
      double qm[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) qm[c] = q[4 * m + c];
#pragma unroll
      for (int j = 0; j <= m; ++j) {
#pragma unroll
        for (int c = 0; c < 3; ++c) R[j][c] = __dadd_rn(R[j][c], __dmul_rn(L.sw[m - j], qm[c]));
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) e[c] = q[60 + c];
  }

  const uint32_t* gprev = im.g[(L.pass & 1) ^ 1];
  uint32_t* gnew = im.g[L.pass & 1];
  uint64_t* ot = L.own + (static_cast<int64_t>(sid) << L.own_bits);
  uint32_t* ol = L.own_list + (static_cast<int64_t>(sid) << L.own_bits);
  const unsigned omask = (1u << L.own_bits) - 1u;
  const uint64_t tag = static_cast<uint64_t>(L.tag) << 32;
  double* qe = L.q_end[L.pass & 1] + static_cast<int64_t>(sid) * 64;
  double* qs = L.q_start + static_cast<int64_t>(sid) * 64;
  uint8_t* out = L.chosen + base;
  const uint8_t* uni = im.uni;
  uint32_t* usemin = im.usemin;
  const int warp_steps = __reduce_max_sync(0xffffffffu, static_cast<unsigned>(steps));
  int n_own = 0;
  uint32_t acc = 0;
#pragma unroll 1
  for (int i = 0; i < warp_steps; ++i) {
    const bool on = i < steps;
    const int t = ws + i;
    const int u = i & 15;
    float f[3] = {0.0f, 0.0f, 0.0f};
    unsigned br = 0, bg = 0, bb = 0, key = 0, h = 0;
    int index = 0;
    bool search = false, record = false, from_g = false, booked = false;
    const bool live = t >= begin;
    const bool keyed = on && memo && live;
    if (on) {
      double p[3] = {0.0, 0.0, 0.0};
      if (t + 16 < end) sample<kFloat>(L, base + t + 16, p);
      double v[3];
      switch (u) {
        case 0: Rotate<0>(L.sw, R, e, v, p); break;
        case 1: Rotate<1>(L.sw, R, e, v, p); break;
        case 2: Rotate<2>(L.sw, R, e, v, p); break;
        case 3: Rotate<3>(L.sw, R, e, v, p); break;
        case 4: Rotate<4>(L.sw, R, e, v, p); break;
        case 5: Rotate<5>(L.sw, R, e, v, p); break;
        case 6: Rotate<6>(L.sw, R, e, v, p); break;
        case 7: Rotate<7>(L.sw, R, e, v, p); break;
        case 8: Rotate<8>(L.sw, R, e, v, p); break;
        case 9: Rotate<9>(L.sw, R, e, v, p); break;
        case 10: Rotate<10>(L.sw, R, e, v, p); break;
        case 11: Rotate<11>(L.sw, R, e, v, p); break;
        case 12: Rotate<12>(L.sw, R, e, v, p); break;
        case 13: Rotate<13>(L.sw, R, e, v, p); break;
        case 14: Rotate<14>(L.sw, R, e, v, p); break;
        default: Rotate<15>(L.sw, R, e, v, p); break;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) f[c] = clamp_pixel(v[c]);
      br = byte_dev(f[0]);
      bg = byte_dev(f[1]);
      bb = byte_dev(f[2]);
      key = (br >> 2) | ((bg >> 2) << 6) | ((bb >> 2) << 12);
      // A uniform key's search result (and so its memo value) is fixed by the
      // key: no search, no memo, no bookkeeping.
      const uint8_t uv = __ldg(uni + key);
      const uint32_t gv = keyed ? __ldg(gprev + key) : kNone;  // both loads in flight together
      search = uv == kNotUniform;
      index = uv;
      booked = keyed && search;
      if (booked) {
        if (gv != kNone && static_cast<int>(gv >> 8) < k) {
          index = static_cast<int>(gv & 0xFFu);
          search = false;
          from_g = true;
        } else {
          h = own_hash(key) & omask;
          bool placed = false;
#pragma unroll 1
          for (unsigned probe = 0; probe <= omask; ++probe) {
            const uint64_t ent = ot[h];
            if ((ent & 0xFFFFFFFF00000000ull) != tag) {
              placed = true;  // free slot for this pass: first own use of the key
              break;
            }
            if ((ent & 0xFFFFFFu) == key) {
              index = static_cast<int>((ent >> 24) & 0xFFu);
              search = false;
              break;
            }
            h = (h + 1u) & omask;
          }
          if (search) {
            if (placed) {
              record = true;
            } else {
              atomicExch(L.status, kDevBadPlan);  // table full: the host sizes it to 2x a segment
            }
          }
        }
      }
    }
    // The warp's searches, one target at a time over all 32 lanes.
    unsigned want = __ballot_sync(0xffffffffu, search);
    const int node = search ? tw::descend<false>(P, br, bg, bb, 0u) : 0;
#pragma unroll 1
    while (want) {
      const int src = __ffs(want) - 1;
      want &= want - 1u;
      const int sn = __shfl_sync(0xffffffffu, node, src);
      const float s0 = __shfl_sync(0xffffffffu, f[0], src);
      const float s1 = __shfl_sync(0xffffffffu, f[1], src);
      const float s2 = __shfl_sync(0xffffffffu, f[2], src);
      const int r = tw::search_warp<false>(P, sn, s0, s1, s2, 0.0, lane);
      if (lane == src) index = r;
    }
    if (booked) red_min(gnew + key, (static_cast<uint32_t>(k) << 8) | static_cast<uint32_t>(index));
    if (from_g) red_min(usemin + key, static_cast<uint32_t>(k));
    if (on) {
      if (record) {
        ot[h] = tag | static_cast<uint64_t>(key) | (static_cast<uint64_t>(index) << 24);
        ol[n_own++] = key | (static_cast<uint32_t>(index) << 24);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) e[c] = __dadd_rn(static_cast<double>(f[c]), -errp[c * kMaxPaletteColors + index]);
      if (live) {
        const int q = (t - begin) & 3;
        acc |= static_cast<uint32_t>(index) << (8 * q);
        if (q == 3) {
          *reinterpret_cast<uint32_t*>(out + t - 3) = acc;
          acc = 0;
        } else if (t == end - 1) {
          for (int r = 0; r <= q; ++r) out[t - q + r] = static_cast<uint8_t>(acc >> (8 * r));
        }
        if (t >= end - 16) {
          double* d = qe + 4 * (t - (end - 16));
          d[0] = e[0];
          d[1] = e[1];
          d[2] = e[2];
          d[3] = 0.0;
        }
      } else if (t >= begin - 16) {
        double* d = qs + 4 * (t - (begin - 16));
        d[0] = e[0];
        d[1] = e[1];
        d[2] = e[2];
        d[3] = 0.0;
      }
    }
  }
  if (active && memo) L.own_count[sid] = n_own;
}

template <bool kFloat>
__global__ void __launch_bounds__(128, 3) TswWalkKernel(TswLaunch L) {
  extern __shared__ __align__(16) unsigned char smem[];
  const TswChunk ch = L.chunks[blockIdx.x];
  const TswImage& im = L.images[ch.image];
  const int front = front_of(L, ch.image, im.nsegs);
  if (ch.k0 + ch.count <= front) return;  // the whole chunk is verified (uniform per CTA)
  {
    const int4* src = reinterpret_cast<const int4*>(im.plan);
    int4* dst = reinterpret_cast<int4*>(smem);
    for (int i = threadIdx.x; i < im.plan_smem / 16; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  // Residual-side colours channel-planar (colour i of channel c at
  // c * 256 + i): lanes holding different indices then spread over the banks
  // instead of meeting in the 32-byte palette rows.
  double* errp = reinterpret_cast<double*>(smem + L.plan_smem_max);
  {
    tw::Plan P0;
    P0.bind(smem);
    for (int i = threadIdx.x; i < 3 * kMaxPaletteColors; i += blockDim.x) {
      const int c = i / kMaxPaletteColors, col = i - c * kMaxPaletteColors;
      errp[i] = col < P0.h->count ? P0.rcol<false>(col)[c] : 0.0;
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  // Warps whose segments are all verified or past the image leave together.
  const int warp_k0 = ch.k0 + static_cast<int>(threadIdx.x & ~31u);
  const int warp_end = min(ch.k0 + ch.count, warp_k0 + 32);
  if (warp_end <= front || warp_k0 >= ch.k0 + ch.count) return;
  const int k = ch.k0 + static_cast<int>(threadIdx.x);
  const bool active = static_cast<int>(threadIdx.x) < ch.count && k >= front;
  tw::Plan P;
  P.bind(smem);
  WalkSegment<kFloat>(L, im, P, errp, active ? k : warp_end - 1, active, lane);
}

// G_new = the entries of G_prev that verified segments made; usemin cleared.
__global__ void TswPrepare(TswLaunch L) {
  const int m = blockIdx.y;
  const int key = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= L.n_images || key >= kKeys) return;
  const TswImage& im = L.images[m];
  const int front = front_of(L, m, im.nsegs);
  const uint32_t gv = im.g[(L.pass & 1) ^ 1][key];
  im.g[L.pass & 1][key] = (gv != kNone && static_cast<int>(gv >> 8) < front) ? gv : kNone;
  im.usemin[key] = kNoUser;
}

// The "from G" check, per key.
__global__ void TswVerifyKeys(TswLaunch L) {
  const int m = blockIdx.y;
  const int key = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= L.n_images || key >= kKeys) return;
  const TswImage& im = L.images[m];
  const uint32_t u = im.usemin[key];
  if (u == kNoUser) return;
  const uint32_t gp = im.g[(L.pass & 1) ^ 1][key];
  const uint32_t gn = im.g[L.pass & 1][key];
  if ((gn & 0xFFu) != (gp & 0xFFu) || (gn >> 8) >= u) atomicMin(L.bad[L.pass & 1] + m, static_cast<int>(u));
}

// The queue and own checks, one warp per walked segment.
__global__ void TswVerifySegments(TswLaunch L, int total_segs) {
  const int sid_lo = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (sid_lo >= total_segs) return;
  const int sid = sid_lo;
  // Owner image of this global segment id.
  int lo = 0, hi = L.n_images - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (L.images[mid].first_seg <= sid) lo = mid; else hi = mid - 1;
  }
  const TswImage& im = L.images[lo];
  const int k = sid - im.first_seg;
  if (k >= im.nsegs) return;
  const int front = front_of(L, lo, im.nsegs);
  if (k < front) return;  // verified earlier, not walked
  // Only the image's FIRST failure matters: segments past one already found
  // need no check.  (A relaxed read; a stale value only costs a check.)
  if (k > *reinterpret_cast<volatile const int*>(L.bad[L.pass & 1] + lo)) return;
  bool ok = true;
  if (k > front) {
    // The first walked segment started from a verified predecessor's queue.
    const double* a = (L.pass == 0) ? L.q_start + static_cast<int64_t>(sid) * 64
                                    : L.q_end[(L.pass & 1) ^ 1] + static_cast<int64_t>(sid - 1) * 64;
    const double* b = L.q_end[L.pass & 1] + static_cast<int64_t>(sid - 1) * 64;
    for (int i = lane; i < 64; i += 32) {
      if (__double_as_longlong(a[i]) != __double_as_longlong(b[i])) ok = false;
    }
  }
  if (L.use_cache) {
    const uint32_t* gn = im.g[L.pass & 1];
    const uint32_t* ol = L.own_list + (static_cast<int64_t>(sid) << L.own_bits);
    const int cnt = L.own_count[sid];
    for (int i = lane; i < cnt; i += 32) {
      const uint32_t w = ol[i];
      const uint32_t g = gn[w & 0xFFFFFFu];
      if (static_cast<int>(g >> 8) < k && (g & 0xFFu) != (w >> 24)) ok = false;
    }
  }
  if (!__all_sync(0xffffffffu, ok) && lane == 0) atomicMin(L.bad[L.pass & 1] + lo, k);
}

__global__ void TswScatter(TswLaunch L, int64_t total) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int m = find_image(L.images, L.n_images, i);
  const TswImage& im = L.images[m];
  const int64_t pos = i - im.cx_offset;
  if (pos >= im.n) return;
  const int pix = im.order[pos];
  if (static_cast<unsigned>(pix) >= static_cast<unsigned>(im.n)) return;
  const uint8_t index = L.chosen[i];
  im.indices[pix] = index;
  if (im.rgba_out) {
    const PlanHeader* h = reinterpret_cast<const PlanHeader*>(im.plan);
    const float4 pc = reinterpret_cast<const float4*>(im.plan + h->off_out)[index];
    const float a = load_sample(im.pixels, im.layout, im.row_stride, im.width, pix).w;
    im.rgba_out[pix] = make_float4(pc.x, pc.y, pc.z, a);
  }
}

}  // namespace

std::size_t TswSmemBytes(int plan_smem_max) {
  return static_cast<std::size_t>(plan_smem_max) + 3 * kMaxPaletteColors * sizeof(double);
}

int TswResidentThreads(int plan_smem_max, int sm_count) {
  const int smem = static_cast<int>(TswSmemBytes(plan_smem_max));
  if (AllowMaxSmem(TswWalkKernel<false>) != cudaSuccess) {
    return 0;
  }
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, TswWalkKernel<false>, 128, smem) !=
      cudaSuccess) {
    return 0;
  }
  return blocks * 128 * sm_count;
}

cudaError_t LaunchTswGather(const TswLaunch& L, int64_t total, cudaStream_t s) {
  if (total <= 0) return cudaSuccess;
  TswGather<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(L, total);
  return cudaGetLastError();
}

cudaError_t LaunchTswPrepare(const TswLaunch& L, cudaStream_t s) {
  if (!L.use_cache || L.n_images <= 0) return cudaSuccess;
  TswPrepare<<<dim3(kKeys / 256, L.n_images), 256, 0, s>>>(L);
  return cudaGetLastError();
}

cudaError_t LaunchTswWalk(const TswLaunch& L, cudaStream_t s) {
  if (L.n_chunks <= 0) return cudaSuccess;
  const int smem = static_cast<int>(TswSmemBytes(L.plan_smem_max));
  cudaError_t e;
  if (L.is_float) {
    e = AllowMaxSmem(TswWalkKernel<true>);
    if (e != cudaSuccess) return e;
    TswWalkKernel<true><<<L.n_chunks, L.chunk_threads, smem, s>>>(L);
  } else {
    e = AllowMaxSmem(TswWalkKernel<false>);
    if (e != cudaSuccess) return e;
    TswWalkKernel<false><<<L.n_chunks, L.chunk_threads, smem, s>>>(L);
  }
  return cudaGetLastError();
}

cudaError_t LaunchTswVerify(const TswLaunch& L, int total_segs, cudaStream_t s) {
  if (L.use_cache && L.n_images > 0) {
    TswVerifyKeys<<<dim3(kKeys / 256, L.n_images), 256, 0, s>>>(L);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (total_segs <= 0) return cudaSuccess;
  TswVerifySegments<<<(total_segs + 7) / 8, 256, 0, s>>>(L, total_segs);
  return cudaGetLastError();
}

cudaError_t LaunchTswScatter(const TswLaunch& L, int64_t total, cudaStream_t s) {
  if (total <= 0) return cudaSuccess;
  TswScatter<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(L, total);
  return cudaGetLastError();
}

}  // namespace rdb
