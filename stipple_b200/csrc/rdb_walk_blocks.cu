// rdb_walk_blocks.cu -- the block-parallel engine, bit-exact with the
// reference's host block walk.
//
// Reference: src/rd_riemersma_cpu.cpp:477-805 (RiemersmaBlocksCpu).  The
// block-mode list (BuildCurveIndex) is cut into blocks of B consecutive
// positions; each block is walked from a zeroed queue with NO memo (every
// lookup descends and searches), and each pixel takes the index of the LAST
// position that visits it (the owner map) -- only the origin is visited
// twice, first at position 0 and last at the final position.  The one cell
// the list never reaches keeps its source value.
//
// Three passes per launch:
//   gather   curve-ordered packed samples (coalesced writes, one 32-bit word
//            per position for 8-bit input)
//   walk     one thread per block; the 16 running sums of the upcoming pixels
//            live in registers under a 16-way unroll so that the register
//            names rotate instead of moving data; the palette plan is staged
//            in shared memory
//   scatter  index per pixel through the order table, skipping position 0
#include <cuda_runtime.h>

#include "rdb_curve.h"
#include "rdb_device.cuh"
#include "rdb_walk.h"

namespace rdb {
namespace {

struct V4 {
  double r, g, b, a;
};

__device__ __forceinline__ int find_image(const BlockImage* imgs, int n, int64_t gb) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (imgs[mid].first_block <= gb) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ uint32_t pack_sample(const unsigned char* img, int layout,
                                                int64_t stride, int width, int pix) {
  const int y = pix / width;
  const int x = pix - y * width;
  const unsigned char* row = img + static_cast<int64_t>(y) * stride;
  if (layout == 4) return reinterpret_cast<const uint32_t*>(row)[x];
  const unsigned char* q = row + 3 * x;
  return static_cast<uint32_t>(q[0]) | (static_cast<uint32_t>(q[1]) << 8) |
         (static_cast<uint32_t>(q[2]) << 16) | 0xFF000000u;
}

// One thread per curve position of every image.
__global__ void BlockGather(BlockLaunch L, int64_t total) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= total) return;
  // Images are laid out back to back in cx; find the owner by offset.
  int lo = 0, hi = L.n_images - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (L.cx_offset[mid] <= i) lo = mid; else hi = mid - 1;
  }
  const BlockImage& im = L.images[lo];
  const int64_t pos = i - L.cx_offset[lo];
  if (pos >= im.n) return;  // alignment padding
  int pix = (pos == im.n - 1) ? 0 : im.order[pos];
  if (static_cast<unsigned>(pix) >= static_cast<unsigned>(im.width * im.height)) {
    atomicExch(L.status, kDevBadItem);
    pix = 0;
  }
  if (im.layout == 16) {
    const float4 s = load_sample(im.pixels, 16, im.row_stride, im.width, pix);
    reinterpret_cast<float4*>(L.cx)[i] = s;
  } else {
    L.cx[i] = pack_sample(im.pixels, im.layout, im.row_stride, im.width, pix);
  }
}

__device__ __forceinline__ V4 unpack(int assoc, uint32_t w) {
  float4 s = make_float4(static_cast<float>(w & 0xFFu) * 257.0f,
                         static_cast<float>((w >> 8) & 0xFFu) * 257.0f,
                         static_cast<float>((w >> 16) & 0xFFu) * 257.0f,
                         static_cast<float>(w >> 24) * 257.0f);
  V4 v;
  associate_sample(assoc, s, v.r, v.g, v.b, v.a);
  return v;
}

template <bool kAssoc, bool kFloat>
__device__ __forceinline__ V4 sample_at(const BlockLaunch& L, int64_t i) {
  if (kFloat) {
    V4 v;
    associate_sample(kAssoc, reinterpret_cast<const float4*>(L.cx)[i], v.r, v.g, v.b, v.a);
    return v;
  }
  return unpack(kAssoc, L.cx[i]);
}

template <bool kAssoc, bool kFloat>
__device__ void WalkBlock(const BlockLaunch& L, const PlanView& P, int64_t base, int begin,
                          int end) {
  double sw[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) sw[k] = L.sw[k];
  V4 R[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    R[j] = (begin + j < end) ? sample_at<kAssoc, kFloat>(L, base + begin + j)
                             : V4{0.0, 0.0, 0.0, 0.0};
  }
  V4 e{0.0, 0.0, 0.0, 0.0};
  for (int g0 = begin; g0 < end; g0 += 16) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int t = g0 + u;
      if (t < end) {
        V4 v;
        v.r = __dadd_rn(R[u].r, __dmul_rn(sw[15], e.r));
        v.g = __dadd_rn(R[u].g, __dmul_rn(sw[15], e.g));
        v.b = __dadd_rn(R[u].b, __dmul_rn(sw[15], e.b));
        if (kAssoc) v.a = __dadd_rn(R[u].a, __dmul_rn(sw[15], e.a));
#pragma unroll
        for (int j = 1; j < 16; ++j) {
          V4& s = R[(u + j) & 15];
          s.r = __dadd_rn(s.r, __dmul_rn(sw[15 - j], e.r));
          s.g = __dadd_rn(s.g, __dmul_rn(sw[15 - j], e.g));
          s.b = __dadd_rn(s.b, __dmul_rn(sw[15 - j], e.b));
          if (kAssoc) s.a = __dadd_rn(s.a, __dmul_rn(sw[15 - j], e.a));
        }
        R[u] = (t + 16 < end) ? sample_at<kAssoc, kFloat>(L, base + t + 16)
                              : V4{0.0, 0.0, 0.0, 0.0};
        const float fr = clamp_pixel(v.r);
        const float fg = clamp_pixel(v.g);
        const float fb = clamp_pixel(v.b);
        const float fa = kAssoc ? clamp_pixel(v.a) : 0.0f;
        const int node = plan_descend(P, byte_dev(fr), byte_dev(fg), byte_dev(fb),
                                      kAssoc ? byte_dev(fa) : 0u);
        const Target tg = make_target(kAssoc, static_cast<double>(fr), static_cast<double>(fg),
                                      static_cast<double>(fb), static_cast<double>(fa));
        const int index = plan_search_serial(P, node, tg);
        L.chosen[base + t] = static_cast<uint8_t>(index);
        const double* rc = P.rcol(index);
        e.r = __dadd_rn(static_cast<double>(fr), -rc[0]);
        e.g = __dadd_rn(static_cast<double>(fg), -rc[1]);
        e.b = __dadd_rn(static_cast<double>(fb), -rc[2]);
        if (kAssoc) e.a = __dadd_rn(static_cast<double>(fa), -rc[3]);
      }
    }
  }
}

__global__ void __launch_bounds__(128) BlockWalkKernel(BlockLaunch L) {
  extern __shared__ __align__(16) unsigned char smem[];
  {
    const int4* src = reinterpret_cast<const int4*>(L.plan);
    int4* dst = reinterpret_cast<int4*>(smem);
    for (int i = threadIdx.x; i < L.plan_smem / 16; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int64_t gb = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (gb >= L.total_blocks) return;
  PlanView P;
  P.bind(smem);
  const int im = find_image(L.images, L.n_images, gb);
  const BlockImage& I = L.images[im];
  const int b = static_cast<int>(gb - I.first_block);
  const int begin = b * L.block;
  const int end = min(begin + L.block, I.n);
  const int64_t base = L.cx_offset[im];
  const bool is_float = I.layout == 16;
  if (P.assoc) {
    if (is_float) WalkBlock<true, true>(L, P, base, begin, end);
    else WalkBlock<true, false>(L, P, base, begin, end);
  } else {
    if (is_float) WalkBlock<false, true>(L, P, base, begin, end);
    else WalkBlock<false, false>(L, P, base, begin, end);
  }
}

// Owner-map scatter (src/rd_riemersma_cpu.cpp:698-710): position 0 is the
// origin's first visit and the final position its last, so every position
// but 0 owns its pixel.  The unvisited cell, if any, is copied from the
// source into the RgbaF output and left alone in the index map.
__global__ void BlockScatter(BlockLaunch L, int64_t total) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= total) return;
  int lo = 0, hi = L.n_images - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (L.cx_offset[mid] <= i) lo = mid; else hi = mid - 1;
  }
  const BlockImage& im = L.images[lo];
  const int64_t pos = i - L.cx_offset[lo];
  if (pos >= im.n) return;
  const int64_t npix = static_cast<int64_t>(im.width) * im.height;
  if (pos == 0 && im.n > 1) {
    // This thread also fills the unvisited cell (2^L-1, 0) when it is inside
    // the image, i.e. when the list is one shorter than pixels + 1.
    if (im.n == npix && im.rgba_out) {
      const int gap = im.width - 1;
      im.rgba_out[gap] = load_sample(im.pixels, im.layout, im.row_stride, im.width, gap);
    }
    return;
  }
  int pix = (pos == im.n - 1) ? 0 : im.order[pos];
  if (static_cast<unsigned>(pix) >= static_cast<unsigned>(im.width * im.height)) return;
  const uint8_t index = L.chosen[i];
  im.indices[pix] = index;
  if (im.rgba_out) {
    const PlanHeader* h = reinterpret_cast<const PlanHeader*>(L.plan);
    const float4 pc = reinterpret_cast<const float4*>(L.plan + h->off_out)[index];
    const float a = h->assoc ? pc.w
                             : load_sample(im.pixels, im.layout, im.row_stride, im.width, pix).w;
    im.rgba_out[pix] = make_float4(pc.x, pc.y, pc.z, a);
  }
}

__global__ void CopySource(const unsigned char* pixels, int64_t stride, int width, int height,
                           int layout, float4* out) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<int64_t>(width) * height) return;
  out[i] = load_sample(pixels, layout, stride, width, static_cast<int>(i));
}

}  // namespace

cudaError_t LaunchCopySource(const unsigned char* pixels, int64_t stride, int width, int height,
                             int layout, float4* out, cudaStream_t stream) {
  const int64_t n = static_cast<int64_t>(width) * height;
  if (n <= 0) return cudaSuccess;
  CopySource<<<static_cast<unsigned>((n + 255) / 256), 256, 0, stream>>>(pixels, stride, width,
                                                                        height, layout, out);
  return cudaGetLastError();
}

cudaError_t LaunchBlockWalk(const BlockLaunch& L, int64_t total_positions, cudaStream_t stream) {
  if (total_positions <= 0 || L.total_blocks <= 0) return cudaSuccess;
  const unsigned g1 = static_cast<unsigned>((total_positions + 255) / 256);
  BlockGather<<<g1, 256, 0, stream>>>(L, total_positions);
  cudaError_t e = cudaFuncSetAttribute(BlockWalkKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       L.plan_smem);
  if (e != cudaSuccess) return e;
  const unsigned g2 = static_cast<unsigned>((L.total_blocks + 127) / 128);
  BlockWalkKernel<<<g2, 128, L.plan_smem, stream>>>(L);
  BlockScatter<<<g1, 256, 0, stream>>>(L, total_positions);
  return cudaGetLastError();
}

}  // namespace rdb
