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
//
// Video frames add the decoder's and encoder's byte formats on either side
// (src/rd_riemersma_cpu.cpp:489-516 gather, :711-753 scatter): the gather
// widens 16-bit or YCbCr input to the Q16 float a reader would have produced,
// and the scatter narrows the palette colour straight to rgba64 or planar
// YCbCr, so no RgbaF frame is ever stored.
#include <cuda_runtime.h>

#include "rdb_curve.h"
#include "rdb_device.cuh"
#include "rdb_walk.h"
#include "rdb_walk_thread.cuh"
#include "../../include/rdb.h"

namespace rdb {
namespace {

// swscale's fixed-point BT.601 limited-range YCbCr -> 16-bit RGB, the
// reference's SwsYuvToRgb16 (include/rd_types.h:75-97): luma (y - 16) scaled
// by 9539 * 512, chroma (c - 128) * 512 by the v2r / v2g / u2g / u2b
// coefficients 13075, -6660, -3209 and 16525, all in 32-bit integers (no
// intermediate exceeds 2^31 for 8-bit inputs), shifted down by 14 and
// clamped around the 2^15 offset.
__device__ __forceinline__ float sws_clip16(int acc) {
  const int v = (acc >> 14) + 32768;
  return static_cast<float>(v < 0 ? 0 : (v > 65535 ? 65535 : v));
}
__device__ __forceinline__ float4 ycbcr_to_q16(unsigned y, unsigned cb, unsigned cr) {
  const int luma = (static_cast<int>(y) - 16) * (9539 * 512) + (1 << 13) - (1 << 29);
  const int u = (static_cast<int>(cb) - 128) * 512;
  const int v = (static_cast<int>(cr) - 128) * 512;
  return make_float4(sws_clip16(luma + v * 13075), sws_clip16(luma - v * 6660 - u * 3209),
                     sws_clip16(luma + u * 16525), 65535.0f);
}

// 4:2:0 chroma at full-resolution pixel (x, y): the 2x bilinear
// reconstruction of the reference's 4:2:0 gather (src/rd_blocks_cuda.cu:
// 660-676): weights (2 - ox, ox) x (2 - oy, oy) over the sample at (x/2, y/2)
// and its right / lower neighbours (edge-replicated), rounded, over 4.
__device__ __forceinline__ unsigned chroma420(const unsigned char* plane, int w2, int h2, int x,
                                              int y) {
  const int cx = x >> 1, cy = y >> 1, ox = x & 1, oy = y & 1;
  const int cx1 = cx + 1 < w2 ? cx + 1 : cx;
  const int cy1 = cy + 1 < h2 ? cy + 1 : cy;
  const unsigned char* r0 = plane + static_cast<int64_t>(cy) * w2;
  const unsigned char* r1 = plane + static_cast<int64_t>(cy1) * w2;
  const int top = r0[cx] * (2 - ox) + r0[cx1] * ox;
  const int bot = r1[cx] * (2 - ox) + r1[cx1] * ox;
  return static_cast<unsigned>((top * (2 - oy) + bot * oy + 2) >> 2);
}

// The source value of pixel `pix` as the reader's RgbaF, for every input
// format (src/rd_riemersma_cpu.cpp:496-516: a uint16 widens exactly; absent
// alpha reads 65535).
__device__ __forceinline__ float4 load_wide(const BlockImage& im, int pix) {
  switch (im.layout) {
    case RDB_RGB16: {
      const uint16_t* q = reinterpret_cast<const uint16_t*>(im.pixels) + 3 * static_cast<int64_t>(pix);
      return make_float4(q[0], q[1], q[2], 65535.0f);
    }
    case RDB_RGBA16: {
      const ushort4 q = reinterpret_cast<const ushort4*>(im.pixels)[pix];
      return make_float4(q.x, q.y, q.z, q.w);
    }
    case RDB_YUV444P8: {
      const int64_t plane = static_cast<int64_t>(im.width) * im.height;
      return ycbcr_to_q16(im.pixels[pix], im.pixels[plane + pix], im.pixels[2 * plane + pix]);
    }
    case RDB_YUV420P8: {
      const int64_t plane = static_cast<int64_t>(im.width) * im.height;
      const int w2 = im.width >> 1, h2 = im.height >> 1;
      const int y = pix / im.width, x = pix - y * im.width;
      const unsigned char* cb = im.pixels + plane;
      const unsigned char* cr = cb + static_cast<int64_t>(w2) * h2;
      return ycbcr_to_q16(im.pixels[pix], chroma420(cb, w2, h2, x, y), chroma420(cr, w2, h2, x, y));
    }
    default:
      return load_sample(im.pixels, im.layout, im.row_stride, im.width, pix);
  }
}

// The encoder-format store of one pixel whose Q16 colour is (r, g, b, a):
// rgba64 takes the uint16 of each float (src/rd_riemersma_cpu.cpp:746-752);
// planar YCbCr takes BT.601 limited range of each channel's top 8 bits
// (:719-731).
__device__ __forceinline__ void store_raw(const BlockImage& im, int pix, float r, float g, float b,
                                          float a) {
  if (im.out_format == RDB_RGBA16) {
    reinterpret_cast<ushort4*>(im.raw_out)[pix] =
        make_ushort4(static_cast<uint16_t>(r), static_cast<uint16_t>(g), static_cast<uint16_t>(b),
                     static_cast<uint16_t>(a));
    return;
  }
  const int r8 = static_cast<int>(r) >> 8;
  const int g8 = static_cast<int>(g) >> 8;
  const int b8 = static_cast<int>(b) >> 8;
  const int y = ((66 * r8 + 129 * g8 + 25 * b8 + 128) >> 8) + 16;
  const int u = ((-38 * r8 - 74 * g8 + 112 * b8 + 128) >> 8) + 128;
  const int v = ((112 * r8 - 94 * g8 - 18 * b8 + 128) >> 8) + 128;
  const int64_t plane = static_cast<int64_t>(im.width) * im.height;
  im.raw_out[pix] = static_cast<unsigned char>(min(max(y, 0), 255));
  im.raw_out[plane + pix] = static_cast<unsigned char>(min(max(u, 0), 255));
  im.raw_out[2 * plane + pix] = static_cast<unsigned char>(min(max(v, 0), 255));
}

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

// The block, image and length of global block gb (the image found by binary
// search over the images' first blocks).
struct BlockRef {
  const BlockImage* im;
  int begin;  // first position of the block in its image's list
  int len;    // positions in the block (the last block of an image may be short)
};
__device__ __forceinline__ BlockRef block_ref(const BlockLaunch& L, int64_t gb) {
  const int m = find_image(L.images, L.n_images, gb);
  const BlockImage& im = L.images[m];
  const int b = static_cast<int>(gb - im.first_block);
  BlockRef r;
  r.im = &im;
  r.begin = b * L.block;
  r.len = min(L.block, im.n - r.begin);
  return r;
}

// The pixel the list visits at position pos: the appended origin last.
__device__ __forceinline__ int list_pixel(const BlockLaunch& L, const BlockImage& im, int pos) {
  int pix = (pos == im.n - 1) ? 0 : im.order[pos];
  if (static_cast<unsigned>(pix) >= static_cast<unsigned>(im.width * im.height)) {
    atomicExch(L.status, kDevBadItem);
    pix = 0;
  }
  return pix;
}

// Packed samples: one thread per (group, 4 positions, lane), lane fastest, so
// a warp writes 512 contiguous bytes; positions past a block's end are zero.
__global__ void BlockGatherPacked(BlockLaunch L, int64_t quads) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= quads) return;
  const int l = static_cast<int>(i & 31);
  const int64_t row = i >> 5;  // g * bpad/4 + t/4
  const int q4 = L.bpad >> 2;
  const int64_t g = row / q4;
  const int t0 = static_cast<int>(row - g * q4) * 4;
  const int64_t gb = g * 32 + l;
  uint4 w = make_uint4(0u, 0u, 0u, 0u);
  if (gb < L.total_blocks) {
    const BlockRef r = block_ref(L, gb);
    uint32_t v[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (t0 + k < r.len) {
        const int pix = list_pixel(L, *r.im, r.begin + t0 + k);
        v[k] = pack_sample(r.im->pixels, r.im->layout, r.im->row_stride, r.im->width, pix);
      }
    }
    w = make_uint4(v[0], v[1], v[2], v[3]);
  }
  reinterpret_cast<uint4*>(L.cx)[i] = w;
}

// Widened (float4) samples: one thread per (group, position, lane).
__global__ void BlockGatherWide(BlockLaunch L, int64_t cells) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= cells) return;
  const int l = static_cast<int>(i & 31);
  const int64_t row = i >> 5;  // g * bpad + t
  const int64_t g = row / L.bpad;
  const int t = static_cast<int>(row - g * L.bpad);
  const int64_t gb = g * 32 + l;
  float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
  if (gb < L.total_blocks) {
    const BlockRef r = block_ref(L, gb);
    if (t < r.len) v = load_wide(*r.im, list_pixel(L, *r.im, r.begin + t));
  }
  reinterpret_cast<float4*>(L.cx)[i] = v;
}

// Channel c of AssociateAlphaPixel (rd_types.h:179-192) for a packed RGBA8
// sample: the Q16 value is v * 257, exact in double.
template <bool kAssoc>
__device__ __forceinline__ void unpack8(uint32_t w, double (&p)[4]) {
  const double r = static_cast<double>((w & 0xFFu) * 257u);
  const double g = static_cast<double>(((w >> 8) & 0xFFu) * 257u);
  const double b = static_cast<double>(((w >> 16) & 0xFFu) * 257u);
  const unsigned a8 = w >> 24;
  p[0] = r;
  p[1] = g;
  p[2] = b;
  if (kAssoc) {
    const double a = static_cast<double>(a8 * 257u);
    p[3] = a;
    if (a8 != 255u) {
      const double alpha = __dmul_rn(kQuantumScale, a);
      p[0] = __dmul_rn(alpha, r);
      p[1] = __dmul_rn(alpha, g);
      p[2] = __dmul_rn(alpha, b);
    }
  }
}

template <bool kAssoc>
__device__ __forceinline__ void unpackf(float4 s, double (&p)[4]) {
  associate_sample(kAssoc, s, p[0], p[1], p[2], p[3]);
}

// One step of the running sums with the rotation fixed at compile time:
// pixel t (slot U) takes its last term, the 15 pixels after it take theirs,
// and slot U is refilled with pixel t+16.
template <int U, int C>
__device__ __forceinline__ void RotateSums(const BlockLaunch& L, double (&R)[16][C],
                                           const double (&e)[C], double (&v)[C],
                                           const double (&p)[4]) {
#pragma unroll
  for (int k = 0; k < C; ++k) v[k] = __dadd_rn(R[U][k], __dmul_rn(L.sw[15], e[k]));
#pragma unroll
  for (int jj = 1; jj < 16; ++jj) {
#pragma unroll
    for (int k = 0; k < C; ++k) {
      R[(U + jj) & 15][k] = __dadd_rn(R[(U + jj) & 15][k], __dmul_rn(L.sw[15 - jj], e[k]));
    }
  }
#pragma unroll
  for (int k = 0; k < C; ++k) R[U][k] = p[k];
}

__device__ __forceinline__ uint32_t pick(const uint4& q, int k) {
  return k == 0 ? q.x : (k == 1 ? q.y : (k == 2 ? q.z : q.w));
}

// One block of `len` positions, zeroed queue, no memo.  Only the register
// rotation is unrolled (16 switch cases of FP64 work); the lookup is written
// once, so the loop stays in the instruction cache.  The lookup takes the
// key's survivors from the candidate table when the palette has one (the
// full descent and search only for keys the table does not cover).
template <bool kAssoc, bool kFloat>
__device__ __forceinline__ void WalkBlock(const BlockLaunch& L, const tw::Plan& P, int64_t gb,
                                          const BlockRef& ref) {
  const int64_t g = gb >> 5;
  const int lane = static_cast<int>(gb & 31);
  const int len = ref.len;
  constexpr int C = kAssoc ? 4 : 3;
  const uint4* cx4 = reinterpret_cast<const uint4*>(L.cx) + g * (L.bpad >> 2) * 32 + lane;
  const float4* cxf = reinterpret_cast<const float4*>(L.cx) + g * L.bpad * 32 + lane;
  uint4* out4 = reinterpret_cast<uint4*>(L.chosen) + g * (L.bpad >> 4) * 32 + lane;
  const int bpad = L.bpad;
  double R[16][C];
  double e[C];
#pragma unroll
  for (int k = 0; k < C; ++k) e[k] = 0.0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint4 w = make_uint4(0u, 0u, 0u, 0u);
    if (!kFloat) w = cx4[q * 32];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      double p[4] = {0.0, 0.0, 0.0, 0.0};
      if (kFloat) unpackf<kAssoc>(cxf[(4 * q + k) * 32], p); else unpack8<kAssoc>(pick(w, k), p);
#pragma unroll
      for (int c = 0; c < C; ++c) R[4 * q + k][c] = p[c];
    }
  }
  const int b = ref.begin / L.block;            // block index within its image
  const bool has_next = b + 1 < ref.im->nblocks;
  if (L.q_in && b > 0) {
    // Start from the predecessor's end queue q[0..15] (oldest first): pixel j
    // holds p + sum_{m=j}^{14} w_{m-j} q[m] in ascending m, and q[15] is the
    // pending residual.
    const double* q = L.q_in + (gb - 1) * 64;
#pragma unroll
    for (int m = 0; m < 15; ++m) {
#pragma unroll
      for (int j = 0; j <= m; ++j) {
#pragma unroll
        for (int c = 0; c < C; ++c) R[j][c] = __dadd_rn(R[j][c], __dmul_rn(L.sw[m - j], q[4 * m + c]));
      }
    }
#pragma unroll
    for (int c = 0; c < C; ++c) e[c] = q[60 + c];
  }
  double* qo = L.q_out ? L.q_out + gb * 64 : nullptr;
  const double* qp = (L.q_in && has_next) ? L.q_in + gb * 64 : nullptr;
  bool changed = false;
  uint4 ahead = make_uint4(0u, 0u, 0u, 0u);  // packed samples t+16 .. t+19
  uint32_t acc[4] = {0u, 0u, 0u, 0u};
  int u = 0;
#pragma unroll 1
  for (int t = 0; t < len; ++t) {
    double p[4] = {0.0, 0.0, 0.0, 0.0};
    if (t + 16 < bpad) {
      if (kFloat) {
        unpackf<kAssoc>(cxf[(t + 16) * 32], p);
      } else {
        if ((t & 3) == 0) ahead = cx4[((t + 16) >> 2) * 32];
        unpack8<kAssoc>(pick(ahead, t & 3), p);
      }
    }
    double v[C];
    switch (u) {
      case 0: RotateSums<0, C>(L, R, e, v, p); break;
      case 1: RotateSums<1, C>(L, R, e, v, p); break;
      case 2: RotateSums<2, C>(L, R, e, v, p); break;
      case 3: RotateSums<3, C>(L, R, e, v, p); break;
      case 4: RotateSums<4, C>(L, R, e, v, p); break;
      case 5: RotateSums<5, C>(L, R, e, v, p); break;
      case 6: RotateSums<6, C>(L, R, e, v, p); break;
      case 7: RotateSums<7, C>(L, R, e, v, p); break;
      case 8: RotateSums<8, C>(L, R, e, v, p); break;
      case 9: RotateSums<9, C>(L, R, e, v, p); break;
      case 10: RotateSums<10, C>(L, R, e, v, p); break;
      case 11: RotateSums<11, C>(L, R, e, v, p); break;
      case 12: RotateSums<12, C>(L, R, e, v, p); break;
      case 13: RotateSums<13, C>(L, R, e, v, p); break;
      case 14: RotateSums<14, C>(L, R, e, v, p); break;
      default: RotateSums<15, C>(L, R, e, v, p); break;
    }
    u = (u + 1) & 15;
    float f[4];
#pragma unroll
    for (int k = 0; k < C; ++k) f[k] = clamp_pixel(v[k]);
    const unsigned br = byte_dev(f[0]), bg = byte_dev(f[1]), bb = byte_dev(f[2]);
    int index;
    if (!kAssoc && L.cand) {
      const uint32_t c = __ldg(L.cand + ((br >> 2) | ((bg >> 2) << 6) | ((bb >> 2) << 12)));
      const unsigned s0 = c & 0xFFu, s1 = (c >> 8) & 0xFFu;
      if (s0 == s1) {
        index = P.seq[s0];
      } else if (s0 < s1) {
        index = tw::search_survivors(P, c, f[0], f[1], f[2]);
      } else {
        index = tw::search<false>(P, tw::descend<false>(P, br, bg, bb, 0u), f[0], f[1], f[2], 0.0);
      }
    } else {
      const unsigned ba = kAssoc ? byte_dev(f[C - 1]) : 0u;
      const int node = tw::descend<kAssoc>(P, br, bg, bb, ba);
      double tr = f[0], tg = f[1], tb = f[2], ta = 0.0;
      if (kAssoc) {
        ta = f[3];
        const double beta = __dmul_rn(kQuantumScale, ta);
        tr = __dmul_rn(beta, tr);
        tg = __dmul_rn(beta, tg);
        tb = __dmul_rn(beta, tb);
      }
      index = tw::search<kAssoc>(P, node, tr, tg, tb, ta);
    }
    const double* rc = P.rcol<kAssoc>(index);
#pragma unroll
    for (int k = 0; k < C; ++k) e[k] = __dadd_rn(static_cast<double>(f[k]), -rc[k]);
    if (qo && t >= len - 16) {
      const int at = 4 * (t - (len - 16));
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const double v = c < C ? e[c < C ? c : 0] : 0.0;
        if (qp) changed |= __double_as_longlong(qp[at + c]) != __double_as_longlong(v);
        qo[at + c] = v;
      }
    }
    const int q = (t >> 2) & 3;
    const uint32_t bits = static_cast<uint32_t>(index) << (8 * (t & 3));
    if (q == 0) acc[0] |= bits; else if (q == 1) acc[1] |= bits; else if (q == 2) acc[2] |= bits; else acc[3] |= bits;
    if ((t & 15) == 15 || t == len - 1) {
      out4[(t >> 4) * 32] = make_uint4(acc[0], acc[1], acc[2], acc[3]);
      acc[0] = acc[1] = acc[2] = acc[3] = 0u;
    }
  }
  if (changed && L.changed) atomicAdd(L.changed, 1);
}
// kThreads per CTA (a multiple of 32: each warp is one group of 32 blocks)
// and kMinCtas resident per SM -- the register budget -- are the launch shape
// the tuner picks among (BlockWalkShape); every shape computes the same bytes.
template <bool kAssoc, bool kFloat, int kThreads, int kMinCtas>
__global__ void __launch_bounds__(kThreads, kMinCtas) BlockWalkKernel(BlockLaunch L) {
  extern __shared__ __align__(16) unsigned char smem[];
  {
    const int4* src = reinterpret_cast<const int4*>(L.plan);
    int4* dst = reinterpret_cast<int4*>(smem);
    for (int i = threadIdx.x; i < L.plan_smem / 16; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int64_t gb = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (gb >= L.total_blocks) return;
  tw::Plan P;
  P.bind(smem);
  const BlockRef r = block_ref(L, gb);
  WalkBlock<kAssoc, kFloat>(L, P, gb, r);
}

template <bool kAssoc, bool kFloat, int kThreads, int kMinCtas>
cudaError_t LaunchShape(const BlockLaunch& L, cudaStream_t stream) {
  cudaError_t e = AllowMaxSmem(BlockWalkKernel<kAssoc, kFloat, kThreads, kMinCtas>);
  if (e != cudaSuccess) return e;
  const unsigned g2 = static_cast<unsigned>((L.total_blocks + kThreads - 1) / kThreads);
  BlockWalkKernel<kAssoc, kFloat, kThreads, kMinCtas><<<g2, kThreads, L.plan_smem, stream>>>(L);
  return cudaGetLastError();
}

// The shapes: (threads, CTAs per SM) -- the same 128-register budget in three
// CTA sizes, and a larger register budget (fewer resident warps, no spills).
constexpr int kShapes[kBlockWalkShapes][2] = {{128, 4}, {256, 2}, {64, 8}, {128, 3}};

template <bool kAssoc, bool kFloat>
cudaError_t LaunchWalk(const BlockLaunch& L, int shape, cudaStream_t stream) {
  // Alpha palettes carry a fourth channel: one CTA less per SM at each size.
  switch (shape) {
    case 1: return LaunchShape<kAssoc, kFloat, 256, kAssoc ? 1 : 2>(L, stream);
    case 2: return LaunchShape<kAssoc, kFloat, 64, kAssoc ? 6 : 8>(L, stream);
    case 3: return LaunchShape<kAssoc, kFloat, 128, kAssoc ? 2 : 3>(L, stream);
    default: return LaunchShape<kAssoc, kFloat, 128, kAssoc ? 3 : 4>(L, stream);
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
    if (L.pos_offset[mid] <= i) lo = mid; else hi = mid - 1;
  }
  const BlockImage& im = L.images[lo];
  const int64_t pos = i - L.pos_offset[lo];
  if (pos >= im.n) return;
  const int64_t npix = static_cast<int64_t>(im.width) * im.height;
  if (pos == 0 && im.n > 1) {
    // This thread also fills the unvisited cell (2^L-1, 0) when it is inside
    // the image, i.e. when the list is one shorter than pixels + 1: the
    // source value, in every output asked for (src/rd_riemersma_cpu.cpp:
    // 776-801 for the encoder formats).
    if (im.n == npix && (im.rgba_out || im.raw_out)) {
      const int gap = im.width - 1;
      const float4 src = load_wide(im, gap);
      if (im.rgba_out) im.rgba_out[gap] = src;
      if (im.raw_out) store_raw(im, gap, src.x, src.y, src.z, src.w);
    }
    return;
  }
  int pix = (pos == im.n - 1) ? 0 : im.order[pos];
  if (static_cast<unsigned>(pix) >= static_cast<unsigned>(im.width * im.height)) return;
  const int64_t gb = im.first_block + pos / L.block;
  const int64_t t = pos - (gb - im.first_block) * L.block;
  const uint8_t index =
      L.chosen[(((gb >> 5) * (L.bpad >> 4) + (t >> 4)) * 32 + (gb & 31)) * 16 + (t & 15)];
  if (im.indices) im.indices[pix] = index;
  if (im.rgba_out || im.raw_out) {
    // The colour as clamp_to_quantum's floats; alpha from the palette when it
    // associates alpha, else the source's, which the scatter leaves in place.
    const PlanHeader* h = reinterpret_cast<const PlanHeader*>(L.plan);
    const float4 pc = reinterpret_cast<const float4*>(L.plan + h->off_out)[index];
    const float a = h->assoc ? pc.w : load_wide(im, pix).w;
    if (im.rgba_out) im.rgba_out[pix] = make_float4(pc.x, pc.y, pc.z, a);
    if (im.raw_out) store_raw(im, pix, pc.x, pc.y, pc.z, a);
  }
}

__global__ void ChosenLinear(BlockLaunch L, int64_t total, uint8_t* out) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= total) return;
  int lo = 0, hi = L.n_images - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (L.pos_offset[mid] <= i) lo = mid; else hi = mid - 1;
  }
  const BlockImage& im = L.images[lo];
  const int64_t pos = i - L.pos_offset[lo];
  const int64_t gb = im.first_block + pos / L.block;
  const int64_t t = pos - (gb - im.first_block) * L.block;
  out[i] = L.chosen[(((gb >> 5) * (L.bpad >> 4) + (t >> 4)) * 32 + (gb & 31)) * 16 + (t & 15)];
}

__global__ void SourceFill(BlockImage im) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<int64_t>(im.width) * im.height) return;
  const int pix = static_cast<int>(i);
  const float4 src = load_wide(im, pix);
  if (im.rgba_out) im.rgba_out[pix] = src;
  if (im.raw_out) store_raw(im, pix, src.x, src.y, src.z, src.w);
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

cudaError_t LaunchSourceFill(const BlockImage& im, cudaStream_t stream) {
  const int64_t n = static_cast<int64_t>(im.width) * im.height;
  if (n <= 0 || (!im.rgba_out && !im.raw_out)) return cudaSuccess;
  SourceFill<<<static_cast<unsigned>((n + 255) / 256), 256, 0, stream>>>(im);
  return cudaGetLastError();
}

cudaError_t LaunchBlockChosenLinear(const BlockLaunch& L, int64_t total_positions, uint8_t* out,
                                    cudaStream_t stream) {
  if (total_positions <= 0) return cudaSuccess;
  ChosenLinear<<<static_cast<unsigned>((total_positions + 255) / 256), 256, 0, stream>>>(
      L, total_positions, out);
  return cudaGetLastError();
}

cudaError_t LaunchBlockGather(const BlockLaunch& L, cudaStream_t stream) {
  if (L.total_blocks <= 0) return cudaSuccess;
  const int64_t cells = (L.total_blocks + 31) / 32 * 32 * L.bpad;  // positions in the scratch
  if (L.is_float) {
    BlockGatherWide<<<static_cast<unsigned>((cells + 255) / 256), 256, 0, stream>>>(L, cells);
  } else {
    BlockGatherPacked<<<static_cast<unsigned>((cells / 4 + 255) / 256), 256, 0, stream>>>(L, cells / 4);
  }
  return cudaGetLastError();
}

cudaError_t LaunchBlockWalkOnly(const BlockLaunch& L, cudaStream_t stream, int shape) {
  if (L.total_blocks <= 0) return cudaSuccess;
  if (shape < 0 || shape >= kBlockWalkShapes) shape = 0;
  return L.assoc ? (L.is_float ? LaunchWalk<true, true>(L, shape, stream) : LaunchWalk<true, false>(L, shape, stream))
                 : (L.is_float ? LaunchWalk<false, true>(L, shape, stream)
                               : LaunchWalk<false, false>(L, shape, stream));
}

void BlockWalkShape(int shape, bool assoc, int* threads, int* min_ctas) {
  if (shape < 0 || shape >= kBlockWalkShapes) shape = 0;
  *threads = kShapes[shape][0];
  *min_ctas = kShapes[shape][1] - (assoc ? (shape == 2 ? 2 : 1) : 0);
}

cudaError_t LaunchBlockScatter(const BlockLaunch& L, int64_t total_positions, cudaStream_t stream) {
  if (total_positions <= 0) return cudaSuccess;
  BlockScatter<<<static_cast<unsigned>((total_positions + 255) / 256), 256, 0, stream>>>(L, total_positions);
  return cudaGetLastError();
}

cudaError_t LaunchBlockWalk(const BlockLaunch& L, int64_t total_positions, cudaStream_t stream, int shape) {
  if (total_positions <= 0 || L.total_blocks <= 0) return cudaSuccess;
  cudaError_t e;
  if ((e = LaunchBlockGather(L, stream)) != cudaSuccess) return e;
  if ((e = LaunchBlockWalkOnly(L, stream, shape)) != cudaSuccess) return e;
  return LaunchBlockScatter(L, total_positions, stream);
}

}  // namespace rdb
