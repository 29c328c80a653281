// rdb_tsw.cu -- kernels of the thread-walker segmented walk (see rdb_tsw.h).
//
// The per-position arithmetic is the block engine's thread walker
// (rdb_walk_thread.cuh): running sums of the 16 upcoming pixels in
// registers, rotated by a 16-way switch, the weights as constant operands,
// FP64 in the reference's operation order (src/rd_riemersma_cpu.cpp:39-113).
// What differs from a block is the start state (a carried or warmed-up
// queue instead of zeros) and the memo (rdb_tsw.h).
#include <cuda_runtime.h>

#include <algorithm>

#include "rdb_device.cuh"
#include "rdb_tsw.h"
#include "rdb_uniform.h"
#include "rdb_uniform_alpha.cuh"
#include "rdb_walk_thread.cuh"

namespace rdb {
namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr uint32_t kNoUser = 0xFFFFFFFFu;
constexpr int kKeys = 1 << 18;
constexpr int kFillBlocks = 64;  // per image: the classification kernel's grid

__device__ __forceinline__ int front_of(const TswLaunch& L, int image, int nsegs) {
  const int b = L.bad[(L.pass & 1) ^ 1][image];
  return b < nsegs ? b : nsegs;
}

// Segments image `image` walks beyond its front this pass (0 = all).
__device__ __forceinline__ int window_of(const TswLaunch& L, int image) {
  return L.win ? L.win[image] : L.window;
}
__device__ __forceinline__ bool windowed(const TswLaunch& L) { return L.window > 0 || L.win != nullptr; }

// The interleaved deal of TswLaunch::spread: CTA c of the g CTAs that take an
// image's segments walks base + s * g + c in its slot s (slots numbered lane
// by lane across the CTA's warps), base being the
// front's chunk start.  One image: the whole grid.  Several (per-image
// windows): the image's first g chunks, g covering its window (one chunk
// more, since the front need not sit on a chunk boundary).  False when this
// CTA takes none.
struct Deal {
  int base, g, c;
};
__device__ __forceinline__ bool deal_of(const TswLaunch& L, const TswChunk& ch, int front, int wnd,
                                        int nsegs, Deal* d) {
  const int ct = L.chunk_threads;
  d->base = front / ct * ct;
  if (L.win) {
    d->c = ch.k0 / ct;
    d->g = min((nsegs - d->base + ct - 1) / ct, (wnd + ct - 1) / ct + 1);
  } else {
    d->c = static_cast<int>(blockIdx.x);
    d->g = static_cast<int>(gridDim.x);
  }
  return d->c < d->g;
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

// One curve position's sample as the walk sees it (AssociateAlphaPixel,
// rd_types.h:179-192, when the palette associates alpha).
template <bool kFloat, int C>
__device__ __forceinline__ void sample(const TswLaunch& L, int64_t at, double (&p)[C]) {
  if (kFloat) {
    const float4 s = reinterpret_cast<const float4*>(L.cx)[at];
    double a4[4];
    associate_sample(C == 4, s, a4[0], a4[1], a4[2], a4[3]);
#pragma unroll
    for (int c = 0; c < C; ++c) p[c] = a4[c];
  } else {
    const uint32_t w = reinterpret_cast<const uint32_t*>(L.cx)[at];
    const double r = static_cast<double>((w & 0xFFu) * 257u);
    const double g = static_cast<double>(((w >> 8) & 0xFFu) * 257u);
    const double b = static_cast<double>(((w >> 16) & 0xFFu) * 257u);
    p[0] = r;
    p[1] = g;
    p[2] = b;
    if constexpr (C == 4) {
      const unsigned a8 = w >> 24;
      p[3] = static_cast<double>(a8 * 257u);
      if (a8 != 255u) {
        const double alpha = __dmul_rn(kQuantumScale, p[3]);
        p[0] = __dmul_rn(alpha, r);
        p[1] = __dmul_rn(alpha, g);
        p[2] = __dmul_rn(alpha, b);
      }
    }
  }
}

// A compile-time slot of the 16-entry running-sum ring.
template <int U>
struct Step {};

// Pixel t (slot U) takes its last term w15 * e_{t-1}: the head of a step,
// the only part its colour lookup waits for.
template <int U, int C>
__device__ __forceinline__ void RotateHead(const double (&sw)[16], const double (&R)[16][C],
                                           const double (&e)[C], double (&v)[C]) {
#pragma unroll
  for (int c = 0; c < C; ++c) v[c] = __dadd_rn(R[U][c], __dmul_rn(sw[15], e[c]));
}

// The rest of the step's rotation: the 15 pixels after pixel t take e_{t-1}
// with their weights and slot U is refilled with pixel t + 16.  Issued after
// the lookup's loads, so their latency overlaps this arithmetic.
template <int U, int C>
__device__ __forceinline__ void RotateTail(const double (&sw)[16], double (&R)[16][C],
                                           const double (&e)[C], const double (&p)[C]) {
#pragma unroll
  for (int jj = 1; jj < 16; ++jj) {
#pragma unroll
    for (int c = 0; c < C; ++c) {
      R[(U + jj) & 15][c] = __dadd_rn(R[(U + jj) & 15][c], __dmul_rn(sw[15 - jj], e[c]));
    }
  }
#pragma unroll
  for (int c = 0; c < C; ++c) R[U][c] = p[c];
}

// The rotations at a compile-time slot (the sum warp's unrolled loop) or at
// a run-time one (a switch over the 16 slots).
template <int C, int U>
__device__ __forceinline__ void RotateTailAt(Step<U>, const double (&sw)[16], double (&R)[16][C],
                                             const double (&e)[C], const double (&p)[C]) {
  RotateTail<U, C>(sw, R, e, p);
}
#define RDB_SLOT_CASES(F) \
  F(0) F(1) F(2) F(3) F(4) F(5) F(6) F(7) F(8) F(9) F(10) F(11) F(12) F(13) F(14)
template <int C>
__device__ __forceinline__ void RotateHeadAt(int u, const double (&sw)[16], const double (&R)[16][C],
                                             const double (&e)[C], double (&v)[C]) {
  switch (u) {
#define RDB_CASE(n) \
  case n: RotateHead<n, C>(sw, R, e, v); break;
    RDB_SLOT_CASES(RDB_CASE)
#undef RDB_CASE
    default: RotateHead<15, C>(sw, R, e, v); break;
  }
}
template <int C>
__device__ __forceinline__ void RotateTailAt(int u, const double (&sw)[16], double (&R)[16][C],
                                             const double (&e)[C], const double (&p)[C]) {
  switch (u) {
#define RDB_CASE(n) \
  case n: RotateTail<n, C>(sw, R, e, p); break;
    RDB_SLOT_CASES(RDB_CASE)
#undef RDB_CASE
    default: RotateTail<15, C>(sw, R, e, p); break;
  }
}
// The ring slot after slot u, and a slot's sums read out.
template <int U>
__device__ __forceinline__ Step<(U + 1) & 15> next_slot(Step<U>) {
  return {};
}
__device__ __forceinline__ int next_slot(int u) { return (u + 1) & 15; }
template <int C, int U>
__device__ __forceinline__ void RingAt(Step<U>, const double (&R)[16][C], double (&out)[C]) {
#pragma unroll
  for (int c = 0; c < C; ++c) out[c] = R[U][c];
}
template <int C>
__device__ __forceinline__ void RingAt(int u, const double (&R)[16][C], double (&out)[C]) {
  switch (u) {
#define RDB_CASE(n)                              \
  case n:                                        \
    for (int c = 0; c < C; ++c) out[c] = R[n][c]; \
    break;
    RDB_SLOT_CASES(RDB_CASE)
#undef RDB_CASE
    default:
      for (int c = 0; c < C; ++c) out[c] = R[15][c];
      break;
  }
}
#undef RDB_SLOT_CASES

// ---- paired walkers: the exchange ------------------------------------------
// In the paired form two warps of a CTA walk the same 32 segments: the chain
// warp runs each step's dependent chain (head, target, key, lookups, index,
// residual), the sum warp the rest of the step (the 15 pending pixels taking
// the new residual, the ring slot refilled with the next sample).  Per step
// the sum warp hands over pixel t's running sum and the chain warp hands back
// its residual, each through one of two mailboxes chosen by step parity, each
// mailbox guarded by an mbarrier that all 32 lanes of the writing warp arrive
// on.  A side can be at most one phase ahead on either barrier: the sum for
// step i + 2 needs the residual of step i, and the residual of step i + 2
// needs the sum for step i + 2.
struct PairBox {
  double s[2][4][32];   // running sums by step parity, channel-planar
  double e[2][4][32];   // residuals by step parity
  uint64_t full_s[2];   // sum warp -> chain warp
  uint64_t full_e[2];   // chain warp -> sum warp
};
constexpr int kPairsPerCta = 4;  // 8 warps: 4 chain warps, then their 4 sum warps
constexpr int kPairCtaThreads = 64 * kPairsPerCta;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void pair_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(32) : "memory");
}
__device__ __forceinline__ void pair_arrive(uint64_t* bar) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
      : "memory");
}
// Waits for the phase of parity `parity` to complete.  Bounded: after about a
// second of clock cycles it sets the status word and returns false, so a
// partner that never arrives ends the launch with an error, never a hang.
__device__ __forceinline__ bool pair_wait(uint64_t* bar, unsigned parity, int* status) {
  const unsigned addr = smem_u32(bar);
  long long start = 0;
#pragma unroll 1
  for (unsigned it = 0;; ++it) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (it == 0) start = clock64();
    if ((it & 63u) == 63u && clock64() - start > (1ll << 31)) {
      atomicExch(status, kDevTimeout);
      return false;
    }
  }
}

__device__ __forceinline__ unsigned own_hash(unsigned key) { return (key * 0x9E3779B1u) >> 8; }

// Fire-and-forget minimum (no value comes back, so nothing waits on it).
__device__ __forceinline__ void red_min(uint32_t* p, uint32_t v) {
  asm volatile("red.relaxed.gpu.global.min.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ---- hashed key maps (alpha keys: 24 bits) ----------------------------------
// keys[slot] = key + 1 (0 = empty), inserted with atomicCAS and never removed;
// every inserted slot is appended to the image's slot list, which the per-key
// kernels walk instead of the whole table.
__device__ __forceinline__ unsigned map_hash(unsigned key) { return key * 0x9E3779B1u; }

// The key's slot (present) or the first empty slot of its probe run (absent);
// -1 when the table is full.  Keys are read plainly: an insert by another
// thread that is not yet visible only sends this one to insert, where the CAS
// sees it.
__device__ __forceinline__ int map_find(const uint32_t* keys, uint32_t mask, unsigned key,
                                        bool* present) {
  unsigned h = map_hash(key) & mask;
#pragma unroll 1
  for (unsigned probe = 0; probe <= mask; ++probe) {
    const uint32_t k1 = reinterpret_cast<const volatile uint32_t*>(keys)[h];
    if (k1 == key + 1u) {
      *present = true;
      return static_cast<int>(h);
    }
    if (k1 == 0u) {
      *present = false;
      return static_cast<int>(h);
    }
    h = (h + 1u) & mask;
  }
  *present = false;
  return -1;
}

__device__ __forceinline__ int map_insert(uint32_t* keys, uint32_t mask, unsigned key, int from,
                                          uint32_t* list, int* count) {
  if (from < 0) return -1;
  unsigned h = static_cast<unsigned>(from);
#pragma unroll 1
  for (unsigned probe = 0; probe <= mask; ++probe) {
    const uint32_t old = atomicCAS(keys + h, 0u, key + 1u);
    if (old == 0u) {
      list[atomicAdd(count, 1)] = h;
      return static_cast<int>(h);
    }
    if (old == key + 1u) return static_cast<int>(h);
    h = (h + 1u) & mask;
  }
  return -1;
}

// Segment k of one image, one thread per segment.  The step loop is
// warp-uniform (every lane runs the warp's longest segment's step count,
// idle past its own), so lanes that need a colour search hand it to the
// whole warp: each search is spread over the 32 lanes instead of running
// serially in one lane while the other 31 wait.  kAssoc: the palette
// associates alpha (four channels, 24-bit keys in hashed maps, no
// uniform-key table); otherwise three channels and direct 2^18-key maps.
template <bool kFloat, bool kAssoc, bool kChain>
__device__ __forceinline__ void WalkSegment(const TswLaunch& L, const TswImage& im,
                                            const tw::Plan& P, const double* errp, int k,
                                            int front, bool active, int lane, PairBox* box) {
  constexpr int C = kAssoc ? 4 : 3;
  const int sid = im.first_seg + k;
  const int begin = k * L.seg_len;
  const int end = active ? min(begin + L.seg_len, im.n) : begin;
  // A cache-free start in pass 0 (after warm_len warm-up positions), and in
  // a window for a segment whose predecessor the previous pass did not walk
  // (it entered the window): that one starts from an empty queue with no
  // warm-up -- it lies far past the front, and a warm-up would hold up the
  // whole launch while buying almost no progress.
  const bool warmup = k > 0 && (L.pass == 0 ||
                                (windowed(L) && k > front && !L.walked[(L.pass & 1) ^ 1][sid - 1]));
  const int ws = (active && warmup) ? begin - min(begin, L.pass == 0 ? L.warm_len : 0) : begin;
  if (active && warmup && ws == begin) {
    // No warm-up position writes the start queue: it is the empty one.
    double* qs0 = L.q_start + static_cast<int64_t>(sid) * 64;
#pragma unroll 4
    for (int i = 0; i < 64; ++i) qs0[i] = 0.0;
  }
  const int steps = end - ws;
  const int64_t base = im.cx_offset;
  const bool memo = L.use_cache != 0;

  double R[16][C];
  double e[C];
#pragma unroll
  for (int c = 0; c < C; ++c) e[c] = 0.0;
  if constexpr (kChain) {
    // The sum warp holds the ring; the chain warp only needs the pending
    // residual q[15] of the predecessor's end queue.
    (void)R;
    if (active && !warmup && k > 0) {
      const double* q = L.q_end[(L.pass & 1) ^ 1] + static_cast<int64_t>(sid - 1) * 64;
#pragma unroll
      for (int c = 0; c < C; ++c) e[c] = q[60 + c];
    }
  } else {
#pragma unroll
  for (int u = 0; u < 16; ++u) {
    double p[C];
#pragma unroll
    for (int c = 0; c < C; ++c) p[c] = 0.0;
    if (ws + u < end) sample<kFloat, C>(L, base + ws + u, p);
#pragma unroll
    for (int c = 0; c < C; ++c) R[u][c] = p[c];
  }
  if (active && !warmup && k > 0) {
    // Start from the predecessor's end queue q[0..15] (oldest first): pixel
    // begin + j holds p + sum_{m=j}^{14} w_{m-j} q[m] in ascending m, and
    // q[15] is the pending residual.
    const double* q = L.q_end[(L.pass & 1) ^ 1] + static_cast<int64_t>(sid - 1) * 64;
#pragma unroll
    for (int m = 0; m < 15; ++m) {
      double qm[C];
#pragma unroll
      for (int c = 0; c < C; ++c) qm[c] = q[4 * m + c];
#pragma unroll
      for (int j = 0; j <= m; ++j) {
#pragma unroll
        for (int c = 0; c < C; ++c) R[j][c] = __dadd_rn(R[j][c], __dmul_rn(L.sw[m - j], qm[c]));
      }
    }
#pragma unroll
    for (int c = 0; c < C; ++c) e[c] = q[60 + c];
  }
  }

  const uint32_t* gprev = im.g[(L.pass & 1) ^ 1];
  uint32_t* gnew = im.g[L.pass & 1];
  uint64_t* ot = L.own + (static_cast<int64_t>(sid) << L.own_bits);
  uint32_t* ol = L.own_list + (static_cast<int64_t>(sid) << L.own_bits);
  const unsigned omask = (1u << L.own_bits) - 1u;
  const uint64_t tag = static_cast<uint64_t>(L.tag_dev ? *L.tag_dev : L.tag) << 32;
  double* qe = L.q_end[L.pass & 1] + static_cast<int64_t>(sid) * 64;
  double* qs = L.q_start + static_cast<int64_t>(sid) * 64;
  uint8_t* out = L.chosen + base;
  const uint8_t* uni = im.uni;
  uint32_t* usemin = im.usemin;
  uint32_t* hkeys = im.hkeys;
  const uint32_t hmask = im.hmask;
  const int warp_steps = __reduce_max_sync(0xffffffffu, static_cast<unsigned>(steps));
  const double* qold = L.q_end[(L.pass & 1) ^ 1] + static_cast<int64_t>(sid) * 64;
  bool changed = false;
  int n_own = 0;
  uint32_t acc = 0;
  // One step of the walk; U = the step index mod 16 is a compile-time
  // constant, so the running sums stay in fixed registers with no
  // indexed jump per step.
  // The paired form compares its end queue step by step: each of the last 16
  // steps loads the previous pass's entry before waiting for its sum, so the
  // comparison waits for nothing (the one-thread form compares once after
  // the walk, below).
  const bool cmp_steps = kChain && active && end - begin >= 16;
  const auto step = [&](auto u, const int i) -> bool {
      const bool on = i < steps;
      const int t = ws + i;
      const bool cmp = cmp_steps && on && t >= end - 16;
      long long qo[C];
      if (cmp) {
#pragma unroll
        for (int c = 0; c < C; ++c) qo[c] = __double_as_longlong(qold[4 * (t - (end - 16)) + c]);
      }
      if constexpr (kChain) {
        // Pixel t's running sum from the sum warp (every lane waits).
        if (!pair_wait(&box->full_s[i & 1], (i >> 1) & 1, L.status)) return false;
      }
      float f[4] = {0.0f, 0.0f, 0.0f, 0.0f};
      unsigned br = 0, bg = 0, bb = 0, ba = 0, key = 0, h = 0;
      int index = 0, slot = 0;
      bool search = false, record = false, from_g = false, booked = false, present = true;
      (void)present;  // hashed maps only
      const bool live = t >= begin;
      const bool keyed = on && memo && live;
      if (on) {
        double p[C];
#pragma unroll
        for (int c = 0; c < C; ++c) p[c] = 0.0;
        double v[C];
        if constexpr (kChain) {
          (void)p;
#pragma unroll
          for (int c = 0; c < C; ++c) v[c] = __dadd_rn(box->s[i & 1][c][lane], __dmul_rn(L.sw[15], e[c]));
        } else {
          if (t + 16 < end) sample<kFloat, C>(L, base + t + 16, p);
          RotateHeadAt<C>(u, L.sw, R, e, v);
        }
#pragma unroll
        for (int c = 0; c < C; ++c) f[c] = clamp_pixel(v[c]);
        br = byte_dev(f[0]);
        bg = byte_dev(f[1]);
        bb = byte_dev(f[2]);
        key = (br >> 2) | ((bg >> 2) << 6) | ((bb >> 2) << 12);
        if constexpr (kAssoc) {
          ba = byte_dev(f[3]);
          key |= (ba >> 2) << 18;
        }
        // A uniform key's search result (and so its memo value) is fixed by the
        // key: no search, no memo, no bookkeeping.
        uint8_t uv = kNotUniform;
        uint32_t gv = kNone;
        if constexpr (kAssoc) {
          // Keys the table has classified uniform need no memo; keys not yet
          // classified, and the rest, go through the hashed map.
          if (uni) {
            uv = __ldg(uni + key);
            if (uv == kUniformUnknown) uv = kNotUniform;
          }
          if (keyed && uv == kNotUniform) {
            slot = map_find(hkeys, hmask, key, &present);
            if (present) gv = __ldg(gprev + slot);
          }
        } else {
          uv = __ldg(uni + key);
          slot = static_cast<int>(key);
          if (keyed) gv = __ldg(gprev + key);  // both loads in flight together
        }
        if constexpr (!kChain) RotateTailAt<C>(u, L.sw, R, e, p);
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
      const int node = search ? tw::descend<kAssoc>(P, br, bg, bb, ba) : 0;
#pragma unroll 1
      while (want) {
        const int src = __ffs(want) - 1;
        want &= want - 1u;
        const int sn = __shfl_sync(0xffffffffu, node, src);
        double t4[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) t4[c] = static_cast<double>(__shfl_sync(0xffffffffu, f[c], src));
        if constexpr (kAssoc) {
          // ClosestColor's target: beta * t with beta = QS * t.a (rd_octree.cpp:190-208).
          const double beta = __dmul_rn(kQuantumScale, t4[3]);
          t4[0] = __dmul_rn(beta, t4[0]);
          t4[1] = __dmul_rn(beta, t4[1]);
          t4[2] = __dmul_rn(beta, t4[2]);
        }
        const int r = tw::search_warp<kAssoc>(P, sn, t4[0], t4[1], t4[2], t4[3], lane);
        if (lane == src) index = r;
      }
      if (booked) {
        if constexpr (kAssoc) {
          if (!present) slot = map_insert(hkeys, hmask, key, slot, im.hlist, im.hcount);
          if (slot < 0) atomicExch(L.status, kDevBadPlan);  // key map full: cannot happen at its size
        }
        if (slot >= 0) red_min(gnew + slot, (static_cast<uint32_t>(k) << 8) | static_cast<uint32_t>(index));
      }
      if (from_g) red_min(usemin + slot, static_cast<uint32_t>(k));
      if (on) {
        if (record) {
          ot[h] = tag | static_cast<uint64_t>(key) | (static_cast<uint64_t>(index) << 24);
          ol[n_own++] = key | (static_cast<uint32_t>(index) << 24);
        }
#pragma unroll
        for (int c = 0; c < C; ++c) e[c] = __dadd_rn(static_cast<double>(f[c]), -errp[c * kMaxPaletteColors + index]);
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
#pragma unroll
            for (int c = 0; c < 4; ++c) d[c] = c < C ? e[c < C ? c : 0] : 0.0;
            if (cmp) {
#pragma unroll
              for (int c = 0; c < C; ++c) changed |= qo[c] != __double_as_longlong(e[c]);
            }
          }
        } else if (t >= begin - 16) {
          double* d = qs + 4 * (t - (begin - 16));
#pragma unroll
          for (int c = 0; c < 4; ++c) d[c] = c < C ? e[c < C ? c : 0] : 0.0;
        }
      }
      if constexpr (kChain) {
        // The residual to the sum warp (every lane arrives).
#pragma unroll
        for (int c = 0; c < C; ++c) box->e[i & 1][c][lane] = e[c];
        pair_arrive(&box->full_e[i & 1]);
      }
      return true;
  };
  if constexpr (kChain) {
    // No ring here: a plain loop.  A wait that gave up ends the walk (the
    // status word says so).
#pragma unroll 1
    for (int i = 0; i < warp_steps; ++i) {
      if (!step(i & 15, i)) return;
    }
  } else {
    // One step per iteration, its ring slot chosen by a switch around the
    // rotations only (sixteen unrolled steps measured 17 % slower a launch,
    // and spill with four channels).
#pragma unroll 1
    for (int i = 0; i < warp_steps; ++i) step(i & 15, i);
  }
  if (L.walk_count) {
    const unsigned mine = active ? static_cast<unsigned>(steps) : 0u;
    const unsigned warp_total = __reduce_add_sync(0xffffffffu, mine);
    if (lane == 0) atomicAdd(L.walk_count, static_cast<unsigned long long>(warp_total));
  }
  if (active && memo) L.own_count[sid] = n_own;
  // One thread a segment: the end queue just written against the previous
  // pass's, once after the walk in batches of independent loads instead of a
  // load on each of the last 16 steps; only the channels a walk reads (without alpha the fourth
  // is never read, so it cannot make a successor's start wrong).  A segment
  // under 16 positions (an image's last) holds no full queue and has no
  // successor: it reports a change.
  if (active && !cmp_steps) {
    if (end - begin >= 16) {
#pragma unroll 16
      for (int q = 0; q < 64; ++q) {
        if ((q & 3) < C) changed |= __double_as_longlong(qe[q]) != __double_as_longlong(qold[q]);
      }
    } else {
      changed = true;
    }
  }
  if (active) {
    L.changed[sid] = changed ? 1 : 0;
    if (windowed(L)) {
      L.walked[L.pass & 1][sid] = 1;
      L.warmed[sid] = warmup ? 1 : 0;
    }
  }
}

template <bool kFloat, bool kAssoc>
__global__ void __launch_bounds__(128, kAssoc ? 2 : 3) TswWalkKernel(TswLaunch L) {
  extern __shared__ __align__(16) unsigned char smem[];
  const bool spread = L.spread != 0;
  int chunk = blockIdx.x;
  if (L.window > 0 && !spread) {
    // One image: chunks are its segments 128 at a time; the grid covers the
    // window, counted from the front's chunk.
    chunk += front_of(L, 0, L.images[0].nsegs) / L.chunk_threads;
    if (chunk >= L.n_chunks) return;
  }
  const TswChunk ch = L.chunks[spread && !L.win ? 0 : chunk];
  const TswImage& im = L.images[ch.image];
  const int front = front_of(L, ch.image, im.nsegs);
  const int wnd = window_of(L, ch.image);
  const int stop = wnd > 0 ? min(front + wnd, im.nsegs) : im.nsegs;
  // Nothing to walk (uniform per CTA).
  Deal deal{0, 0, 0};
  if (spread ? !deal_of(L, ch, front, wnd, im.nsegs, &deal)
             : (ch.k0 + ch.count <= front || ch.k0 >= stop)) {
    return;
  }
  {
    const int4* src = reinterpret_cast<const int4*>(im.plan);
    int4* dst = reinterpret_cast<int4*>(smem);
    for (int i = threadIdx.x; i < im.plan_smem / 16; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  // Residual-side colours channel-planar (colour i of channel c at
  // c * 256 + i): lanes holding different indices then spread over the banks
  // instead of meeting in the palette rows.
  constexpr int C = kAssoc ? 4 : 3;
  double* errp = reinterpret_cast<double*>(smem + L.plan_smem_max);
  {
    tw::Plan P0;
    P0.bind(smem);
    for (int i = threadIdx.x; i < C * kMaxPaletteColors; i += blockDim.x) {
      const int c = i / kMaxPaletteColors, col = i - c * kMaxPaletteColors;
      errp[i] = col < P0.h->count ? P0.rcol<kAssoc>(col)[c] : 0.0;
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  int k, kk;
  bool active;
  if (spread) {
    // Slots lane-major across the CTA's warps, so every warp gets segments
    // from the whole window, the nearest ones included.
    k = deal.base + (lane * 4 + static_cast<int>(threadIdx.x >> 5)) * deal.g + deal.c;
    active = k >= front && k < stop;
    if (__ballot_sync(0xffffffffu, active) == 0u) return;  // the warp leaves together
    kk = active ? k : front;
  } else {
    // Warps whose segments are all verified, past the window or past the
    // image leave together.
    const int warp_k0 = ch.k0 + static_cast<int>(threadIdx.x & ~31u);
    const int warp_end = min(ch.k0 + ch.count, warp_k0 + 32);
    if (warp_end <= front || warp_k0 >= ch.k0 + ch.count || warp_k0 >= stop) return;
    k = ch.k0 + static_cast<int>(threadIdx.x);
    active = static_cast<int>(threadIdx.x) < ch.count && k >= front && k < stop;
    kk = active ? k : warp_end - 1;
  }
  tw::Plan P;
  P.bind(smem);
  WalkSegment<kFloat, kAssoc, false>(L, im, P, errp, kk, front, active, lane, nullptr);
}

// The sum warp of a pair: the 16-slot ring of running sums for one segment
// per lane, one step ahead of the chain warp.  It hands over pixel t's sum
// (everything but the w15 * e_{t-1} term, which the chain adds) before step t,
// and after the residual of step i - 1 arrives it adds that residual to the
// 15 pending pixels and refills the slot of the pixel just taken with the
// sample 16 positions on -- the same operations in the same order as the
// single-thread walker's rotation, so the same sums bit for bit.
template <bool kFloat, bool kAssoc>
__device__ __forceinline__ void WalkSums(const TswLaunch& L, const TswImage& im, int k, int front,
                                         bool active, int lane, PairBox* box) {
  constexpr int C = kAssoc ? 4 : 3;
  const int sid = im.first_seg + k;
  const int begin = k * L.seg_len;
  const int end = active ? min(begin + L.seg_len, im.n) : begin;
  const bool warmup = k > 0 && (L.pass == 0 ||
                                (windowed(L) && k > front && !L.walked[(L.pass & 1) ^ 1][sid - 1]));
  const int ws = (active && warmup) ? begin - min(begin, L.pass == 0 ? L.warm_len : 0) : begin;
  const int steps = end - ws;
  const int64_t base = im.cx_offset;
  double R[16][C];
  double e0[C];
#pragma unroll
  for (int c = 0; c < C; ++c) e0[c] = 0.0;
#pragma unroll
  for (int u = 0; u < 16; ++u) {
    double p[C];
#pragma unroll
    for (int c = 0; c < C; ++c) p[c] = 0.0;
    if (ws + u < end) sample<kFloat, C>(L, base + ws + u, p);
#pragma unroll
    for (int c = 0; c < C; ++c) R[u][c] = p[c];
  }
  if (active && !warmup && k > 0) {
    const double* q = L.q_end[(L.pass & 1) ^ 1] + static_cast<int64_t>(sid - 1) * 64;
#pragma unroll
    for (int m = 0; m < 15; ++m) {
      double qm[C];
#pragma unroll
      for (int c = 0; c < C; ++c) qm[c] = q[4 * m + c];
#pragma unroll
      for (int j = 0; j <= m; ++j) {
#pragma unroll
        for (int c = 0; c < C; ++c) R[j][c] = __dadd_rn(R[j][c], __dmul_rn(L.sw[m - j], qm[c]));
      }
    }
#pragma unroll
    for (int c = 0; c < C; ++c) e0[c] = q[60 + c];
  }
  const int warp_steps = __reduce_max_sync(0xffffffffu, static_cast<unsigned>(steps));
  if (warp_steps <= 0) return;
  // Step 0's sum.
#pragma unroll
  for (int c = 0; c < C; ++c) box->s[0][c][lane] = R[0][c];
  pair_arrive(&box->full_s[0]);
  // Iteration i: the residual of step i - 1 (the queue's pending one for
  // i = 0), slot i mod 16 refilled, then step i + 1's sum handed over.
  const auto iter = [&](auto u, const int i) -> bool {
    double p[C];
#pragma unroll
    for (int c = 0; c < C; ++c) p[c] = 0.0;
    const int t = ws + i;
    if (i < steps && t + 16 < end) sample<kFloat, C>(L, base + t + 16, p);
    double e[C];
    if (i == 0) {
#pragma unroll
      for (int c = 0; c < C; ++c) e[c] = e0[c];
    } else {
      if (!pair_wait(&box->full_e[(i - 1) & 1], ((i - 1) >> 1) & 1, L.status)) return false;
#pragma unroll
      for (int c = 0; c < C; ++c) e[c] = box->e[(i - 1) & 1][c][lane];
    }
    RotateTailAt<C>(u, L.sw, R, e, p);
    double nx[C];
    RingAt<C>(next_slot(u), R, nx);
#pragma unroll
    for (int c = 0; c < C; ++c) box->s[(i + 1) & 1][c][lane] = nx[c];
    pair_arrive(&box->full_s[(i + 1) & 1]);
    return true;
  };
  const int last = warp_steps - 1;  // iterations 0 .. last - 1 hand over sums 1 .. last
  if constexpr (kAssoc) {
#pragma unroll 1
    for (int i = 0; i < last; ++i) {
      if (!iter(i & 15, i)) return;
    }
  } else {
#pragma unroll 1
    for (int i0 = 0; i0 < last; i0 += 16) {
#define RDB_ITER(n)                                  \
  if (i0 + (n) >= last) break;                       \
  if (!iter(Step<(n)>{}, i0 + (n))) return;
      RDB_ITER(0) RDB_ITER(1) RDB_ITER(2) RDB_ITER(3) RDB_ITER(4) RDB_ITER(5) RDB_ITER(6) RDB_ITER(7)
      RDB_ITER(8) RDB_ITER(9) RDB_ITER(10) RDB_ITER(11) RDB_ITER(12) RDB_ITER(13) RDB_ITER(14) RDB_ITER(15)
#undef RDB_ITER
    }
  }
}

// The paired form of the walk: 8 warps per CTA, warp w < 4 the chain warp and
// warp w + 4 the sum warp of the same 32 segments of the chunk.  Two CTAs per
// SM without alpha (128 registers a thread); one with alpha, whose four-channel
// ring does not fit in 128.
template <bool kFloat, bool kAssoc>
__global__ void __launch_bounds__(kPairCtaThreads, kAssoc ? 1 : 2) TswWalkPairKernel(TswLaunch L) {
  extern __shared__ __align__(16) unsigned char smem[];
  const bool spread = L.spread != 0;
  int chunk = blockIdx.x;
  if (L.window > 0 && !spread) {
    chunk += front_of(L, 0, L.images[0].nsegs) / L.chunk_threads;
    if (chunk >= L.n_chunks) return;
  }
  const TswChunk ch = L.chunks[spread && !L.win ? 0 : chunk];
  const TswImage& im = L.images[ch.image];
  const int front = front_of(L, ch.image, im.nsegs);
  const int wnd = window_of(L, ch.image);
  const int stop = wnd > 0 ? min(front + wnd, im.nsegs) : im.nsegs;
  // Nothing to walk (uniform per CTA).
  Deal deal{0, 0, 0};
  if (spread ? !deal_of(L, ch, front, wnd, im.nsegs, &deal)
             : (ch.k0 + ch.count <= front || ch.k0 >= stop)) {
    return;
  }
  constexpr int C = kAssoc ? 4 : 3;
  double* errp = reinterpret_cast<double*>(smem + L.plan_smem_max);
  // After the plan and the residual-side colours, 16-byte aligned (as the
  // host sizes it).
  const int box_off = (L.plan_smem_max + 4 * kMaxPaletteColors * static_cast<int>(sizeof(double)) + 15) & ~15;
  PairBox* boxes = reinterpret_cast<PairBox*>(smem + box_off);
  {
    const int4* src = reinterpret_cast<const int4*>(im.plan);
    int4* dst = reinterpret_cast<int4*>(smem);
    for (int i = threadIdx.x; i < im.plan_smem / 16; i += blockDim.x) dst[i] = src[i];
  }
  if (threadIdx.x < 4 * kPairsPerCta) {
    PairBox& b = boxes[threadIdx.x >> 2];
    const int which = threadIdx.x & 3;
    pair_init(which < 2 ? &b.full_s[which] : &b.full_e[which - 2]);
  }
  __syncthreads();
  {
    tw::Plan P0;
    P0.bind(smem);
    for (int i = threadIdx.x; i < C * kMaxPaletteColors; i += blockDim.x) {
      const int c = i / kMaxPaletteColors, col = i - c * kMaxPaletteColors;
      errp[i] = col < P0.h->count ? P0.rcol<kAssoc>(col)[c] : 0.0;
    }
  }
  // Barrier initialisation and the staged tables, visible to every warp.
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int pair = warp % kPairsPerCta;
  // Both warps of a pair see the same 32 segments and leave together.
  int kk;
  bool active;
  if (spread) {
    // Slots lane-major across the pairs, so every pair gets segments from the
    // whole window, the nearest ones included.
    const int k = deal.base + (lane * kPairsPerCta + pair) * deal.g + deal.c;
    active = k >= front && k < stop;
    if (__ballot_sync(0xffffffffu, active) == 0u) return;
    kk = active ? k : front;
  } else {
    const int warp_k0 = ch.k0 + 32 * pair;
    const int warp_end = min(ch.k0 + ch.count, warp_k0 + 32);
    if (warp_end <= front || warp_k0 >= ch.k0 + ch.count || warp_k0 >= stop) return;
    const int k = warp_k0 + lane;
    active = k < warp_end && k >= front && k < stop;
    kk = active ? k : warp_end - 1;
  }
  if (warp < kPairsPerCta) {
    tw::Plan P;
    P.bind(smem);
    WalkSegment<kFloat, kAssoc, true>(L, im, P, errp, kk, front, active, lane, &boxes[pair]);
  } else {
    WalkSums<kFloat, kAssoc>(L, im, kk, front, active, lane, &boxes[pair]);
  }
}

// G_new = the entries of G_prev that verified segments made; usemin cleared;
// this pass's first failure of the image reset to "none".
// Direct maps: one thread per key; hashed maps: the inserted slots.
__global__ void TswPrepare(TswLaunch L) {
  const int m = blockIdx.y;
  if (m >= L.n_images) return;
  const TswImage& im = L.images[m];
  const int front = front_of(L, m, im.nsegs);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    L.bad[L.pass & 1][m] = 0x7F7F7F7F;
    // Hashed maps: the slot list entries the last classification covered
    // (hcount[1] .. hcount[2] of TswUniformFill) are done.
    if (im.hkeys) im.hcount[1] = im.hcount[2];
  }
  const uint32_t* gp = im.g[(L.pass & 1) ^ 1];
  uint32_t* gn = im.g[L.pass & 1];
  const int stride = gridDim.x * blockDim.x;
  const int n = im.hkeys ? *im.hcount : kKeys;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int slot = im.hkeys ? static_cast<int>(im.hlist[i]) : i;
    const uint32_t gv = gp[slot];
    gn[slot] = (gv != kNone && static_cast<int>(gv >> 8) < front) ? gv : kNone;
    im.usemin[slot] = kNoUser;
  }
}

// Classifies the keys of alpha-associated palettes that this pass's walk met
// for the first time (every key it booked is in the image's hashed map):
// rdb_uniform_alpha.cuh.  Later passes then answer the uniform ones without
// the memo.  Images sharing a palette write the same values.  Slots are
// listed in insertion order and never removed, so only the list entries added
// since the last classification need it: hcount[1] is where the last one
// stopped, hcount[2] records where this one stops (the next pass's prepare
// kernel moves it into hcount[1]).
__global__ void TswUniformFill(TswLaunch L) {
  const int m = blockIdx.y;
  if (m >= L.n_images) return;
  const TswImage& im = L.images[m];
  if (!im.hkeys || !im.uni) return;
  uint8_t* table = const_cast<uint8_t*>(im.uni);
  const int n = im.hcount[0];
  const int done = im.hcount[1];
  if (blockIdx.x == 0 && threadIdx.x == 0) im.hcount[2] = n;
  tw::Plan P;
  P.bind(im.plan);
  for (int i = done + blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned key = im.hkeys[im.hlist[i]] - 1u;
    if (table[key] == kUniformUnknown) table[key] = uniform_alpha_key(P, key);
  }
}

// The "from G" check, per key.
__global__ void TswVerifyKeys(TswLaunch L) {
  const int m = blockIdx.y;
  if (m >= L.n_images) return;
  const TswImage& im = L.images[m];
  const int stride = gridDim.x * blockDim.x;
  const int n = im.hkeys ? *im.hcount : kKeys;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int slot = im.hkeys ? static_cast<int>(im.hlist[i]) : i;
    const uint32_t u = im.usemin[slot];
    if (u == kNoUser) continue;
    const uint32_t gp = im.g[(L.pass & 1) ^ 1][slot];
    const uint32_t gn = im.g[L.pass & 1][slot];
    if ((gn & 0xFFu) != (gp & 0xFFu) || (gn >> 8) >= u) atomicMin(L.bad[L.pass & 1] + m, static_cast<int>(u));
  }
}

// The queue and own checks, one thread per walked segment (a window's
// segments fit one wave, and a segment's own list is short).
__global__ void TswVerifySegments(TswLaunch L, int total_segs) {
  int sid = blockIdx.x * blockDim.x + threadIdx.x;
  if (L.window > 0) sid += front_of(L, 0, L.images[0].nsegs);  // the grid covers the window
  if (sid >= total_segs) return;
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
  const int wnd = window_of(L, lo);
  if (wnd > 0 && k >= front + wnd) {
    // Not walked this pass: the front stops at the window's end.
    if (k == front + wnd) atomicMin(L.bad[L.pass & 1] + lo, k);
    return;
  }
  // Only the image's FIRST failure matters: segments past one already found
  // need no check.  (A relaxed read; a stale value only costs a check.)
  if (k > *reinterpret_cast<volatile const int*>(L.bad[L.pass & 1] + lo)) return;
  bool ok = true;
  if (k > front) {
    // The first walked segment started from a verified predecessor's queue;
    // the others from their predecessor's end queue of the previous pass,
    // which the predecessor compared with its new one (L.changed), or from a
    // warm-up (pass 0, and segments entering a window), whose queue is
    // compared with the predecessor's end queue itself.
    if (L.pass == 0 || (windowed(L) && L.warmed[sid])) {
      const double* a = L.q_start + static_cast<int64_t>(sid) * 64;
      const double* b = L.q_end[L.pass & 1] + static_cast<int64_t>(sid - 1) * 64;
#pragma unroll 8
      for (int i = 0; i < 64; ++i) {
        if (__double_as_longlong(a[i]) != __double_as_longlong(b[i])) ok = false;
      }
    } else if (L.changed[sid - 1]) {
      ok = false;
    }
  }
  if (ok && L.use_cache) {
    const uint32_t* gn = im.g[L.pass & 1];
    const uint32_t* ol = L.own_list + (static_cast<int64_t>(sid) << L.own_bits);
    const int cnt = L.own_count[sid];
    if (im.hkeys) {
      for (int i = 0; i < cnt && ok; ++i) {
        const uint32_t w = ol[i];
        uint32_t g = kNone;
        bool present = false;
        const int slot = map_find(im.hkeys, im.hmask, w & 0xFFFFFFu, &present);
        if (present) g = gn[slot];
        if (static_cast<int>(g >> 8) < k && (g & 0xFFu) != (w >> 24)) ok = false;
      }
    } else {
      // Direct maps: eight entries at a time, their list words and then their
      // map words loaded independently, so a long list costs a few round
      // trips instead of two dependent loads an entry.
      for (int i0 = 0; i0 < cnt && ok; i0 += 8) {
        uint32_t w[8], g[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) w[j] = i0 + j < cnt ? ol[i0 + j] : 0u;
#pragma unroll
        for (int j = 0; j < 8; ++j) g[j] = i0 + j < cnt ? gn[w[j] & 0xFFFFFFu] : kNone;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          if (static_cast<int>(g[j] >> 8) < k && (g[j] & 0xFFu) != (w[j] >> 24)) ok = false;
        }
      }
    }
  }
  if (!ok) atomicMin(L.bad[L.pass & 1] + lo, k);
}

// The same checks, one warp per walked segment: for long segments, whose own
// lists run to hundreds of keys, the lanes share the list.
__global__ void TswVerifySegmentsWarp(TswLaunch L, int total_segs) {
  int sid_lo = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (L.window > 0) sid_lo += front_of(L, 0, L.images[0].nsegs);  // the grid covers the window
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
  const int wnd = window_of(L, lo);
  if (wnd > 0 && k >= front + wnd) {
    // Not walked this pass: the front stops at the window's end.
    if (k == front + wnd && lane == 0) atomicMin(L.bad[L.pass & 1] + lo, k);
    return;
  }
  // Only the image's FIRST failure matters: segments past one already found
  // need no check.  (A relaxed read; a stale value only costs a check.)
  if (k > *reinterpret_cast<volatile const int*>(L.bad[L.pass & 1] + lo)) return;
  bool ok = true;
  if (k > front) {
    // The first walked segment started from a verified predecessor's queue;
    // the others from their predecessor's end queue of the previous pass,
    // which the predecessor compared with its new one (L.changed), or from a
    // warm-up (pass 0, and segments entering a window), whose queue is
    // compared with the predecessor's end queue itself.
    if (L.pass == 0 || (windowed(L) && L.warmed[sid])) {
      const double* a = L.q_start + static_cast<int64_t>(sid) * 64;
      const double* b = L.q_end[L.pass & 1] + static_cast<int64_t>(sid - 1) * 64;
      for (int i = lane; i < 64; i += 32) {
        if (__double_as_longlong(a[i]) != __double_as_longlong(b[i])) ok = false;
      }
    } else if (L.changed[sid - 1]) {
      ok = false;
    }
  }
  if (L.use_cache) {
    const uint32_t* gn = im.g[L.pass & 1];
    const uint32_t* ol = L.own_list + (static_cast<int64_t>(sid) << L.own_bits);
    const int cnt = L.own_count[sid];
    for (int i = lane; i < cnt; i += 32) {
      const uint32_t w = ol[i];
      const unsigned key = w & 0xFFFFFFu;
      uint32_t g = kNone;
      if (im.hkeys) {
        bool present = false;
        const int slot = map_find(im.hkeys, im.hmask, key, &present);
        if (present) g = gn[slot];
      } else {
        g = gn[key];
      }
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
    const float a = h->assoc ? pc.w : load_sample(im.pixels, im.layout, im.row_stride, im.width, pix).w;
    im.rgba_out[pix] = make_float4(pc.x, pc.y, pc.z, a);
  }
}

// Per-image windows for the next pass (one block): every unfinished image
// gets its share of the resident segments in proportion to the segments it
// has left, at least win_min and at most what it has left.
__global__ void TswWindows(TswLaunch L) {
  __shared__ long long total;
  if (threadIdx.x == 0) total = 0;
  __syncthreads();
  const int* bad = L.bad[L.pass & 1];
  long long mine = 0;
  for (int i = threadIdx.x; i < L.n_images; i += blockDim.x) {
    const int ns = L.images[i].nsegs;
    mine += ns - min(bad[i], ns);
  }
  atomicAdd(reinterpret_cast<unsigned long long*>(&total), static_cast<unsigned long long>(mine));
  __syncthreads();
  const long long all = total > 0 ? total : 1;
  for (int i = threadIdx.x; i < L.n_images; i += blockDim.x) {
    const int ns = L.images[i].nsegs;
    const long long rem = ns - min(bad[i], ns);
    long long w = (static_cast<long long>(L.resident_segs) * rem + all - 1) / all;
    w = max(w, static_cast<long long>(L.win_min));
    L.win[i] = static_cast<int>(max(1ll, min(w, rem)));
  }
}

// The loop's control step (see BuildTswLoopGraph), one block.
__global__ void TswControl(TswLaunch L, cudaGraphConditionalHandle handle, int* ctl,
                           uint32_t* tag_dev, int max_passes) {
  __shared__ int done_all, stalled_any;
  if (threadIdx.x == 0) {
    done_all = 1;
    stalled_any = 0;
  }
  __syncthreads();
  const bool finished = ctl[1] != 0;
  if (!finished) {
    const int* cur = L.bad[L.pass & 1];
    const int* prev = L.bad[(L.pass & 1) ^ 1];
    for (int i = threadIdx.x; i < L.n_images; i += blockDim.x) {
      const int ns = L.images[i].nsegs;
      const int nf = min(cur[i], ns);
      const int of = min(prev[i], ns);
      if (nf < ns) {
        atomicAnd(&done_all, 0);
        if (nf <= of) atomicOr(&stalled_any, 1);
      }
    }
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  if (finished) {
    cudaGraphSetConditional(handle, 0);
    return;
  }
  const int passes = ++ctl[0];
  if (done_all) {
    ctl[1] = 1;
    ctl[2] = passes;
    cudaGraphSetConditional(handle, 0);
  } else if (stalled_any || passes >= max_passes) {
    ctl[1] = 1;
    atomicExch(L.status, stalled_any ? kDevBadItem : kDevTimeout);
    cudaGraphSetConditional(handle, 0);
  }
  *tag_dev += 1u;
}

// Grids: every chunk and every segment, or with a window the chunks and
// segments it can reach from wherever the front is (one more chunk: the
// window need not start on a chunk boundary; one more segment: the first one
// past the window stops the front).
unsigned TswWalkGrid(const TswLaunch& L) {
  if (L.window <= 0) return static_cast<unsigned>(L.n_chunks);
  return static_cast<unsigned>(std::min(L.n_chunks, (L.window + L.chunk_threads - 1) / L.chunk_threads + 1));
}
// Segments up to kThreadCheckLen positions are checked one thread each,
// longer ones one warp each.
constexpr int kThreadCheckLen = 256;
const void* VerifyFunc(const TswLaunch& L) {
  return L.seg_len <= kThreadCheckLen ? reinterpret_cast<const void*>(TswVerifySegments)
                                      : reinterpret_cast<const void*>(TswVerifySegmentsWarp);
}
unsigned TswVerifyGrid(const TswLaunch& L, int total_segs) {
  const int segs = L.window > 0 ? std::min(total_segs, L.window + 1) : total_segs;
  const int per_block = L.seg_len <= kThreadCheckLen ? 256 : 8;
  return static_cast<unsigned>((segs + per_block - 1) / per_block);
}

// The walk kernel of a launch's form and its shape: one thread per segment
// (128-thread CTAs), or a chain warp and a sum warp per 32 segments
// (256-thread CTAs, the same 128 segments, plus the pairs' mailboxes).
struct WalkShape {
  const void* fn;
  unsigned threads;
  std::size_t smem;
};
WalkShape WalkShapeOf(bool paired, bool is_float, bool assoc, int plan_smem_max) {
  const std::size_t base = (TswSmemBytes(plan_smem_max) + 15) & ~std::size_t{15};
  if (paired) {
    const void* fn = assoc ? (is_float ? reinterpret_cast<const void*>(TswWalkPairKernel<true, true>)
                                       : reinterpret_cast<const void*>(TswWalkPairKernel<false, true>))
                           : (is_float ? reinterpret_cast<const void*>(TswWalkPairKernel<true, false>)
                                       : reinterpret_cast<const void*>(TswWalkPairKernel<false, false>));
    return {fn, static_cast<unsigned>(kPairCtaThreads), base + kPairsPerCta * sizeof(PairBox)};
  }
  const void* fn = assoc ? (is_float ? reinterpret_cast<const void*>(TswWalkKernel<true, true>)
                                     : reinterpret_cast<const void*>(TswWalkKernel<false, true>))
                         : (is_float ? reinterpret_cast<const void*>(TswWalkKernel<true, false>)
                                     : reinterpret_cast<const void*>(TswWalkKernel<false, false>));
  return {fn, 128u, base};
}
WalkShape WalkShapeOf(const TswLaunch& L) {
  return WalkShapeOf(L.paired != 0, L.is_float != 0, L.assoc != 0, L.plan_smem_max);
}

}  // namespace

std::size_t TswSmemBytes(int plan_smem_max) {
  return static_cast<std::size_t>(plan_smem_max) + 4 * kMaxPaletteColors * sizeof(double);
}

int TswResidentThreads(int plan_smem_max, int sm_count, int assoc, int paired) {
  const WalkShape w = WalkShapeOf(paired != 0, false, assoc != 0, plan_smem_max);
  if (AllowMaxSmem(w.fn) != cudaSuccess) return 0;
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, w.fn, static_cast<int>(w.threads),
                                                    w.smem) != cudaSuccess) {
    return 0;
  }
  return blocks * 128 * sm_count;  // 128 segments per CTA in either form
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
  const WalkShape w = WalkShapeOf(L);
  cudaError_t e = AllowMaxSmem(w.fn);
  if (e != cudaSuccess) return e;
  void* args[] = {const_cast<TswLaunch*>(&L)};
  return cudaLaunchKernel(w.fn, dim3(TswWalkGrid(L)), dim3(w.threads), args, w.smem, s);
}

cudaError_t LaunchTswWindows(const TswLaunch& L, cudaStream_t s) {
  if (!L.win || L.n_images <= 0) return cudaSuccess;
  TswWindows<<<1, 256, 0, s>>>(L);
  return cudaGetLastError();
}

cudaError_t LaunchTswVerify(const TswLaunch& L, int total_segs, cudaStream_t s) {
  if (L.use_cache && L.n_images > 0) {
    TswVerifyKeys<<<dim3(kKeys / 256, L.n_images), 256, 0, s>>>(L);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (L.assoc) {
      TswUniformFill<<<dim3(kFillBlocks, L.n_images), 256, 0, s>>>(L);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
  }
  if (total_segs <= 0) return cudaSuccess;
  void* args[] = {const_cast<TswLaunch*>(&L), &total_segs};
  const cudaError_t e2 = cudaLaunchKernel(VerifyFunc(L), dim3(TswVerifyGrid(L, total_segs)), dim3(256), args, 0, s);
  if (e2 != cudaSuccess) return e2;
  return cudaGetLastError();
}

namespace {

cudaError_t AddKernel(cudaGraph_t g, cudaGraphNode_t* last, const void* func, dim3 grid,
                      dim3 block, unsigned smem, void** args) {
  cudaKernelNodeParams kp{};
  kp.func = const_cast<void*>(func);
  kp.gridDim = grid;
  kp.blockDim = block;
  kp.sharedMemBytes = smem;
  kp.kernelParams = args;
  cudaGraphNode_t node;
  const cudaError_t e = cudaGraphAddKernelNode(&node, g, *last ? last : nullptr, *last ? 1 : 0, &kp);
  if (e == cudaSuccess) *last = node;
  return e;
}

// One pass into graph g after *last: clear this parity's failures, prepare,
// walk, check, control.
cudaError_t AddPass(cudaGraph_t g, cudaGraphNode_t* last, TswLaunch* L, int total_segs,
                    cudaGraphConditionalHandle* h, int** ctl, uint32_t** tag_dev, int* max_passes) {
  cudaError_t e;
  if (!L->use_cache || L->n_images <= 0) {
    // Without the memo no prepare kernel runs to reset this pass's failures.
    cudaMemsetParams ms{};
    ms.dst = L->bad[L->pass & 1];
    ms.value = 0x7F;
    ms.elementSize = 1;
    ms.width = static_cast<std::size_t>(L->n_images) * sizeof(int);
    ms.height = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddMemsetNode(&node, g, *last ? last : nullptr, *last ? 1 : 0, &ms);
    if (e != cudaSuccess) return e;
    *last = node;
  }
  void* args1[] = {L};
  if (L->use_cache && L->n_images > 0) {
    e = AddKernel(g, last, reinterpret_cast<const void*>(TswPrepare), dim3(kKeys / 256, L->n_images),
                  dim3(256), 0, args1);
    if (e != cudaSuccess) return e;
  }
  if (L->n_chunks > 0) {
    const WalkShape w = WalkShapeOf(*L);
    e = AddKernel(g, last, w.fn, dim3(TswWalkGrid(*L)), dim3(w.threads), static_cast<unsigned>(w.smem),
                  args1);
    if (e != cudaSuccess) return e;
  }
  if (L->use_cache && L->n_images > 0) {
    e = AddKernel(g, last, reinterpret_cast<const void*>(TswVerifyKeys), dim3(kKeys / 256, L->n_images),
                  dim3(256), 0, args1);
    if (e != cudaSuccess) return e;
    if (L->assoc) {
      e = AddKernel(g, last, reinterpret_cast<const void*>(TswUniformFill),
                    dim3(kFillBlocks, L->n_images), dim3(256), 0, args1);
      if (e != cudaSuccess) return e;
    }
  }
  if (total_segs > 0) {
    void* args2[] = {L, &total_segs};
    e = AddKernel(g, last, VerifyFunc(*L), dim3(TswVerifyGrid(*L, total_segs)),
                  dim3(256), 0, args2);
    if (e != cudaSuccess) return e;
  }
  if (L->win && L->n_images > 0) {
    e = AddKernel(g, last, reinterpret_cast<const void*>(TswWindows), dim3(1), dim3(256), 0, args1);
    if (e != cudaSuccess) return e;
  }
  void* args3[] = {L, h, ctl, tag_dev, max_passes};
  return AddKernel(g, last, reinterpret_cast<const void*>(TswControl), dim3(1), dim3(256), 0, args3);
}

}  // namespace

cudaError_t BuildTswLoopGraph(const TswLaunch& even, const TswLaunch& odd, int total_segs,
                              int* ctl, uint32_t* tag_dev, int max_passes, cudaGraph_t* out) {
  cudaError_t e;
  if (even.n_chunks > 0) {
    if ((e = AllowMaxSmem(WalkShapeOf(even).fn)) != cudaSuccess) return e;
  }
  cudaGraph_t g = nullptr;
  if ((e = cudaGraphCreate(&g, 0)) != cudaSuccess) return e;
  cudaGraphConditionalHandle h;
  if ((e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault)) != cudaSuccess) {
    cudaGraphDestroy(g);
    return e;
  }
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  if ((e = cudaGraphAddNode(&cnode, g, nullptr, 0, &cp)) != cudaSuccess) {
    cudaGraphDestroy(g);
    return e;
  }
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  TswLaunch L0 = even, L1 = odd;
  cudaGraphNode_t last = nullptr;
  if ((e = AddPass(body, &last, &L0, total_segs, &h, &ctl, &tag_dev, &max_passes)) != cudaSuccess ||
      (e = AddPass(body, &last, &L1, total_segs, &h, &ctl, &tag_dev, &max_passes)) != cudaSuccess) {
    cudaGraphDestroy(g);
    return e;
  }
  *out = g;
  return cudaSuccess;
}

cudaError_t LaunchTswScatter(const TswLaunch& L, int64_t total, cudaStream_t s) {
  if (total <= 0) return cudaSuccess;
  TswScatter<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(L, total);
  return cudaGetLastError();
}

}  // namespace rdb
