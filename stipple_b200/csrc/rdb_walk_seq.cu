// rdb_walk_seq.cu -- the sequential-exact Riemersma walk, one warp per image.
//
// Reference: src/rd_riemersma_cpu.cpp:39-113 (Visit) and :359-417
// (RiemersmaWalkCpu).  Output is bit-identical to the reference CPU walk.
//
// The walk is a dependent chain: pixel t's target needs the residual of
// pixel t-1.  The target is
//     v_t = (((p_t + w0 e_{t-16}) + w1 e_{t-15}) + ...) + w15 e_{t-1}
// summed in that order (the oldest queue entry first).  Only the LAST term
// depends on the previous pixel, so the warp keeps a running partial sum per
// upcoming pixel: lane j holds pixel t+1+j's sum (j = 0..14), every lane
// holds pixel t's ("the head").  When e_{t-1} is known, each lane adds its
// own term (lane j: w_{14-j} * e) and the critical path is a single
// DMUL + DADD.  The sums are then shifted one lane down by shuffles while the
// warp does the lookup -- off the critical path.  All lanes compute the head
// pixel redundantly, so every branch is warp-uniform.
//
// The memo (quantize.c's cache, rd_types.h:111-153) is observable: the first
// target to touch a 6-bit-per-channel key decides the index for every later
// target with that key.  It is reproduced exactly by a per-walk table in
// global memory (uint16 per key: generation << 8 | index, so a slab is reused
// across walks without clearing), fronted by a tagged direct-mapped cache in
// shared memory that holds recently used keys.  On a first touch the warp
// descends the octree (child table in shared memory) and searches the
// subtree's slots in parallel.
//
// Pixels enter through a 3-chunk ring of 32 positions in shared memory that
// is filled two chunks ahead with register-staged loads, so no load latency
// lands on the chain.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/rdb.h"
#include "rdb_curve.h"
#include "rdb_device.cuh"
#include "rdb_runtime.h"
#include "rdb_walk.h"

namespace rdb {
namespace {

constexpr int kRing = 96;

struct Vec4 {
  double r, g, b, a;
};

__device__ __forceinline__ Vec4 shfl_vec(const Vec4& v, int src, bool assoc) {
  Vec4 o;
  o.r = __shfl_sync(0xffffffffu, v.r, src);
  o.g = __shfl_sync(0xffffffffu, v.g, src);
  o.b = __shfl_sync(0xffffffffu, v.b, src);
  o.a = assoc ? __shfl_sync(0xffffffffu, v.a, src) : 0.0;
  return o;
}

__device__ __forceinline__ Vec4 shfl_down_vec(const Vec4& v, bool assoc) {
  Vec4 o;
  o.r = __shfl_down_sync(0xffffffffu, v.r, 1);
  o.g = __shfl_down_sync(0xffffffffu, v.g, 1);
  o.b = __shfl_down_sync(0xffffffffu, v.b, 1);
  o.a = assoc ? __shfl_down_sync(0xffffffffu, v.a, 1) : 0.0;
  return o;
}

__device__ __forceinline__ Vec4 sample_to_vec(int assoc, float4 s) {
  Vec4 v;
  associate_sample(assoc, s, v.r, v.g, v.b, v.a);
  return v;
}

template <bool kAssoc>
__device__ void WalkOne(const SeqItem& it, const SeqLaunch& L, const PlanView& P,
                        uint32_t* cache, int cache_bits, int32_t* ring_ord, float4* ring_pix,
                        uint16_t* memo, unsigned gen, int lane) {
  const int n = it.n;
  const int width = it.width;
  const unsigned char* img = it.pixels;
  const int layout = it.layout;
  const int64_t stride = it.row_stride;
  const int32_t* order = it.order;
  const bool use_cache = L.use_cache != 0;
  const unsigned tag_bits = 24u - static_cast<unsigned>(cache_bits);
  const unsigned tag_mask = (1u << tag_bits) - 1u;

  const double w15 = L.sw[15];
  const double wl = (lane < 15) ? L.sw[14 - lane] : 0.0;

  // Ring preload: chunks 0 and 1 directly, chunk 2's order prefetched.
  for (int c = 0; c < 2; ++c) {
    const int q = 32 * c + lane;
    int o = -1;
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
    if (q < n) {
      o = order[q];
      if (static_cast<unsigned>(o) >= static_cast<unsigned>(n)) {
        atomicExch(L.status, kDevBadItem);
        o = 0;
      }
      s = load_sample(img, layout, stride, width, o);
    }
    ring_ord[32 * c + lane] = o;
    ring_pix[32 * c + lane] = s;
  }
  int ord_stage = (64 + lane < n) ? order[64 + lane] : -1;
  float4 pix_stage = make_float4(0.f, 0.f, 0.f, 0.f);
  __syncwarp();

  // Head = pixel 0, lane j holds pixel 1+j.  The queue starts at zero, and a
  // zero term adds nothing, so the sums start as the bare pixel values.
  const auto ring_slot = [](int q) { return ((q >> 5) % 3) * 32 + (q & 31); };
  Vec4 head = sample_to_vec(kAssoc, ring_pix[0]);
  Vec4 run;
  {
    const int q = 1 + lane;
    run = (lane < 15 && q < n) ? sample_to_vec(kAssoc, ring_pix[ring_slot(q)])
                               : Vec4{0.0, 0.0, 0.0, 0.0};
  }
  Vec4 e{0.0, 0.0, 0.0, 0.0};
  int my_index = 0;

#pragma unroll 1
  for (int t = 0; t < n; ++t) {
    const int phase = t & 31;
    if (phase == 0 && t > 0) {
      // Chunk c+1 lands in its ring slot; chunk c+2's order load starts.
      const int c = t >> 5;
      const int slot = ((c + 1) % 3) * 32 + lane;
      ring_ord[slot] = ord_stage;
      ring_pix[slot] = pix_stage;
      const int q2 = 32 * (c + 2) + lane;
      ord_stage = (q2 < n) ? order[q2] : -1;
      __syncwarp();
    } else if (phase == 16) {
      if (ord_stage >= n) {
        atomicExch(L.status, kDevBadItem);
        ord_stage = 0;
      }
      pix_stage = (ord_stage >= 0) ? load_sample(img, layout, stride, width, ord_stage)
                                   : make_float4(0.f, 0.f, 0.f, 0.f);
    }

    // (1) The head pixel's target: the only FP64 work on the chain.
    Vec4 v;
    v.r = __dadd_rn(head.r, __dmul_rn(w15, e.r));
    v.g = __dadd_rn(head.g, __dmul_rn(w15, e.g));
    v.b = __dadd_rn(head.b, __dmul_rn(w15, e.b));
    if (kAssoc) v.a = __dadd_rn(head.a, __dmul_rn(w15, e.a));

    // (2) Fold e_{t-1} into the upcoming pixels' sums and shift them down.
    {
      Vec4 rn;
      rn.r = __dadd_rn(run.r, __dmul_rn(wl, e.r));
      rn.g = __dadd_rn(run.g, __dmul_rn(wl, e.g));
      rn.b = __dadd_rn(run.b, __dmul_rn(wl, e.b));
      rn.a = kAssoc ? __dadd_rn(run.a, __dmul_rn(wl, e.a)) : 0.0;
      head = shfl_vec(rn, 0, kAssoc);
      run = shfl_down_vec(rn, kAssoc);
      const int q = t + 16;
      const Vec4 fresh = (q < n) ? sample_to_vec(kAssoc, ring_pix[ring_slot(q)])
                                 : Vec4{0.0, 0.0, 0.0, 0.0};
      if (lane == 14) run = fresh;
    }

    // (3) ClampPixel narrows through float (rd_types.h:39-43).
    const float fr = clamp_pixel(v.r);
    const float fg = clamp_pixel(v.g);
    const float fb = clamp_pixel(v.b);
    const float fa = kAssoc ? clamp_pixel(v.a) : 0.0f;

    // (4) Memo key and lookup.
    unsigned key = key6_dev(fr) | (key6_dev(fg) << 6) | (key6_dev(fb) << 12);
    if (kAssoc) key |= key6_dev(fa) << 18;
    int index;
    bool found = false;
    unsigned h24 = 0, slot = 0;
    if (use_cache) {
      h24 = (key * 0x9E3779B1u) & 0xFFFFFFu;
      slot = h24 >> tag_bits;
      const unsigned ent = cache[slot];
      index = static_cast<int>(ent & 0xFFu);
      found = (ent >> 8) == (0x800000u | (h24 & tag_mask));
      if (!found) {
        const unsigned g = memo[key];
        if ((g >> 8) == gen) {
          index = static_cast<int>(g & 0xFFu);
          found = true;
        }
      }
    }
    if (!found) {
      // First touch (or no memo): descend and search the subtree
      // (src/rd_riemersma_cpu.cpp:77-92).
      const unsigned br = byte_dev(fr), bg = byte_dev(fg), bb = byte_dev(fb);
      const unsigned ba = kAssoc ? byte_dev(fa) : 0u;
      const int node = plan_descend(P, br, bg, bb, ba);
      const Target tg = make_target(kAssoc, static_cast<double>(fr), static_cast<double>(fg),
                                    static_cast<double>(fb), static_cast<double>(fa));
      index = plan_search_warp(P, node, tg, lane);
      if (use_cache) memo[key] = static_cast<uint16_t>((gen << 8) | static_cast<unsigned>(index));
    }
    if (use_cache) cache[slot] = 0x80000000u | ((h24 & tag_mask) << 8) | static_cast<unsigned>(index);

    // (5) Residual against the associated palette colour (rd_riemersma_cpu.cpp:104-112).
    const double* rc = P.rcol(index);
    e.r = __dadd_rn(static_cast<double>(fr), -rc[0]);
    e.g = __dadd_rn(static_cast<double>(fg), -rc[1]);
    e.b = __dadd_rn(static_cast<double>(fb), -rc[2]);
    if (kAssoc) e.a = __dadd_rn(static_cast<double>(fa), -rc[3]);

    if (lane == phase) my_index = index;
    if (phase == 31 || t == n - 1) {
      const int q = (t & ~31) + lane;
      if (q <= t) {
        const int rs = ring_slot(q);
        const int o = ring_ord[rs];
        it.indices[o] = static_cast<uint8_t>(my_index);
        if (it.rgba_out) {
          const float4 pc = reinterpret_cast<const float4*>(it.plan + P.h->off_out)[my_index];
          const float a = kAssoc ? pc.w : ring_pix[rs].w;
          it.rgba_out[o] = make_float4(pc.x, pc.y, pc.z, a);
        }
      }
      __syncwarp();
    }
  }
}

__global__ void __launch_bounds__(32) SeqWalkKernel(SeqLaunch L) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x;
  unsigned char* plan_smem = smem;
  uint32_t* cache = reinterpret_cast<uint32_t*>(smem + L.plan_smem_max);
  const int cache_entries = L.use_cache ? (1 << L.cache_bits) : 0;
  // The ring's float4 half needs 16-byte alignment whatever the cache size.
  const int ring_off = (L.plan_smem_max + 4 * cache_entries + 15) & ~15;
  int32_t* ring_ord = reinterpret_cast<int32_t*>(smem + ring_off);
  float4* ring_pix = reinterpret_cast<float4*>(ring_ord + kRing);

  uint16_t* memo = L.use_cache ? L.memo + static_cast<int64_t>(blockIdx.x) * L.slab_entries
                               : nullptr;
  unsigned gen = L.use_cache ? L.memo_gen[blockIdx.x] : 0u;

#pragma unroll 1
  for (;;) {
    int item_id = 0;
    if (lane == 0) item_id = atomicAdd(L.work_counter, 1);
    item_id = __shfl_sync(0xffffffffu, item_id, 0);
    if (item_id >= L.n_items) break;
    const SeqItem it = L.items[item_id];
    if (it.n <= 0) continue;
    if (it.plan_smem > L.plan_smem_max) {
      if (lane == 0) atomicExch(L.status, kDevBadPlan);
      continue;
    }
    // Stage the plan (a multiple of 16 bytes).
    {
      const int4* src = reinterpret_cast<const int4*>(it.plan);
      int4* dst = reinterpret_cast<int4*>(plan_smem);
      for (int i = lane; i < it.plan_smem / 16; i += 32) dst[i] = src[i];
    }
    if (L.use_cache) {
      for (int i = lane; i < cache_entries; i += 32) cache[i] = 0u;
      // Next generation; at the wrap the slab is cleared once.
      gen += 1;
      if (gen > 255u) {
        gen = 1;
        const int64_t words = L.slab_entries / 8;
        int4* m = reinterpret_cast<int4*>(memo);
        for (int64_t i = lane; i < words; i += 32) m[i] = make_int4(0, 0, 0, 0);
        __threadfence_block();
      }
    }
    __syncwarp();
    PlanView P;
    P.bind(plan_smem);
    if (P.assoc) {
      WalkOne<true>(it, L, P, cache, L.cache_bits, ring_ord, ring_pix, memo, gen, lane);
    } else {
      WalkOne<false>(it, L, P, cache, L.cache_bits, ring_ord, ring_pix, memo, gen, lane);
    }
    __syncwarp();
  }
  if (lane == 0 && L.use_cache) L.memo_gen[blockIdx.x] = gen;
}

}  // namespace

std::size_t SeqSmemBytes(int plan_smem_max, int cache_bits, bool use_cache) {
  const std::size_t ring_off =
      (static_cast<std::size_t>(plan_smem_max) +
       (use_cache ? (static_cast<std::size_t>(4) << cache_bits) : 0) + 15) & ~static_cast<std::size_t>(15);
  return ring_off + kRing * (sizeof(int32_t) + sizeof(float4));
}

cudaError_t LaunchSeqWalk(const SeqLaunch& L, int grid, cudaStream_t stream) {
  const std::size_t smem = SeqSmemBytes(L.plan_smem_max, L.cache_bits, L.use_cache != 0);
  cudaError_t e = AllowMaxSmem(SeqWalkKernel);
  if (e != cudaSuccess) return e;
  SeqWalkKernel<<<grid, 32, smem, stream>>>(L);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------
// The allocation-free sequential walk (rdb_dither_seq_noalloc in rdb.h).
//
// Everything the walk needs beyond the caller's pixels and index map -- the
// memo table, the visit order, the curve-builder scratch, the palette plan
// and the launch descriptor -- lives in one fixed array in device memory that
// the library declares at file scope.  Every GPU that loads the library holds
// it (a little over 5 MiB) until the process exits.  Host code never uses the
// array's name as an address: the device address is fetched once per device
// with cudaGetSymbolAddress.
namespace noalloc {

constexpr int kMaxSide = 4096;
constexpr int64_t kMaxPixels = int64_t{1} << 20;
constexpr std::size_t kMemoEntries = std::size_t{1} << 18;  // RGB keys: 6 bits per channel
constexpr std::size_t kOffMemo = 0;
constexpr std::size_t kOffMisc = kOffMemo + kMemoEntries * sizeof(uint16_t);  // 512 KiB
constexpr std::size_t kOffItem = kOffMisc + 256;   // gen (4 B), counter (4 B), status (4 B)
constexpr std::size_t kOffPlan = kOffItem + 256;
constexpr std::size_t kPlanBytes = 64 * 1024;
constexpr std::size_t kOffCurve = kOffPlan + kPlanBytes;
constexpr std::size_t kCurveBytes = 512 * 1024;
constexpr std::size_t kOffOrder = kOffCurve + kCurveBytes;
constexpr std::size_t kBytes = kOffOrder + static_cast<std::size_t>(kMaxPixels) * sizeof(int32_t);
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kBytes];

std::mutex g_mu;
unsigned char* g_base[kMaxDevices] = {};

// Device address of g_scratch for the current device, looked up on the first
// call made on that device.
cudaError_t Base(int device, unsigned char** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_base[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return e;
    g_base[device] = static_cast<unsigned char*>(p);
  }
  *out = g_base[device];
  return cudaSuccess;
}

// Writes the call's launch descriptor into the array and clears the work
// counter and the status word.  The descriptor travels as a kernel parameter,
// so no host buffer of the call has to outlive it.
__global__ void Stage(SeqItem item, SeqItem* dst, uint32_t* misc) {
  if (threadIdx.x == 0) {
    *dst = item;
    misc[1] = 0u;
    misc[2] = 0u;
  }
}

}  // namespace noalloc

}  // namespace rdb

extern "C" int rdb_dither_seq_noalloc(const void* plan, size_t plan_bytes, const void* pixels,
                                      size_t row_stride, int width, int height, int layout,
                                      uint8_t* indices, double diffusion, int use_cache,
                                      void* stream) {
  using namespace rdb;
  namespace na = rdb::noalloc;
  if (!plan || !pixels || !indices) return Fail(RDB_E_INVALID, "rdb_dither_seq_noalloc: null argument");
  if (width < 1 || height < 1) return Fail(RDB_E_INVALID, "image must be at least 1x1");
  if (width > na::kMaxSide || height > na::kMaxSide ||
      static_cast<int64_t>(width) * height > na::kMaxPixels) {
    return Fail(RDB_E_UNSUPPORTED,
                "rdb_dither_seq_noalloc handles at most 4096 pixels per side and 1048576 pixels "
                "(its scratch is a fixed 5 MiB device array); use rdb_dither for larger images");
  }
  if (layout != RDB_RGB8 && layout != RDB_RGBA8 && layout != RDB_RGBAF32) {
    return Fail(RDB_E_INVALID, "unknown pixel layout");
  }
  const std::size_t bpp = layout == RDB_RGBAF32 ? 16 : static_cast<std::size_t>(layout);
  const std::size_t stride = row_stride ? row_stride : static_cast<std::size_t>(width) * bpp;
  if (stride < static_cast<std::size_t>(width) * bpp) return Fail(RDB_E_INVALID, "row stride shorter than a row");
  if ((layout == RDB_RGBAF32 && ((reinterpret_cast<uintptr_t>(pixels) | stride) & 15u)) ||
      (layout == RDB_RGBA8 && ((reinterpret_cast<uintptr_t>(pixels) | stride) & 3u))) {
    return Fail(RDB_E_INVALID, "pixels or row stride misaligned for the layout");
  }
  if (plan_bytes < sizeof(PlanHeader)) return Fail(RDB_E_INVALID, "plan blob too short");
  PlanHeader h;
  std::memcpy(&h, plan, sizeof(h));
  if (h.total_bytes != static_cast<int32_t>(plan_bytes) || h.smem_bytes <= 0 ||
      h.smem_bytes > h.total_bytes || h.count < 1 || h.count > kMaxPaletteColors) {
    return Fail(RDB_E_INVALID, "not a plan blob from rdb_plan_build");
  }
  if (h.assoc) {
    return Fail(RDB_E_UNSUPPORTED,
                "rdb_dither_seq_noalloc takes palettes without associated alpha only (an alpha "
                "memo table has 2^24 keys and does not fit the fixed scratch)");
  }
  if (plan_bytes > na::kPlanBytes) return Fail(RDB_E_UNSUPPORTED, "palette plan larger than 64 KiB");
  const int level = CurveLevel(width, height);
  if (CurveScratchBytes(level) > na::kCurveBytes) return Fail(RDB_E_UNSUPPORTED, "curve scratch too small");

  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return CudaFail(e, "cudaGetDevice");
  if (device < 0 || device >= na::kMaxDevices) return Fail(RDB_E_UNSUPPORTED, "device index too large");
  unsigned char* base = nullptr;
  if ((e = na::Base(device, &base)) != cudaSuccess) return CudaFail(e, "cudaGetSymbolAddress");
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  uint32_t* misc = reinterpret_cast<uint32_t*>(base + na::kOffMisc);  // [0] gen, [1] counter, [2] status
  int32_t* order = reinterpret_cast<int32_t*>(base + na::kOffOrder);
  unsigned char* dplan = base + na::kOffPlan;
  SeqItem item{};
  item.pixels = static_cast<const unsigned char*>(pixels);
  item.row_stride = static_cast<int64_t>(stride);
  item.width = width;
  item.height = height;
  item.layout = layout;
  item.n = width * height;
  item.order = order;
  item.indices = indices;
  item.rgba_out = nullptr;
  item.plan = dplan;
  item.plan_smem = h.smem_bytes;
  // The counter and status start at zero on every call; the memo slab keeps
  // its contents and is told apart by the generation in misc[0].  The plan is
  // copied from the caller's buffer, which must stay unchanged until the
  // stream reaches this call (from pinned memory the copy is asynchronous).
  if ((e = cudaMemcpyAsync(dplan, plan, plan_bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess) {
    return CudaFail(e, "rdb_dither_seq_noalloc plan copy");
  }
  na::Stage<<<1, 32, 0, s>>>(item, reinterpret_cast<SeqItem*>(base + na::kOffItem), misc);
  if ((e = cudaGetLastError()) != cudaSuccess) return CudaFail(e, "rdb_dither_seq_noalloc staging");
  if ((e = BuildSeqOrder(width, height, order, base + na::kOffCurve, na::kCurveBytes, s)) != cudaSuccess) {
    return CudaFail(e, "visit order kernel");
  }
  SeqLaunch L{};
  L.items = reinterpret_cast<const SeqItem*>(base + na::kOffItem);
  L.n_items = 1;
  L.work_counter = reinterpret_cast<int*>(misc + 1);
  L.memo = reinterpret_cast<uint16_t*>(base + na::kOffMemo);
  L.memo_gen = misc;
  L.slab_entries = static_cast<int64_t>(na::kMemoEntries);
  L.use_cache = use_cache ? 1 : 0;
  L.cache_bits = use_cache ? 15 : 0;
  L.plan_smem_max = h.smem_bytes;
  while (use_cache && L.cache_bits > 8 && SeqSmemBytes(L.plan_smem_max, L.cache_bits, true) > 227 * 1024) {
    --L.cache_bits;
  }
  scaled_weights(diffusion, L.sw);
  L.status = reinterpret_cast<int*>(misc + 2);
  if ((e = LaunchSeqWalk(L, 1, s)) != cudaSuccess) return CudaFail(e, "sequential walk launch");
  return RDB_OK;
}
