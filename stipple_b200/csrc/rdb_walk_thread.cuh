// rdb_walk_thread.cuh -- the thread walker: one thread advances one chain.
//
// Thirty-two independent chains share every warp instruction, so the walk is
// issue- and FP64-bound rather than latency-bound, given enough warps.  The
// block engine (independent blocks) and the speculative segmented walk
// (independent segments) both run on it.
//
// Per position (src/rd_riemersma_cpu.cpp:647-696): the 16-term error sum is
// kept as running sums of the next 16 pixels in registers R[16][C]; a 16-way
// unroll rotates their names instead of moving data, so each residual costs
// exactly its 16 x C products and sums (the minimum the reference's operation
// order allows).  The weights are kernel parameters and enter the FP64
// instructions as constant operands.  The lookup is the octree descent -- the
// first three levels as one table read -- and a thread-serial scan of the
// stopping node's run of post-order slots over slot-ordered, channel-planar
// colour rows.
#pragma once

#include <cstdint>

#include "rdb_device.cuh"

namespace rdb {
namespace tw {

struct Plan {
  const PlanHeader* h;
  const unsigned char* pal;
  const int16_t* child;
  const uint16_t* range;
  const uint8_t* seq;
  const double* slotpal;
  const uint16_t* jump;
  int fan;
  int stride;
  int slot_stride;

  __device__ __forceinline__ void bind(const unsigned char* base) {
    h = reinterpret_cast<const PlanHeader*>(base);
    pal = base + h->off_pal;
    child = reinterpret_cast<const int16_t*>(base + h->off_child);
    range = reinterpret_cast<const uint16_t*>(base + h->off_range);
    seq = base + h->off_seq;
    slotpal = reinterpret_cast<const double*>(base + h->off_slotpal);
    jump = reinterpret_cast<const uint16_t*>(base + h->off_jump);
    fan = h->fan;
    stride = h->pal_stride;
    slot_stride = h->slot_stride;
  }
  template <bool kAssoc>
  __device__ __forceinline__ const double* rcol(int i) const {
    return reinterpret_cast<const double*>(pal + i * stride) + (kAssoc ? 4 : 0);
  }
};

// Descent (src/rd_riemersma_cpu.cpp:82-89): the jump table covers levels 1-3.
template <bool kAssoc>
__device__ __forceinline__ int descend(const Plan& P, unsigned br, unsigned bg, unsigned bb,
                                       unsigned ba) {
  unsigned idx = (br >> 5) | ((bg >> 5) << 3) | ((bb >> 5) << 6);
  if (kAssoc) idx |= (ba >> 5) << 9;
  const unsigned jt = P.jump[idx];
  int node = static_cast<int>(jt & 0x7FFFu);
  if (!(jt & 0x8000u)) {
#pragma unroll 1
    for (int i = kMaxTreeDepth - 1 - kJumpLevels; i > 0; --i) {
      int id = static_cast<int>(((br >> i) & 1u) | (((bg >> i) & 1u) << 1) | (((bb >> i) & 1u) << 2));
      if (kAssoc) id |= static_cast<int>(((ba >> i) & 1u) << 3);
      const int c = P.child[node * (kAssoc ? 16 : 8) + id];
      if (c < 0) break;
      node = c;
    }
  }
  return node;
}

// ClosestColor over the run of slots (src/rd_octree.cpp:178-217): minimum
// full distance, the last equal minimum in post-order winning.  Returns the
// colour number.
template <bool kAssoc>
__device__ __forceinline__ int search(const Plan& P, int node, double tr, double tg, double tb,
                                      double ta) {
  const int start = P.range[2 * node];
  const int len = P.range[2 * node + 1];
  const double* dr = P.slotpal;
  const double* dg = dr + P.slot_stride;
  const double* db = dg + P.slot_stride;
  const double* da = db + P.slot_stride;
  double best = kSearchStart;
  int slot = -1;
#pragma unroll 2
  for (int s = start; s < start + len; ++s) {
    const double x = __dadd_rn(dr[s], -tr);
    const double y = __dadd_rn(dg[s], -tg);
    const double z = __dadd_rn(db[s], -tb);
    double d = __dmul_rn(x, x);
    d = __dadd_rn(d, __dmul_rn(y, y));
    d = __dadd_rn(d, __dmul_rn(z, z));
    if (kAssoc) {
      const double w = __dadd_rn(da[s], -ta);
      d = __dadd_rn(d, __dmul_rn(w, w));
    }
    if (d <= best) {
      best = d;
      slot = s;
    }
  }
  return slot < 0 ? 0 : static_cast<int>(P.seq[slot]);
}

// ClosestColor restricted to a key's survivors (a candidate-table entry,
// rdb_cand.h: up to four slots in ascending post-order, the last repeated):
// the same distances in the same order with the same "<=", so the same winner.
__device__ __forceinline__ int search_survivors(const Plan& P, uint32_t cand, double tr, double tg,
                                                double tb) {
  const double* dr = P.slotpal;
  const double* dg = dr + P.slot_stride;
  const double* db = dg + P.slot_stride;
  double best = kSearchStart;
  int slot = static_cast<int>(cand & 0xFFu);
  unsigned prev = 0x100u;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const unsigned s = (cand >> (8 * i)) & 0xFFu;
    if (s == prev) break;
    prev = s;
    const double x = __dadd_rn(dr[s], -tr);
    const double y = __dadd_rn(dg[s], -tg);
    const double z = __dadd_rn(db[s], -tb);
    double d = __dmul_rn(x, x);
    d = __dadd_rn(d, __dmul_rn(y, y));
    d = __dadd_rn(d, __dmul_rn(z, z));
    if (d <= best) {
      best = d;
      slot = static_cast<int>(s);
    }
  }
  return static_cast<int>(P.seq[slot]);
}

// The same search spread over the 32 lanes of a warp for ONE target (every
// lane passes the same node and target): lane l scans slots start+l,
// start+l+32, ..., keeping its last minimum; the butterfly then keeps the
// smaller distance and, between equal distances, the later slot -- the
// reference's "last equal minimum in post-order" rule.  All 32 lanes must
// call it together.
template <bool kAssoc>
__device__ __forceinline__ int search_warp(const Plan& P, int node, double tr, double tg,
                                           double tb, double ta, int lane) {
  const int start = P.range[2 * node];
  const int len = P.range[2 * node + 1];
  const double* dr = P.slotpal;
  const double* dg = dr + P.slot_stride;
  const double* db = dg + P.slot_stride;
  const double* da = db + P.slot_stride;
  double best = kSearchStart;
  int slot = -1;
#pragma unroll 1
  for (int s = start + lane; s < start + len; s += 32) {
    const double x = __dadd_rn(dr[s], -tr);
    const double y = __dadd_rn(dg[s], -tg);
    const double z = __dadd_rn(db[s], -tb);
    double d = __dmul_rn(x, x);
    d = __dadd_rn(d, __dmul_rn(y, y));
    d = __dadd_rn(d, __dmul_rn(z, z));
    if (kAssoc) {
      const double w = __dadd_rn(da[s], -ta);
      d = __dadd_rn(d, __dmul_rn(w, w));
    }
    if (d <= best) {
      best = d;
      slot = s;
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, off);
    const int os = __shfl_xor_sync(0xffffffffu, slot, off);
    if (ob < best || (ob == best && os > slot)) {
      best = ob;
      slot = os;
    }
  }
  return slot < 0 ? 0 : static_cast<int>(P.seq[slot]);
}

}  // namespace tw
}  // namespace rdb
