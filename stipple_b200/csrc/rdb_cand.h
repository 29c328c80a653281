// rdb_cand.h -- per memo key, the palette slots that can win its search.
//
// The lookup (src/rd_riemersma_cpu.cpp:82-92) descends by byte bits 7..1 and
// runs ClosestColor (src/rd_octree.cpp:178-217) over the stopping node's
// parent's post-order run; the memo key keeps the top 6 bits of each byte, so
// one key stands for a box of targets (rdb_uniform.h).  When every target of
// the box stops at the same node, a slot j of the run can only win if no
// other slot w is nearer than j by a margin everywhere in the box: the
// distance difference d(x, w) - d(x, j) is affine in the target, so its
// maximum over the box sits at a corner chosen channel by channel.  The slots
// that survive that test, in ascending post-order, are the only ones the
// search has to evaluate; evaluating them in that order with the reference's
// "<=" keeps its result, ties included, because a dominated slot is strictly
// farther than the winner (the margin, 1.0 in squared Q16 units, dwarfs the
// double rounding of distances below 2^35).
//
// One 32-bit entry per key (2^18 keys, palettes without associated alpha):
// up to four survivor slots, one per byte in ascending order, the last one
// repeated into the unused bytes -- byte 0 == byte 1 means a single survivor
// (the key is uniform: no distance needs computing); byte 0 > byte 1 marks a
// key the table does not cover (the descent varies inside its box, or more
// than four slots survive), which the walk searches in full.  On the
// synthetic 256-colour workloads about 80 % of keys have one survivor, 17 %
// two, 3 % three and 0.05 % need the full search, against a mean run of
// about 87 slots.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace rdb {

constexpr int kCandKeys = 1 << 18;
constexpr uint32_t kCandFallback = 0x000000FFu;
constexpr double kCandMargin = 1.0;

// `plan`: a device plan blob (rdb_plan.h) without associated alpha; `out`:
// kCandKeys words.
cudaError_t LaunchCandidateTable(const unsigned char* plan, uint32_t* out, cudaStream_t s);

}  // namespace rdb
