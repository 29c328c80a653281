// rdb_plan.h -- the device-resident form of one palette and its colour tree.
//
// The Riemersma lookup (src/rd_riemersma_cpu.cpp:82-92) descends the octree
// by the pixel's bits, stops at the first missing child, and runs
// ClosestColor (src/rd_octree.cpp:178-217) over the subtree of the stopping
// node's PARENT in post-order, the last equal-minimum candidate winning.
//
// A subtree is a contiguous run of the post-order sequence, so the plan
// stores, per live node, the run [start, start+len) of post-order "slots"
// that the lookup searches when the descent stops at that node; `seq[slot]`
// is the colour number at that slot.  For trees built by the octree the
// colour numbers are assigned in the same post-order (rd_octree.cpp:142-176)
// so seq[slot] == slot, but the plan does not rely on it.  The search is then
// a range argmin -- minimum distance, ties to the highest slot -- which a
// warp evaluates in parallel.
//
// Layout (one blob, 16-byte aligned sections, staged into shared memory by
// the kernels; `out` is not staged):
//   PlanHeader
//   pal   count x PalEntry   distance-side and residual-side colours
//   child nodes x fan x int16 live child ids (-1 = none)
//   range nodes x {uint16 start, uint16 len}
//   seq   slots x uint8
//   out   count x float4     (float)entry, for the RgbaF scatter
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace rdb {

constexpr int kMaxPaletteColors = 256;   // one palette index per byte
constexpr int kMaxPlanNodes = 8192;

struct PlanHeader {
  int32_t count;      // palette entries
  int32_t assoc;      // associate_alpha
  int32_t nodes;      // live nodes (root = 0)
  int32_t fan;        // 8 or 16 children
  int32_t slots;      // coloured nodes in post-order
  int32_t smem_bytes; // bytes staged into shared memory (everything before `out`)
  int32_t total_bytes;
  int32_t off_pal;
  int32_t off_child;
  int32_t off_range;
  int32_t off_seq;
  int32_t off_out;
  int32_t pal_stride; // bytes per PalEntry: 32 (no alpha) or 64 (alpha)
  int32_t off_slotpal;  // channel-planar distance-side colours in slot order: 4 x slot_stride doubles
  int32_t off_jump;     // descent after the first kJumpLevels levels, indexed by the top bits
  int32_t slot_stride;  // doubles per channel row of slotpal (slots rounded up to even)
};
// The first three levels of the descent collapse into one table lookup: the
// index is the top three bits of each channel's byte (r | g << 3 | b << 6 |
// a << 9), the entry the live node reached (bit 15 set when the descent had
// already stopped at a missing child within those levels).
constexpr int kJumpLevels = 3;
static_assert(sizeof(PlanHeader) == 64, "header is one 64-byte block");

// Without alpha the distance-side and residual-side colours coincide, so an
// entry is {r, g, b, a} (32 B).  With alpha it is
// {dr, dg, db, a, cr, cg, cb, a}: d* = (QS*a)*c as ClosestColor forms it
// (rd_octree.cpp:193-196), c* = AssociateAlphaPixelInfo (rd_types.h:195-208).

struct PlanInput {
  int count = 0;
  bool assoc = false;
  const double* colors = nullptr;         // count x 4: palette.entries (output, residual)
  const double* search_colors = nullptr;  // count x 4: the tree's colormap (distance)
  int node_count = 0;
  int root = 0;
  const int32_t* child = nullptr;         // node_count x 16
  const int32_t* parent = nullptr;        // node_count (may be null)
  const uint32_t* color_number = nullptr; // node_count
  const uint64_t* number_unique = nullptr;// node_count
};

// Builds the blob.  Returns an empty string on success, else why the input
// cannot be planned (palette too large, colour number out of range, ...).
std::string BuildPlan(const PlanInput& in, std::vector<uint8_t>* blob);

}  // namespace rdb
