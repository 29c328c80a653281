// rdb_uniform.h -- memo keys on which the colour search cannot vary.
//
// The memo key (rd_types.h:141-153) keeps the top 6 bits of each channel's
// byte, so one key stands for a box of targets.  The lookup descends the tree
// by byte bits 7..1 and runs ClosestColor over the stopping node's parent
// (src/rd_riemersma_cpu.cpp:82-92, src/rd_octree.cpp:178-217).  When every
// target in the box stops at the same node and one candidate of that node's
// run is nearer than every other by a margin over the whole box, every
// target in the box gets that candidate: the search result is a function of
// the key alone.  Such a key is uniform.  Its memo value is that candidate
// whichever target touched the key first, so an exact walk may take it
// without consulting any memo, and a cache-free walk without searching.
//
// Distances are affine in the target once the squared terms cancel:
// d(x, w) - d(x, j) = sum_c (w_c^2 - j_c^2) - 2 x_c (w_c - j_c), so its
// maximum over the box sits at a corner chosen channel by channel.  The
// margin (1.0 in squared Q16 units) dwarfs the double rounding of distances
// below 2^35, so the walk's own comparisons cannot disagree.
//
// Palettes without associated alpha only (2^18 keys).  One byte per key: the
// colour number, or kNotUniform (also used for colour 255, which is then
// always looked up).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace rdb {

constexpr int kUniformKeys = 1 << 18;
constexpr uint8_t kNotUniform = 0xFF;
constexpr int kUniformKeysAlpha = 1 << 24;  // alpha-associated palettes (rdb_uniform_alpha.cuh)
constexpr uint8_t kUniformUnknown = 0xFE;   // their lazily filled entries: not yet classified

// `plan`: a device plan blob (rdb_plan.h); `out`: kUniformKeys bytes.
cudaError_t LaunchUniformTable(const unsigned char* plan, uint8_t* out, cudaStream_t s);

// Alpha-associated palettes (rdb_uniform_alpha.cuh): 2^24 bytes, classified
// lazily by the walk (0xFE = not yet); this classifies every key still 0xFE.
cudaError_t LaunchUniformTableAlpha(const unsigned char* plan, uint8_t* out, cudaStream_t s);

}  // namespace rdb
