// rdb_octree_dev.h -- the octree build's second classification loop on the
// device (rdb_octree_dev.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "rdb_octree.h"

namespace rdb {

struct OctreeRowsLaunch {
  const unsigned char* pixels;  // device, row-major
  int64_t row_stride;           // bytes
  int64_t width;
  int64_t y0;                   // first row of the loop
  int64_t pixels_n;             // width * (height - y0)
  int layout;                   // 3 = RGB8, 4 = RGBA8, 16 = RGBA float (Q16)
  int assoc;
  int levels;                   // the loop's depth
  int init_n;                   // nodes after the first loop (keys ascending)
  const uint64_t* init_keys;    // device
  const double* init_qerr;
  const uint64_t* init_count;
  const double* init_total;     // 4 per node
};

// Device bytes the loop needs for `pixels` pixels at `levels` levels.
std::size_t OctreeRowsScratch(int64_t pixels, int levels, bool assoc);
// Runs the loop and copies its result to the host (synchronous on `s`).
cudaError_t ClassifyRowsDevice(const OctreeRowsLaunch& L, void* scratch, std::size_t scratch_bytes,
                               cudaStream_t s, OctreeRows* out);

}  // namespace rdb
