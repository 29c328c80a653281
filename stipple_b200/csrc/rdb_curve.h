// rdb_curve.h -- device construction of the Riemersma visit order.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace rdb {

// include/rd_riemersma.h:88-94 (ComputeCurveLevel): ceil(log2(max(w, h))),
// 0 for a 1x1 image.  Integer form; identical for every image size.
int CurveLevel(int64_t width, int64_t height);

// Scratch bytes BuildSeqOrder needs for an order-`level` curve.
std::size_t CurveScratchBytes(int level);

// Writes the W*H pixel indices of the sequential walk's visit order into
// `order` (device memory).
cudaError_t BuildSeqOrder(int width, int height, int32_t* order, void* scratch,
                          std::size_t scratch_bytes, cudaStream_t stream);

// The block-mode list (BuildCurveIndex, src/rd_riemersma_cpu.cpp:269-356) in
// terms of the sequential order of length n = W*H: the cell (2^L-1, 0) is in
// the image exactly when W == 2^L (L >= 1); it is then the last sequential
// entry and is dropped.  The list ends with the origin, pixel 0.
inline int64_t BlockListLength(int64_t width, int64_t height) {
  const int level = CurveLevel(width, height);
  if (level == 0) return 0;  // BuildCurveIndex returns an empty list at level 0
  const bool gap_in_image = width == (static_cast<int64_t>(1) << level);
  return width * height - (gap_in_image ? 1 : 0) + 1;
}

}  // namespace rdb
