// rdb_curve.cu -- the Riemersma visit order on the device.
//
// The sequential walk visits the order-L Hilbert curve (L = ceil(log2 of the
// longer side), include/rd_riemersma.h:88-94) clipped to the image: the
// recursion's 4^L - 1 leaves plus the trailing visit at the resting cursor
// (2^L-1, 0), which is exactly HilbertPoint(n) for n in [0, 4^L)
// (src/rd_riemersma_cpu.cpp:167-189, 403-416).  Every in-image pixel appears
// once, so the order is a permutation of the W*H pixel indices.
//
// The block and Jacobi engines use BuildCurveIndex's list instead
// (src/rd_riemersma_cpu.cpp:269-356): n in [0, 4^L - 1) plus the origin
// appended.  That is this order with the cell (2^L-1, 0) dropped when it is in
// the image (it is the last element here) and pixel 0 appended; the engines
// derive it on the fly and never store a second table.
//
// Work is cut into tiles of 4^k consecutive curve indices (k = min(L, 5)):
// each tile is an aligned 2^k x 2^k square, so its in-image count is a
// rectangle intersection computed in O(1).  A scan of the counts gives every
// tile its output offset, and only tiles that touch the image are enumerated
// -- a 4096x64 strip at L = 12 touches 256 of 16384 tiles.
#include <cub/cub.cuh>

#include "rdb_curve.h"
#include "rdb_device.cuh"

namespace rdb {
namespace {

__global__ void TileCounts(int width, int height, int level, int k, int64_t tiles,
                           uint32_t* counts) {
  const int64_t m = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (m >= tiles) return;
  int x, y;
  hilbert_point(static_cast<uint64_t>(m) << (2 * k), level, x, y);
  const int side = 1 << k;
  const int x0 = (x >> k) << k;
  const int y0 = (y >> k) << k;
  const int cw = min(max(width - x0, 0), side);
  const int ch = min(max(height - y0, 0), side);
  counts[m] = static_cast<uint32_t>(cw) * static_cast<uint32_t>(ch);
}

// One CTA of 256 threads per tile; each thread owns 4^k/256 consecutive cells
// (k = 5: 4 cells).  For k < 4 a single warp-sized tile is handled by the
// same code with idle threads.
__global__ void __launch_bounds__(256) TileEmit(int width, int height, int level, int k,
                                                const uint32_t* counts,
                                                const uint32_t* offsets, int32_t* order) {
  const int64_t m = blockIdx.x;
  const uint32_t count = counts[m];
  if (count == 0) return;
  const uint32_t base = offsets[m];
  const int cells = 1 << (2 * k);
  const int per = (cells + 255) / 256;
  const int t = threadIdx.x;
  const uint64_t n0 = (static_cast<uint64_t>(m) << (2 * k)) + static_cast<uint64_t>(t) * per;
  int pix[4];
  int mine = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    pix[j] = -1;
    if (j < per && t * per + j < cells) {
      int x, y;
      hilbert_point(n0 + j, level, x, y);
      if (x < width && y < height) {
        pix[j] = y * width + x;
        ++mine;
      }
    }
  }
  if (count == static_cast<uint32_t>(cells)) {
    // Whole tile inside: rank is the cell's own position.
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (pix[j] >= 0) order[base + t * per + j] = pix[j];
    }
    return;
  }
  using Scan = cub::BlockScan<int, 256>;
  __shared__ typename Scan::TempStorage tmp;
  int rank = 0;
  Scan(tmp).ExclusiveSum(mine, rank);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (pix[j] >= 0) order[base + rank++] = pix[j];
  }
}

}  // namespace

int CurveLevel(int64_t width, int64_t height) {
  const int64_t extent = width > height ? width : height;
  if (extent <= 1) return 0;
  int level = 0;
  while ((static_cast<int64_t>(1) << level) < extent) ++level;
  return level;
}

std::size_t CurveScratchBytes(int level) {
  const int k = level < 5 ? level : 5;
  const int64_t tiles = static_cast<int64_t>(1) << (2 * (level - k));
  std::size_t scan_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, static_cast<const uint32_t*>(nullptr),
                                static_cast<uint32_t*>(nullptr), static_cast<int>(tiles));
  return 2 * static_cast<std::size_t>(tiles) * sizeof(uint32_t) + 256 + scan_bytes;
}

cudaError_t BuildSeqOrder(int width, int height, int32_t* order, void* scratch,
                          std::size_t scratch_bytes, cudaStream_t stream) {
  const int level = CurveLevel(width, height);
  if (level == 0) return cudaMemsetAsync(order, 0, sizeof(int32_t), stream);
  const int k = level < 5 ? level : 5;
  const int64_t tiles = static_cast<int64_t>(1) << (2 * (level - k));
  uint32_t* counts = static_cast<uint32_t*>(scratch);
  uint32_t* offsets = counts + tiles;
  void* scan_tmp = reinterpret_cast<unsigned char*>(offsets + tiles) + 256 -
                   (reinterpret_cast<uintptr_t>(offsets + tiles) & 255u);
  std::size_t scan_bytes = scratch_bytes - (static_cast<unsigned char*>(scan_tmp) -
                                            static_cast<unsigned char*>(scratch));
  TileCounts<<<static_cast<unsigned>((tiles + 255) / 256), 256, 0, stream>>>(width, height, level,
                                                                          k, tiles, counts);
  cudaError_t e = cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, counts, offsets,
                                                static_cast<int>(tiles), stream);
  if (e != cudaSuccess) return e;
  TileEmit<<<static_cast<unsigned>(tiles), 256, 0, stream>>>(width, height, level, k, counts,
                                                           offsets, order);
  return cudaGetLastError();
}

}  // namespace rdb
