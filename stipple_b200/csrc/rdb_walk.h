// rdb_walk.h -- launch descriptors shared by the engines and the host runtime.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace rdb {

// One image walked by the sequential-exact engine.
struct SeqItem {
  const unsigned char* pixels;  // device, row-major, `layout`
  int64_t row_stride;           // bytes
  int width;
  int height;
  int layout;                   // 3 = RGB8, 4 = RGBA8, 16 = RGBA float (Q16)
  int n;                        // positions = width * height
  const int32_t* order;         // visit order (pixel indices), n entries
  uint8_t* indices;             // palette index per pixel, row-major
  float4* rgba_out;             // optional RgbaF result (may alias `pixels` for layout 16)
  const unsigned char* plan;    // device plan blob (rdb_plan.h)
  int plan_smem;                // PlanHeader::smem_bytes
  int pad;
};

struct SeqLaunch {
  const SeqItem* items;
  int n_items;
  int* work_counter;            // zero before launch
  uint16_t* memo;               // grid x slab_entries, generation-tagged
  uint32_t* memo_gen;           // per CTA: last generation used in its slab
  int64_t slab_entries;         // 2^18, or 2^24 when any item associates alpha
  int cache_bits;               // log2 of the shared-memory memo cache entries
  int plan_smem_max;            // bytes reserved for a plan in shared memory
  int use_cache;                // 0: --no-cache, every lookup searched
  int pad;
  double sw[16];                // scaled error weights
  int* status;
};

std::size_t SeqSmemBytes(int plan_smem_max, int cache_bits, bool use_cache);
cudaError_t LaunchSeqWalk(const SeqLaunch& L, int grid, cudaStream_t stream);

// The block engine: every image is cut into blocks of `block` consecutive
// positions of the block-mode list, each walked from a zeroed queue with no
// memo (src/rd_riemersma_cpu.cpp:632-697).
struct BlockImage {
  const unsigned char* pixels;
  int64_t row_stride;           // bytes (packed frames: width * bytes per pixel)
  int width;
  int height;
  int layout;                   // any RDB_* input format (rdb.h)
  int n;                        // block-list length (BlockListLength)
  const int32_t* order;         // sequential order of the geometry (W*H entries)
  uint8_t* indices;             // optional palette index per pixel, row-major
  float4* rgba_out;             // optional RgbaF result
  int64_t first_block;          // prefix over images
  int nblocks;
  int out_format;               // raw_out's format: RDB_RGBA16 or RDB_YUV444P8
  unsigned char* raw_out;       // optional encoder-format result
};

// Writes every pixel's source value into the image's outputs (RgbaF and/or
// raw) -- the result the block engine leaves where it visits nothing (a 1x1
// image).
cudaError_t LaunchSourceFill(const BlockImage& im, cudaStream_t stream);

// The walk's scratch is laid out for a warp: blocks are numbered across the
// launch's images and grouped 32 at a time (group g = block / 32, lane
// l = block % 32), and each block owns bpad positions (its length rounded up
// to a multiple of 16; positions past the block's end hold zeros).  Position t
// of block (g, l) sits at
//   packed samples  32-bit word ((g * bpad/4 + t/4) * 32 + l) * 4 + t % 4
//   float samples   float4      (g * bpad + t) * 32 + l
//   chosen indices  byte        ((g * bpad/16 + t/16) * 32 + l) * 16 + t % 16
// so a warp reads 4 positions of each of its 32 blocks with one 16-byte load
// per lane (512 contiguous bytes) and writes 16 indices per lane with one
// 16-byte store.
struct BlockLaunch {
  const BlockImage* images;
  int n_images;
  int block;                    // positions per block (>= 16)
  int64_t total_blocks;
  uint32_t* cx;                 // scratch: samples, laid out as above
  uint8_t* chosen;              // scratch: index per position, laid out as above
  const int64_t* pos_offset;    // per image: its first position among all images' lists
  const unsigned char* plan;    // one palette for the launch
  const uint32_t* cand;         // candidate table (rdb_cand.h), null with associated alpha
  int plan_smem;
  int assoc;                    // the palette associates alpha
  int is_float;                 // cx holds the sample widened to float4 (every layout but
                                // RGB8 / RGBA8, which pack into one word)
  int bpad;                     // positions per block in the scratch (multiple of 16)
  // Block sweeps (the Jacobi engine's default form): each block starts from
  // its predecessor's end queue of the previous sweep, q_in[(block - 1) * 64 ..]
  // (16 entries of 4 doubles, oldest first), where the predecessor is in the
  // same image; blocks that start an image, and every block when q_in is
  // null, start from zeros.  Each block writes its end queue to q_out
  // (when not null) and, when q_in is not null, counts into *changed the
  // blocks with a successor whose end queue differs from their q_in entry.
  const double* q_in;
  double* q_out;
  int* changed;
  double sw[16];
  int* status;
};

// Launch shapes of the walk kernel (threads per CTA, CTAs per SM); results do
// not depend on the shape.
constexpr int kBlockWalkShapes = 4;
void BlockWalkShape(int shape, bool assoc, int* threads, int* min_ctas);
cudaError_t LaunchBlockWalk(const BlockLaunch& L, int64_t total_positions, cudaStream_t stream,
                            int shape = 0);
// The three phases of LaunchBlockWalk separately (block sweeps walk many times
// between one gather and one scatter).
cudaError_t LaunchBlockGather(const BlockLaunch& L, cudaStream_t stream);
cudaError_t LaunchBlockWalkOnly(const BlockLaunch& L, cudaStream_t stream, int shape = 0);
cudaError_t LaunchBlockScatter(const BlockLaunch& L, int64_t total_positions, cudaStream_t stream);
// The chosen index of every position of every image, in list order, images
// back to back (`out`: total_positions bytes).
cudaError_t LaunchBlockChosenLinear(const BlockLaunch& L, int64_t total_positions, uint8_t* out,
                                    cudaStream_t stream);

// Writes every pixel's source value, as RgbaF, into `out` -- the result an
// engine that visits nothing leaves (a 1x1 image in block mode).
cudaError_t LaunchCopySource(const unsigned char* pixels, int64_t stride, int width, int height,
                             int layout, float4* out, cudaStream_t stream);

// The Jacobi engine (src/rd_approx_cuda.cu): an order-free fixed-point
// iteration t = q + F (x - q) along the block-mode list.
struct JacobiLaunch {
  const unsigned char* pixels;
  int64_t row_stride;
  int width;
  int height;
  int layout;
  int n;                        // block-list length
  const int32_t* order;
  uint8_t* indices;
  float4* rgba_out;
  const unsigned char* plan;
  int plan_smem;
  int iterations;
  int taps;
  int fp64;
  void* cx;                     // scratch: n x 4 samples (float or double)
  uint8_t* q0;                  // scratch: n
  uint8_t* q1;                  // scratch: n
  const double* g;              // taps + 1 filter coefficients (device)
  int* status;
};

cudaError_t LaunchJacobi(const JacobiLaunch& L, cudaStream_t stream);

}  // namespace rdb
