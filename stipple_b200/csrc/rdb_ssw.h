// rdb_ssw.h -- the speculative segmented walk: an exact, parallel form of the
// sequential Riemersma walk.
//
// The walk (src/rd_riemersma_cpu.cpp:359-417) is a dependent chain whose
// whole state at a position is (a) the 16 most recent residuals and (b) the
// memo table: for every 6-bit-per-channel key touched so far, the index the
// FIRST target with that key received (rd_types.h:111-153).  Given the exact
// state at a position, the walk from there on is determined.
//
// The image's visit order is cut into K segments, each walked by one warp.
// Segment k starts from a guessed queue -- in pass 0 the end of a cache-free
// warm-up over the positions before it, later the predecessor's end queue
// from the previous pass -- and answers memo lookups from its own first
// touches, else from G, the previous pass's map of each key's EARLIEST first
// touch (segment, index), taken only when that segment precedes k.  Every
// run records the distinct keys it touched and how it answered each (its own
// first touch, or taken from G).
//
// After a pass, G is rebuilt from all runs and each segment is checked: its
// start queue must equal its predecessor's end queue bit for bit, each of its
// own first touches must have no earlier segment touching the same key, and
// each key it took from G must still come from an earlier segment with the
// same index.  By induction from segment 0 (which starts from the true zero
// queue and an empty memo), every segment in the checked prefix replayed the
// true walk exactly.  Unchecked segments run again from the new states; the
// prefix grows by at least one segment per pass, so the loop always ends, and
// in practice after a few passes.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace rdb {

struct SswImage {
  const unsigned char* pixels;
  int64_t row_stride;
  int width;
  int height;
  int layout;
  int n;                     // positions (= pixels)
  const int32_t* order;
  uint8_t* indices;
  float4* rgba_out;
  const unsigned char* plan;
  int plan_smem;
  int assoc;
  int first_seg;             // segments [first_seg, first_seg + nsegs)
  int nsegs;
  uint32_t* g_vals[2];       // G ping-pong: (segment << 8 | index), 0xFFFFFFFF = none
  uint32_t* g_keys[2];       // hashed G (alpha keys): key + 1, 0 = empty; null = direct 2^18 table
  uint32_t g_mask;           // hashed G capacity - 1
  int pad;
};

struct SswSeg {
  int image;
  int k;                     // index within its image
  int begin;
  int end;
  int warm;                  // warm-up positions walked before `begin` (pass 0)
  int run_tag;               // tag of the last run's L-table entries
};

struct SswLaunch {
  const SswImage* images;
  SswSeg* segs;
  const int* work;           // active segment ids
  int n_work;
  int pass;                  // G buffer parity: reads g_*[pass & 1], G build writes the other
  int tag;                   // L-table tag of this pass's runs (1..255)
  double* q_start;           // per segment: 16 x 4 doubles, oldest residual first
  double* q_end;
  uint64_t* ltab;            // per segment: 2^ltab_bits entries
  int ltab_bits;
  int use_cache;
  int cache_bits;            // shared-memory memo cache (4-byte entries)
  int plan_smem_max;
  int* counter;
  int* first_bad;            // per image
  int* status;
  double sw[16];
};

cudaError_t LaunchSswWalk(const SswLaunch& L, int grid, cudaStream_t s);
// Rebuilds G (the buffer the next pass reads) from every segment's L table.
cudaError_t LaunchSswBuildG(const SswLaunch& L, int total_segs, cudaStream_t s);
// Checks the active segments; records the first failing segment per image.
cudaError_t LaunchSswVerify(const SswLaunch& L, cudaStream_t s);
// RgbaF output of every image with one, from its final indices.
cudaError_t LaunchSswRgba(const SswLaunch& L, int n_images, cudaStream_t s);
// q_start[k] = q_end[k-1] for the active segments with k > 0.
cudaError_t LaunchSswCarry(const SswLaunch& L, cudaStream_t s);
std::size_t SswSmemBytes(int plan_smem_max, int cache_bits);

}  // namespace rdb
