// rdb_tsw.h -- the speculative segmented walk on thread walkers: one thread
// per segment, or (the paired form) per 32 segments a chain warp that walks
// each step's dependent chain and a sum warp that keeps their running sums.
//
// The exactness argument is the one of rdb_ssw.h (segments replayed from
// guessed states, checked against their predecessors, a verified prefix that
// grows by at least one segment a pass); what changes is the bookkeeping,
// which no longer keeps a per-segment table of every key touched:
//
//   G_prev  the previous pass's first-touch map, (segment << 8 | index) per
//           6-bit key, 0xFFFFFFFF = untouched.  A segment k answers a key from
//           G_prev whenever G_prev names an earlier segment, and then records
//           only "k took this key from G" (usemin[key] = min k).
//   own     keys G_prev gives no earlier segment for are searched by the
//           segment itself on first use and memoised in its own table (the
//           reference's first-touch rule, rd_types.h:111-153, inside the
//           segment); each such first use is also appended to the segment's
//           own list.
//   G_new   every touch does atomicMin(G_new[key], k << 8 | index).  G_new
//           starts as G_prev with only the entries of verified segments kept,
//           so after the walk it is the first-touch map of this pass.
//
// Checks after the walk, all of which must hold for a segment to be exact
// given exact predecessors:
//   queue   its start queue equals its predecessor's end queue bit for bit;
//   from G  for every key with usemin = u: G_new still names a segment before
//           u and with the index G_prev gave (the earliest taker fails first,
//           so u alone decides the verified prefix);
//   own     for every own first use (key, index) of segment k: no earlier
//           segment touched the key in G_new, or it gave the same index.
// The first failing segment per image bounds the next verified prefix.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace rdb {

struct TswImage {
  const unsigned char* pixels;
  int64_t row_stride;
  int width;
  int height;
  int layout;                // 3, 4 (8-bit) or 16 (float4 Q16)
  int n;                     // positions (= pixels)
  const int32_t* order;      // sequential visit order
  uint8_t* indices;
  float4* rgba_out;
  const unsigned char* plan; // device plan blob
  const uint8_t* uni;        // uniform-key table of the palette (rdb_uniform.h)
  int plan_smem;
  int first_seg;             // global id of segment 0
  int nsegs;
  int64_t cx_offset;         // first position in the gathered sample / index buffers
  uint32_t* g[2];            // first-touch maps; pass p writes g[p & 1]
  uint32_t* usemin;          // earliest segment that took the key from G_prev
  // Direct maps (no alpha): g and usemin have 2^18 entries indexed by key and
  // hkeys is null.  Hashed maps (alpha keys, 24 bits): hmask + 1 slots,
  // hkeys[slot] = key + 1 (0 = empty), every inserted slot listed in
  // hlist[0 .. *hcount).
  uint32_t* hkeys;
  uint32_t* hlist;
  int* hcount;               // [0] listed slots, [1] .. [2]: uniform-key classification progress
  uint32_t hmask;
  int pad2;
};

// A CTA's work: segments k0 .. k0 + count - 1 of one image (one plan per CTA).
struct TswChunk {
  int image;
  int k0;
  int count;
  int pad;
};

struct TswLaunch {
  const TswImage* images;
  int n_images;
  const TswChunk* chunks;
  int n_chunks;
  int pass;
  uint32_t tag;              // own-table tag of this pass (nonzero)
  int seg_len;
  int warm_len;
  double* q_start;           // per segment, pass 0: queue at its start after the warm-up
  double* q_end[2];          // per segment, by pass parity: 16 x 4 doubles, oldest first
  uint64_t* own;             // per segment: 2^own_bits entries (key | index << 24 | tag << 32)
  uint32_t* own_list;        // per segment: 2^own_bits words (key | index << 24)
  int* own_count;            // per segment
  int own_bits;
  const void* cx;            // gathered samples: uint32 RGBA8 or float4 per position
  uint8_t* chosen;           // per position
  int use_cache;
  int is_float;
  int assoc;                 // every palette of the launch associates alpha (or none does)
  int plan_smem_max;
  int chunk_threads;
  // Per image, by pass parity: the first failing segment of that pass (large
  // = none).  Pass p walks from min(bad[(p-1) & 1], nsegs) -- its verified
  // prefix -- and writes bad[p & 1].
  int* bad[2];
  // Per segment, written by every walk from pass 1 on: 1 when the segment's end
  // queue differs from the one it ended with in the previous pass, in the
  // channels a walk reads -- exactly when the next segment, which started
  // from that previous queue, started from the wrong one.
  uint8_t* changed;
  // Window (single-image launches; 0 = none): a pass walks only segments
  // [front, front + window) of the image, so a whole wave of resident threads
  // works at the front; the grids of the walk and of the segment checks cover
  // the window only (chunk / segment ids counted from the front's chunk).  A
  // segment whose predecessor the previous pass did not walk starts from the
  // empty queue, without warm-up positions, and its start queue is checked
  // like pass 0's (walked[pass & 1] marks the walked ones, warmed[] the ones
  // that started cache-free this pass).
  int window;
  // One image (with a window or without): the walk's grid of G CTAs takes
  // the segments from the front's chunk start on interleaved (CTA c, slot s
  // of its 128 walks segment base + s * G + c, the slots numbered lane by
  // lane across its warps) instead of 128 consecutive ones per CTA; with
  // per-image windows, the image's first G chunks take its window that way,
  // G covering the window plus one chunk.  So the
  // segments just past the front -- where new memo keys, and with them
  // searches, are densest -- spread over every CTA and warp rather than
  // holding up the launch in a few.  Same segments, same results.
  int spread;
  // Per-image windows (launches of several images; null = none): image i
  // walks segments [front, front + win[i]) each pass.  TswWindows sets them
  // after every pass from the segments each image has left: resident_segs
  // shared in proportion, at least win_min each, so the largest image, whose
  // passes are the launch's critical path, gets the widest window.
  int* win;
  int resident_segs;
  int win_min;
  uint8_t* walked[2];
  uint8_t* warmed;
  // Walk form: 0 = one thread per segment; 1 = paired warps, a chain warp
  // and a sum warp per 32 segments (same results bit for bit).
  int paired;
  int* status;
  // Profiling (null otherwise): positions walked, warm-ups included, summed
  // over the launches.
  unsigned long long* walk_count;
  // Device-side loop: the own-table tag of the running pass (null: use `tag`).
  const uint32_t* tag_dev;
  double sw[16];
};

std::size_t TswSmemBytes(int plan_smem_max);
// Segments the device walks at once in the given form (0 if the query fails).
int TswResidentThreads(int plan_smem_max, int sm_count, int assoc, int paired);
// Samples of every image in visit order, into L.cx.
cudaError_t LaunchTswGather(const TswLaunch& L, int64_t total_positions, cudaStream_t s);
// G_new = verified entries of G_prev, usemin cleared (memo only).
cudaError_t LaunchTswPrepare(const TswLaunch& L, cudaStream_t s);
cudaError_t LaunchTswWalk(const TswLaunch& L, cudaStream_t s);
// The three checks; the first failing segment per image into L.bad[pass & 1].
cudaError_t LaunchTswVerify(const TswLaunch& L, int total_segs, cudaStream_t s);
// Per-image windows for the next pass from the fronts in L.bad[L.pass & 1]
// (no-op without L.win).
cudaError_t LaunchTswWindows(const TswLaunch& L, cudaStream_t s);
// Indices (and RgbaF output) of every position into the images.
cudaError_t LaunchTswScatter(const TswLaunch& L, int64_t total_positions, cudaStream_t s);

// The pass loop as one CUDA graph: a while-conditional node whose body runs
// an even-parity pass, a control kernel, an odd-parity pass and the control
// kernel again.  `even` and `odd` are the launch parameters of the two
// passes (`pass` of matching parity and not 0; `tag_dev` set).  The control
// kernel (one block) reads every image's first failure of the pass just
// run: all images verified -> it stops the loop and records the pass count;
// an unfinished image whose verified prefix did not grow, or `max_passes`
// passes run -> it sets the status word and stops the loop; otherwise it
// advances the tag.  ctl[0] counts the loop's passes, ctl[1] is set once the
// loop is finished (later control launches then only stop it), ctl[2] is the
// loop's pass count at convergence.
cudaError_t BuildTswLoopGraph(const TswLaunch& even, const TswLaunch& odd, int total_segs,
                              int* ctl, uint32_t* tag_dev, int max_passes, cudaGraph_t* out);

}  // namespace rdb
