// rdb_runtime.h -- the host runtime behind the C ABI: one device context with
// resident palettes, per-geometry visit orders, memo slabs and scratch.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/rdb.h"
#include "rdb_plan.h"
#include "rdb_octree.h"
#include "rdb_walk.h"

namespace rdb {

// Thread-local error message (rdb_last_error).
void SetError(const std::string& msg);
const char* LastError();
std::size_t BytesPerPixel(int layout);
// Bytes of one packed frame of an RDB_* format, 0 when unknown or invalid.
std::size_t FrameBytes(int format, int width, int height);

// Palette text files (rdb_palette_file.cpp).  ReadPaletteText returns the
// sorted colours as a one-row RgbaF strip for the tree build.
int WritePaletteText(const double* colors, int count, const std::string& path);
// Palette PNG strips (rdb_palette_png.cpp).  ReadPalettePng returns the RgbaF
// swatch image the tree is built from, its size, and the colour count.
int WritePalettePng(const double* colors, int count, const std::string& path);
int ReadPalettePng(const std::string& path, int expect_colors, std::vector<float>* swatch,
                   std::size_t* width, std::size_t* height, int* count, bool* grayscale);
int ReadPaletteText(const std::string& path, int expect_colors, std::vector<float>* strip,
                    int* count, bool* associate_alpha, bool* grayscale);
int Fail(int code, const std::string& msg);
int CudaFail(cudaError_t e, const char* what);

// Upper bound of the device bytes one host image adds to a call of `engine`
// on a context: its staging, its visit order, its palette's tables and the
// scratch of the path the call takes for it (the segmented walk's samples,
// queues, memo tables and key maps; the plain walk's memo slab; the block
// copies).  The request loop admits by it.
std::size_t ScratchBound(int engine, int width, int height, int layout, bool assoc, bool rgba_out,
                         const rdb_options& o);
std::string CudaErr(cudaError_t e, const char* what);

// A device buffer that only grows.
struct DevBuf {
  void* ptr = nullptr;
  std::size_t bytes = 0;
};

struct DevPlan {
  unsigned char* dev = nullptr;
  std::size_t dev_bytes = 0;
  std::vector<uint8_t> host;
  int smem = 0;
  int count = 0;
  bool assoc = false;
  uint8_t* uniform = nullptr;  // uniform-key table (rdb_uniform.h), built on first use
  uint32_t* cand = nullptr;    // candidate table (rdb_cand.h), built on first use
};

// Segment-length autotuner of the segmented walk: per (device, log2 of the
// call's pixels, alpha) it times the occupancy rule's length, a half, a
// quarter and twice that on the first calls (device time of the passes) and
// keeps the fastest.  Results are exact whichever length runs, so exploring
// costs time only.  The table is shared by every context of the process
// (one lock), so the device workers of a server do not each explore afresh.
struct SegTune {
  std::vector<int> cand;
  std::vector<double> ms;  // -1 = not yet measured, -2 = being measured
  // The first call of a workload runs untimed: it pays one-time costs (module
  // loading on first launch, uniform tables) that would bias whichever
  // candidate came first.
  bool warmed = false;
};

class Context {
 public:
  ~Context();
  int Init(int device, std::size_t budget);

  int CreatePalette(const PlanInput& in, int* id);
  int DestroyPalette(int id);
  const DevPlan* Plan(int id) const;
  // The palette's uniform-key table, built on the stream on first use.
  int Uniform(int id, cudaStream_t s, const uint8_t** out);
  // The palette's candidate table (rdb_cand.h); palettes without associated
  // alpha only.
  int Candidates(int id, cudaStream_t s, const uint32_t** out);
  int DumpBlockIndices(const BlockLaunch& L, int64_t positions, cudaStream_t s);
  int StageHostJobs(const rdb_host_job* jobs, int n, std::vector<rdb_job>* out);
  int FinishHostJobs(const rdb_host_job* jobs, int n, const std::vector<rdb_job>& dj);
  // ColorTree::Build of an image in device memory (rdb_octree_build_device):
  // the first classification loop on the host over rows copied back, the
  // second on the device (rdb_octree_dev.cu), the reduction on the host.
  // *device_rows receives how many rows the device classified.  When the
  // caller still holds the image in host memory (host_pixels, host_stride),
  // the first loop reads its rows there instead.
  int BuildOctree(const void* pixels, int layout, int width, int height, std::size_t row_stride,
                  int max_colors, bool assoc, bool gray, cudaStream_t s, Octree* out,
                  int* device_rows, const void* host_pixels = nullptr, std::size_t host_stride = 0);

  // Visit order of a geometry, built on first use and kept resident.
  int Order(int width, int height, cudaStream_t s, const int32_t** out);

  int Dither(int engine, const rdb_job* jobs, int n, const rdb_options& o, cudaStream_t s);
  int DitherHost(int engine, const rdb_host_job* jobs, int n, const rdb_options& o);
  // Host jobs whose palettes are built here, each on the device from its own
  // uploaded pixels (BuildOctree): `colors` and `assoc` per job, their
  // palette_id ignored; build_ms (may be null) receives each build's time.
  int DitherHostBuilding(int engine, const rdb_host_job* jobs, const int* colors, const int* assoc,
                         int n, const rdb_options& o, double* build_ms);
  int CreatePaletteFromTree(const Octree& t, int* id);
  // Video frames through the blocks engine (rdb_dither_frames).
  int Frames(const rdb_frames& f, const rdb_options& o, cudaStream_t s);
  int FramesHost(const rdb_frames& f, const rdb_options& o);
  int Synchronize(cudaStream_t s);

  std::size_t bytes() const { return bytes_; }
  // The request loop's controls: the budget Reserve and the caches keep
  // within, and the release of every cached buffer -- scratch, memo slabs,
  // visit orders, idle palette blocks -- once the context's stream is done
  // (resident palettes stay).
  void SetBudget(std::size_t budget) { budget_ = budget; }
  std::size_t budget() const { return budget_; }
  void ReleaseScratch();
  cudaStream_t stream() const { return stream_; }
  int device() const { return device_; }
  int sm_count() const { return sm_count_; }

  // Grows `b` to at least `bytes`; frees and reallocates (contents lost).
  int Reserve(DevBuf* b, std::size_t bytes, const char* what);

 private:
  int Seq(const rdb_job* jobs, int n, const rdb_options& o, cudaStream_t s);
  int SeqSegmented(const rdb_job* jobs, int n, const rdb_options& o, cudaStream_t s);
  int SeqThreadSegmented(const rdb_job* jobs, int n, const rdb_options& o, cudaStream_t s);
  int SeqAuto(const rdb_job* jobs, int n, const rdb_options& o, cudaStream_t s);
  int Blocks(const rdb_job* jobs, int n, const rdb_options& o, cudaStream_t s);
  // `sweeps` > 1: block sweeps (rdb_options.jacobi_form 0), stopping early at
  // the first sweep that changes no block's end queue.
  int RunBlocks(int pid, int layout, std::vector<BlockImage>& imgs, const rdb_options& o,
                cudaStream_t s, int sweeps = 1);
  int JacobiSweeps(const rdb_job* jobs, int n, const rdb_options& o, cudaStream_t s);
  int CheckFrames(const rdb_frames& f) const;
  int Jacobi(const rdb_job* jobs, int n, const rdb_options& o, cudaStream_t s);
  int CheckJob(const rdb_job& j) const;
  void Release(DevBuf* b);
  // Small per-palette device blocks are recycled instead of freed: cudaFree
  // waits for the whole device, which would stall every other stream's work
  // each time a request's palette is dropped.
  void* AllocBlock(std::size_t bytes, const char* what, int* rc);
  void FreeBlock(void* p, std::size_t bytes);
  std::multimap<std::size_t, void*> free_blocks_;

  int device_ = 0;
  int sm_count_ = 148;
  std::size_t smem_optin_ = 227 * 1024;
  std::size_t budget_ = 0;
  std::size_t bytes_ = 0;
  cudaStream_t stream_ = nullptr;
  int next_palette_ = 1;
  std::map<int, DevPlan> plans_;
  // Visit orders by geometry; `use` is the call that last asked for one, so
  // an order the running call holds is never evicted under it.
  struct OrderEntry {
    int32_t* dev = nullptr;
    std::size_t bytes = 0;
    uint64_t use = 0;
  };
  std::map<std::pair<int, int>, OrderEntry> orders_;
  std::size_t order_bytes_ = 0;
  uint64_t call_ = 0;  // public calls so far (Dither, Frames)
  // Frees least recently used orders the running call does not hold, and idle
  // palette blocks, until `need` more bytes fit the budget; false if they
  // cannot.
  bool MakeRoom(std::size_t need);
  // Every scratch buffer a call may grow (not the work counter, the status
  // word or the pass-loop control words, which live as long as the context).
  std::vector<DevBuf*> CachedBufs();

  // Sequential engine state.
  // Plain-walk memo slabs, one set for RGB keys (2^18 per slab) and one for
  // alpha keys (2^24), each grown to the most CTAs a call of its kind used.
  DevBuf memo_[2];
  DevBuf memo_gen_[2];
  int memo_grid_[2] = {0, 0};
  DevBuf seq_items_;
  DevBuf counter_;
  DevBuf status_;
  // Blocks / Jacobi scratch.
  DevBuf curve_scratch_;
  DevBuf block_images_;
  DevBuf block_offsets_;
  DevBuf block_cx_;
  DevBuf block_chosen_;
  DevBuf jac_cx_;
  DevBuf jac_q_;
  DevBuf jac_g_;
  // Host-form staging.
  DevBuf host_in_;
  DevBuf host_idx_;
  DevBuf host_rgba_;
  // Segmented walk.
  DevBuf ssw_images_;
  DevBuf ssw_segs_;
  DevBuf ssw_work_;
  DevBuf ssw_q_;
  DevBuf ssw_ltab_;
  DevBuf ssw_g_;
  DevBuf ssw_bad_;
  // Thread-walker segmented walk.
  DevBuf tsw_images_;
  DevBuf tsw_chunks_;
  DevBuf tsw_bad_;
  DevBuf tsw_q_;
  DevBuf tsw_own_;
  DevBuf tsw_list_;
  DevBuf tsw_count_;
  DevBuf tsw_cx_;
  DevBuf tsw_chosen_;
  DevBuf tsw_g_;
  int last_passes_ = 0;
  bool profiling_ = false;
  std::string dump_prefix_;   // rdb_context_dump_indices: "" = off
  DevBuf dump_buf_;
  DevBuf octree_scratch_;
  DevBuf tsw_changed_;
  DevBuf sweep_q_;
  int last_sweeps_ = 0;
  bool last_sweeps_converged_ = false;
  DevBuf octree_init_;
  rdb_kernel_stats stats_{};
  cudaEvent_t ev_[2] = {nullptr, nullptr};
  // Pipelined pass loop of the segmented walk: a pinned ring of per-pass
  // results and the events that mark each pass done (and time its walk).
  cudaEvent_t tune_ev_[2] = {nullptr, nullptr};
  // Device-side pass loop: control words, the cached executable graph and the
  // launch parameters it was built for.
  DevBuf tsw_ctl_;
  cudaGraphExec_t loop_exec_ = nullptr;
  std::vector<unsigned char> loop_key_;
  bool loop_pending_ = false;       // last_passes_ still to be read from the device
  cudaStream_t loop_stream_ = nullptr;
  int PinnedRing(std::size_t ints);
  int PassEvents(int depth);
  int* ring_h_ = nullptr;
  std::size_t ring_cap_ = 0;
  std::vector<cudaEvent_t> pass_ev_;
  cudaEvent_t scratch_ev_ = nullptr;   // end of the last call's work (scratch reuse)
  cudaStream_t scratch_stream_ = nullptr;
  std::vector<cudaEvent_t> walk_ev_;

 public:
  // Passes of the last segmented walk; after a device-side loop this waits
  // for that call's stream and reads the loop's own count.
  int last_passes();
  int last_sweeps() const { return last_sweeps_; }
  bool last_sweeps_converged() const { return last_sweeps_converged_; }
  int Profile(bool on);
  // Block walks write `<prefix>.idx.bin` (every image's chosen index at every
  // block-list position, in list order, images in call order); "" = off.
  void DumpIndices(const std::string& prefix) { dump_prefix_ = prefix; }
  const rdb_kernel_stats& stats() const { return stats_; }
};

}  // namespace rdb

struct rdb_context {
  rdb::Context impl;
};
