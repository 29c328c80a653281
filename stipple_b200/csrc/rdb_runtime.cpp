// rdb_runtime.cpp -- host runtime of the engines (see rdb_runtime.h).
#include "rdb_runtime.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <map>
#include <tuple>
#include <mutex>
#include <cstring>
#include <numeric>

#include "rdb_curve.h"
#include "rdb_numeric.h"
#include "rdb_ssw.h"
#include "rdb_tsw.h"
#include "rdb_cand.h"
#include "rdb_octree_dev.h"
#include "rdb_uniform.h"

namespace rdb {
namespace {

thread_local std::string g_error;

constexpr std::size_t kMaxOrders = 1024;  // resident geometries before eviction
constexpr std::size_t kOrderCacheBytes = std::size_t{1} << 30;  // and their bytes
constexpr int kMaxAlphaSlabs = 64;  // plain walk: alpha memo slabs (32 MiB each) per launch
constexpr int kBatchWindowMin = 256;  // segmented walk of several images: the least window each

std::size_t RowStride(const rdb_job& j) {
  return j.row_stride ? j.row_stride : static_cast<std::size_t>(j.width) * BytesPerPixel(j.layout);
}

}  // namespace

std::mutex& SegTuneLock() {
  static std::mutex mu;
  return mu;
}

std::map<std::tuple<int, int, int>, SegTune>& SegTuneTable() {
  static std::map<std::tuple<int, int, int>, SegTune> table;
  return table;
}

// The block walk's launch-shape table (BlockWalkShape), keyed by device,
// alpha, float samples, log2 of the blocks and log2 of the padded block length;
// shared by the process's contexts like the segment-length table.
std::map<std::tuple<int, int, int, int, int>, SegTune>& ShapeTuneTable() {
  static std::map<std::tuple<int, int, int, int, int>, SegTune> table;
  return table;
}

std::size_t BytesPerPixel(int layout) { return layout == RDB_RGBAF32 ? 16 : static_cast<std::size_t>(layout); }

void SetError(const std::string& msg) { g_error = msg; }
const char* LastError() { return g_error.c_str(); }

int Fail(int code, const std::string& msg) {
  g_error = msg;
  return code;
}

std::string CudaErr(cudaError_t e, const char* what) {
  return std::string(what) + ": " + cudaGetErrorString(e);
}

int CudaFail(cudaError_t e, const char* what) {
  return Fail(e == cudaErrorMemoryAllocation ? RDB_E_NOMEM : RDB_E_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

Context::~Context() {
  cudaSetDevice(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  for (auto& p : plans_) {
    cudaFree(p.second.dev);
    cudaFree(p.second.uniform);
  }
  for (auto& b : free_blocks_) cudaFree(b.second);
  for (auto& o : orders_) cudaFree(o.second.dev);
  for (DevBuf* b : CachedBufs()) Release(b);
  Release(&counter_);
  Release(&status_);
  for (cudaEvent_t& ev : ev_) {
    if (ev) cudaEventDestroy(ev);
  }
  if (loop_exec_) cudaGraphExecDestroy(loop_exec_);
  Release(&tsw_ctl_);
  for (cudaEvent_t ev : pass_ev_) cudaEventDestroy(ev);
  for (cudaEvent_t ev : tune_ev_) {
    if (ev) cudaEventDestroy(ev);
  }
  if (scratch_ev_) cudaEventDestroy(scratch_ev_);
  for (cudaEvent_t ev : walk_ev_) cudaEventDestroy(ev);
  if (ring_h_) cudaFreeHost(ring_h_);
  if (stream_) cudaStreamDestroy(stream_);
}

int Context::last_passes() {
  if (loop_pending_) {
    int words[3] = {0, 0, 0};
    cudaSetDevice(device_);
    if (cudaStreamSynchronize(loop_stream_) == cudaSuccess &&
        cudaMemcpy(words, tsw_ctl_.ptr, sizeof(words), cudaMemcpyDeviceToHost) == cudaSuccess) {
      last_passes_ = 2 + words[2];  // two passes enqueued by the host, then the loop's
    }
    loop_pending_ = false;
  }
  return last_passes_;
}

int Context::PinnedRing(std::size_t ints) {
  if (ring_cap_ >= ints) return RDB_OK;
  if (ring_h_) {
    cudaStreamSynchronize(stream_);
    cudaFreeHost(ring_h_);
    ring_h_ = nullptr;
    ring_cap_ = 0;
  }
  const std::size_t want = std::max<std::size_t>(ints, 1024);
  const cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&ring_h_), want * sizeof(int),
                                      cudaHostAllocDefault);
  if (e != cudaSuccess) {
    ring_h_ = nullptr;
    return CudaFail(e, "pinned pass results");
  }
  ring_cap_ = want;
  return RDB_OK;
}

int Context::PassEvents(int depth) {
  while (static_cast<int>(pass_ev_.size()) < depth) {
    cudaEvent_t ev = nullptr;
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return CudaFail(e, "pass events");
    pass_ev_.push_back(ev);
  }
  while (static_cast<int>(walk_ev_.size()) < 2 * depth) {
    cudaEvent_t ev = nullptr;
    cudaError_t e = cudaEventCreate(&ev);
    if (e != cudaSuccess) return CudaFail(e, "walk events");
    walk_ev_.push_back(ev);
  }
  return RDB_OK;
}

int Context::Profile(bool on) {
  cudaSetDevice(device_);
  for (cudaEvent_t& ev : ev_) {
    if (!ev) {
      const cudaError_t e = cudaEventCreate(&ev);
      if (e != cudaSuccess) return CudaFail(e, "profiling events");
    }
  }
  profiling_ = on;
  stats_ = rdb_kernel_stats{};
  return RDB_OK;
}

int Context::Init(int device, std::size_t budget) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) return Fail(RDB_E_CUDA, "no CUDA device available");
  if (device < 0 || device >= count) return Fail(RDB_E_INVALID, "device index out of range");
  device_ = device;
  if ((e = cudaSetDevice(device)) != cudaSuccess) return CudaFail(e, "cudaSetDevice");
  cudaDeviceProp prop{};
  if ((e = cudaGetDeviceProperties(&prop, device)) != cudaSuccess) {
    return CudaFail(e, "cudaGetDeviceProperties");
  }
  if (prop.major < 10) {
    return Fail(RDB_E_CUDA, std::string("device ") + prop.name +
                                " is not sm_100 class; this library is built for sm_100a only");
  }
  sm_count_ = prop.multiProcessorCount;
  smem_optin_ = prop.sharedMemPerBlockOptin;
  std::size_t free_b = 0, total_b = 0;
  if ((e = cudaMemGetInfo(&free_b, &total_b)) != cudaSuccess) return CudaFail(e, "cudaMemGetInfo");
  budget_ = budget ? budget : (free_b / 10) * 9;
  if ((e = cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking)) != cudaSuccess) {
    return CudaFail(e, "cudaStreamCreate");
  }
  if (Reserve(&counter_, 256, "work counter") || Reserve(&status_, 256, "status word")) {
    return RDB_E_NOMEM;
  }
  cudaMemset(status_.ptr, 0, 256);
  return RDB_OK;
}

std::vector<DevBuf*> Context::CachedBufs() {
  return {&memo_[0],     &memo_gen_[0],   &memo_[1],     &memo_gen_[1],   &seq_items_,   &curve_scratch_, &block_images_,
          &block_offsets_, &block_cx_,    &block_chosen_, &jac_cx_,       &jac_q_,
          &jac_g_,       &host_in_,       &host_idx_,    &host_rgba_,     &ssw_images_,
          &ssw_segs_,    &ssw_work_,      &ssw_q_,       &ssw_ltab_,      &ssw_g_,
          &ssw_bad_,     &tsw_images_,    &tsw_chunks_,  &tsw_bad_,       &tsw_q_,
          &tsw_own_,     &tsw_list_,      &tsw_count_,   &tsw_cx_,        &tsw_chosen_,
          &tsw_g_,       &dump_buf_,      &octree_scratch_, &tsw_changed_, &sweep_q_,
          &octree_init_};
}

void Context::ReleaseScratch() {
  cudaSetDevice(device_);
  cudaStreamSynchronize(scratch_stream_ ? scratch_stream_ : stream_);
  for (DevBuf* b : CachedBufs()) Release(b);
  memo_grid_[0] = memo_grid_[1] = 0;
  for (auto& o : orders_) {
    cudaFree(o.second.dev);
    bytes_ -= o.second.bytes;
  }
  orders_.clear();
  order_bytes_ = 0;
  for (auto& b : free_blocks_) {
    cudaFree(b.second);
    bytes_ -= b.first;
  }
  free_blocks_.clear();
}

bool Context::MakeRoom(std::size_t need) {
  if (bytes_ + need <= budget_) return true;
  // The device may still read what is freed here: wait for this context's
  // work first.
  cudaStreamSynchronize(scratch_stream_ ? scratch_stream_ : stream_);
  for (auto& b : free_blocks_) {
    cudaFree(b.second);
    bytes_ -= b.first;
  }
  free_blocks_.clear();
  while (bytes_ + need > budget_) {
    auto victim = orders_.end();
    for (auto it = orders_.begin(); it != orders_.end(); ++it) {
      if (it->second.use != call_ && (victim == orders_.end() || it->second.use < victim->second.use)) {
        victim = it;
      }
    }
    if (victim == orders_.end()) return false;
    cudaFree(victim->second.dev);
    bytes_ -= victim->second.bytes;
    order_bytes_ -= victim->second.bytes;
    orders_.erase(victim);
  }
  return true;
}

void Context::Release(DevBuf* b) {
  if (b->ptr) {
    cudaFree(b->ptr);
    bytes_ -= b->bytes;
  }
  b->ptr = nullptr;
  b->bytes = 0;
}

int Context::Reserve(DevBuf* b, std::size_t bytes, const char* what) {
  if (b->bytes >= bytes) return RDB_OK;
  // Grow geometrically so a stream of slightly larger jobs does not thrash.
  std::size_t want = std::max(bytes, b->bytes + b->bytes / 2);
  if (bytes_ - b->bytes + want > budget_) want = bytes;
  if (bytes_ - b->bytes + want > budget_ && !MakeRoom(want - b->bytes)) {
    return Fail(RDB_E_NOMEM, std::string(what) + ": device memory budget exceeded");
  }
  if (b->ptr) {
    // Every stream that may still read the old buffer must be done with it.
    cudaDeviceSynchronize();
  }
  Release(b);
  void* p = nullptr;
  const cudaError_t e = cudaMalloc(&p, want);
  if (e != cudaSuccess) return CudaFail(e, what);
  b->ptr = p;
  b->bytes = want;
  bytes_ += want;
  return RDB_OK;
}

void* Context::AllocBlock(std::size_t bytes, const char* what, int* rc) {
  auto it = free_blocks_.find(bytes);
  if (it != free_blocks_.end()) {
    void* p = it->second;
    free_blocks_.erase(it);
    *rc = RDB_OK;
    return p;
  }
  if (bytes_ + bytes > budget_ && !MakeRoom(bytes)) {
    *rc = Fail(RDB_E_NOMEM, std::string(what) + ": budget exceeded");
    return nullptr;
  }
  void* p = nullptr;
  const cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    *rc = CudaFail(e, what);
    return nullptr;
  }
  bytes_ += bytes;
  *rc = RDB_OK;
  return p;
}

void Context::FreeBlock(void* p, std::size_t bytes) {
  if (p) free_blocks_.emplace(bytes, p);
}

int Context::CreatePalette(const PlanInput& in, int* id) {
  DevPlan p;
  const std::string err = BuildPlan(in, &p.host);
  if (!err.empty()) return Fail(RDB_E_UNSUPPORTED, err);
  const PlanHeader* h = reinterpret_cast<const PlanHeader*>(p.host.data());
  p.smem = h->smem_bytes;
  p.count = h->count;
  p.assoc = h->assoc != 0;
  // Size classes of 16 KB keep recycled blocks interchangeable.
  p.dev_bytes = (p.host.size() + 16383) & ~static_cast<std::size_t>(16383);
  int rc = RDB_OK;
  p.dev = static_cast<unsigned char*>(AllocBlock(p.dev_bytes, "palette", &rc));
  if (!p.dev) return rc;
  // Ordered on the context stream, complete before any other stream can use it.
  cudaError_t e = cudaMemcpyAsync(p.dev, p.host.data(), p.host.size(), cudaMemcpyHostToDevice, stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) {
    FreeBlock(p.dev, p.dev_bytes);
    return CudaFail(e, "palette upload");
  }
  const int pid = next_palette_++;
  plans_[pid] = std::move(p);
  *id = pid;
  return RDB_OK;
}

// The caller has finished (synchronised) every stream other than the
// context's own on which it used the palette; the context's own stream is
// drained here.  Its blocks go back to the context's pool.
int Context::DestroyPalette(int id) {
  auto it = plans_.find(id);
  if (it == plans_.end()) return Fail(RDB_E_INVALID, "unknown palette id");
  cudaStreamSynchronize(stream_);
  FreeBlock(it->second.dev, it->second.dev_bytes);
  FreeBlock(it->second.uniform, it->second.assoc ? kUniformKeysAlpha : kUniformKeys);
  FreeBlock(it->second.cand, kCandKeys * sizeof(uint32_t));
  plans_.erase(it);
  return RDB_OK;
}

int Context::Uniform(int id, cudaStream_t s, const uint8_t** out) {
  auto it = plans_.find(id);
  if (it == plans_.end()) return Fail(RDB_E_INVALID, "unknown palette id");
  DevPlan& p = it->second;
  if (p.assoc) {
    // 2^24 keys, classified lazily: every entry starts "not yet classified"
    // and the segmented walk classifies the keys it meets after each pass.
    if (!p.uniform) {
      int rc = RDB_OK;
      p.uniform = static_cast<uint8_t*>(AllocBlock(kUniformKeysAlpha, "uniform-key table", &rc));
      if (!p.uniform) return rc;
      cudaError_t e;
      if ((e = cudaMemsetAsync(p.uniform, kUniformUnknown, kUniformKeysAlpha, s)) != cudaSuccess ||
          (e = cudaStreamSynchronize(s)) != cudaSuccess) {
        return CudaFail(e, "uniform-key table");
      }
    }
    *out = p.uniform;
    return RDB_OK;
  }
  if (!p.uniform) {
    int rc = RDB_OK;
    p.uniform = static_cast<uint8_t*>(AllocBlock(kUniformKeys, "uniform-key table", &rc));
    if (!p.uniform) return rc;
    // Built once; other streams may read it later, so it is complete on return.
    cudaError_t e;
    if ((e = LaunchUniformTable(p.dev, p.uniform, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
      return CudaFail(e, "uniform-key table");
    }
  }
  *out = p.uniform;
  return RDB_OK;
}

int Context::Candidates(int id, cudaStream_t s, const uint32_t** out) {
  auto it = plans_.find(id);
  if (it == plans_.end()) return Fail(RDB_E_INVALID, "unknown palette id");
  DevPlan& p = it->second;
  if (p.assoc) return Fail(RDB_E_INVALID, "candidate tables cover palettes without associated alpha");
  if (!p.cand) {
    int rc = RDB_OK;
    p.cand = static_cast<uint32_t*>(AllocBlock(kCandKeys * sizeof(uint32_t), "candidate table", &rc));
    if (!p.cand) return rc;
    // Built once; other streams may read it later, so it is complete on return.
    cudaError_t e;
    if ((e = LaunchCandidateTable(p.dev, p.cand, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
      return CudaFail(e, "candidate table");
    }
  }
  *out = p.cand;
  return RDB_OK;
}

const DevPlan* Context::Plan(int id) const {
  auto it = plans_.find(id);
  return it == plans_.end() ? nullptr : &it->second;
}

int Context::Order(int width, int height, cudaStream_t s, const int32_t** out) {
  const auto key = std::make_pair(width, height);
  auto it = orders_.find(key);
  if (it != orders_.end()) {
    it->second.use = call_;
    *out = it->second.dev;
    return RDB_OK;
  }
  const std::size_t n = static_cast<std::size_t>(width) * height;
  const std::size_t bytes = std::max<std::size_t>(n, 1) * sizeof(int32_t);
  // The cache keeps at most kMaxOrders geometries and kOrderCacheBytes:
  // beyond either, least recently used orders the running call does not
  // hold are evicted (after the device is done with them).
  bool synced = false;
  while (orders_.size() >= kMaxOrders || order_bytes_ + bytes > kOrderCacheBytes) {
    auto victim = orders_.end();
    for (auto v = orders_.begin(); v != orders_.end(); ++v) {
      if (v->second.use != call_ && (victim == orders_.end() || v->second.use < victim->second.use)) victim = v;
    }
    if (victim == orders_.end()) break;  // all held by this call: grow past the cap
    if (!synced) {
      cudaStreamSynchronize(scratch_stream_ ? scratch_stream_ : stream_);
      synced = true;
    }
    cudaFree(victim->second.dev);
    bytes_ -= victim->second.bytes;
    order_bytes_ -= victim->second.bytes;
    orders_.erase(victim);
  }
  if (!MakeRoom(bytes)) return Fail(RDB_E_NOMEM, "visit order: budget exceeded");
  int32_t* d = nullptr;
  cudaError_t e = cudaMalloc(&d, bytes);
  if (e != cudaSuccess) return CudaFail(e, "visit order allocation");
  bytes_ += bytes;
  const int level = CurveLevel(width, height);
  const std::size_t scratch = CurveScratchBytes(level);
  if (int rc = Reserve(&curve_scratch_, scratch, "curve scratch")) {
    cudaFree(d);
    bytes_ -= bytes;
    return rc;
  }
  e = BuildSeqOrder(width, height, d, curve_scratch_.ptr, curve_scratch_.bytes, s);
  if (e != cudaSuccess) {
    cudaFree(d);
    bytes_ -= bytes;
    return CudaFail(e, "visit order kernel");
  }
  orders_[key] = OrderEntry{d, bytes, call_};
  order_bytes_ += bytes;
  *out = d;
  return RDB_OK;
}

int Context::CheckJob(const rdb_job& j) const {
  if (j.width < 1 || j.height < 1) return Fail(RDB_E_INVALID, "image must be at least 1x1");
  if (static_cast<int64_t>(j.width) * j.height >= (static_cast<int64_t>(1) << 31) - 1) {
    return Fail(RDB_E_UNSUPPORTED, "image larger than 2^31 - 2 pixels");
  }
  if (j.layout != RDB_RGB8 && j.layout != RDB_RGBA8 && j.layout != RDB_RGBAF32) {
    return Fail(RDB_E_INVALID, "unknown pixel layout");
  }
  if (!j.pixels || !j.indices) return Fail(RDB_E_INVALID, "null pixel or index buffer");
  if (j.layout == RDB_RGBAF32 && (reinterpret_cast<uintptr_t>(j.pixels) & 15u)) {
    return Fail(RDB_E_INVALID, "RgbaF pixels must be 16-byte aligned");
  }
  if (j.layout == RDB_RGBA8 && (reinterpret_cast<uintptr_t>(j.pixels) & 3u)) {
    return Fail(RDB_E_INVALID, "RGBA8 pixels must be 4-byte aligned");
  }
  const std::size_t stride = RowStride(j);
  if (stride < static_cast<std::size_t>(j.width) * BytesPerPixel(j.layout)) {
    return Fail(RDB_E_INVALID, "row stride shorter than a row");
  }
  if ((j.layout == RDB_RGBAF32 && stride % 16) || (j.layout == RDB_RGBA8 && stride % 4)) {
    return Fail(RDB_E_INVALID, "row stride breaks pixel alignment");
  }
  if (j.rgba_out && (reinterpret_cast<uintptr_t>(j.rgba_out) & 15u)) {
    return Fail(RDB_E_INVALID, "RgbaF output must be 16-byte aligned");
  }
  if (!Plan(j.palette_id)) return Fail(RDB_E_INVALID, "unknown palette id");
  return RDB_OK;
}

int Context::Dither(int engine, const rdb_job* jobs, int n, const rdb_options& o,
                    cudaStream_t s) {
  if (n < 0 || (n > 0 && !jobs)) return Fail(RDB_E_INVALID, "bad job list");
  if (n == 0) return RDB_OK;
  for (int i = 0; i < n; ++i) {
    if (int rc = CheckJob(jobs[i])) return rc;
  }
  ++call_;
  if (!s) s = stream_;
  cudaSetDevice(device_);
  // The context's scratch buffers are shared by every call: a call on a new
  // stream waits (on the device) for the work the previous call enqueued.
  if (!scratch_ev_) {
    const cudaError_t e = cudaEventCreateWithFlags(&scratch_ev_, cudaEventDisableTiming);
    if (e != cudaSuccess) return CudaFail(e, "scratch event");
  } else if (scratch_stream_ != s) {
    cudaStreamWaitEvent(s, scratch_ev_, 0);
  }
  int rc;
  switch (engine) {
    case RDB_ENGINE_SEQ:
      if (o.seq_mode == 1) {
        rc = Seq(jobs, n, o, s);
      } else if (o.seq_mode == 2) {
        rc = SeqSegmented(jobs, n, o, s);
      } else if (o.seq_mode == 3) {
        rc = SeqThreadSegmented(jobs, n, o, s);
      } else if (o.seq_mode != 0) {
        rc = Fail(RDB_E_INVALID, "seq_mode must be 0..3");
      } else {
        rc = SeqAuto(jobs, n, o, s);
      }
      break;
    case RDB_ENGINE_BLOCKS: rc = Blocks(jobs, n, o, s); break;
    case RDB_ENGINE_JACOBI: rc = Jacobi(jobs, n, o, s); break;
    default: rc = Fail(RDB_E_INVALID, "unknown engine");
  }
  cudaEventRecord(scratch_ev_, s);
  scratch_stream_ = s;
  return rc;
}

int Context::Seq(const rdb_job* jobs, int n, const rdb_options& o, cudaStream_t s) {
  std::vector<SeqItem> items(static_cast<std::size_t>(n));
  int plan_max = 0;
  bool any_assoc = false;
  for (int i = 0; i < n; ++i) {
    const rdb_job& j = jobs[i];
    const DevPlan* p = Plan(j.palette_id);
    const int32_t* order = nullptr;
    if (int rc = Order(j.width, j.height, s, &order)) return rc;
    SeqItem& it = items[static_cast<std::size_t>(i)];
    it.pixels = static_cast<const unsigned char*>(j.pixels);
    it.row_stride = static_cast<int64_t>(RowStride(j));
    it.width = j.width;
    it.height = j.height;
    it.layout = j.layout;
    it.n = j.width * j.height;
    it.order = order;
    it.indices = j.indices;
    it.rgba_out = reinterpret_cast<float4*>(j.rgba_out);
    it.plan = p->dev;
    it.plan_smem = p->smem;
    it.pad = 0;
    plan_max = std::max(plan_max, p->smem);
    any_assoc = any_assoc || p->assoc;
  }
  // Longest walk first: the makespan is bounded below by it.
  std::stable_sort(items.begin(), items.end(),
                   [](const SeqItem& a, const SeqItem& b) { return a.n > b.n; });

  const bool use_cache = o.use_cache != 0;
  // One warp per CTA.  Several CTAs share an SM once the batch is larger than
  // the SM count; shared memory is split between them.
  int per_sm = std::min(8, std::max(1, (n + sm_count_ - 1) / sm_count_));
  int grid = std::min(n, sm_count_ * per_sm);
  // Memo slabs: one per CTA, 2^18 keys (2^24 with alpha), generation-tagged.
  const int set = any_assoc ? 1 : 0;
  const int64_t entries = any_assoc ? (int64_t{1} << 24) : (int64_t{1} << 18);
  if (use_cache) {
    // CTAs take images from the work counter, so fewer CTAs only walk more
    // images each: an alpha slab is 32 MiB, so at most kMaxAlphaSlabs of
    // them, and no more than half the budget left once the old slabs go.
    const std::size_t slab = static_cast<std::size_t>(entries) * sizeof(uint16_t) + sizeof(uint32_t);
    const std::size_t held = memo_[set].bytes + memo_gen_[set].bytes;
    const std::size_t left = budget_ > bytes_ - held ? budget_ - (bytes_ - held) : 0;
    int cap = static_cast<int>(std::min<std::size_t>(left / 2 / slab, 1 << 20));
    if (any_assoc) cap = std::min(cap, kMaxAlphaSlabs);
    grid = std::max(1, std::min(grid, std::max(cap, memo_grid_[set])));
    per_sm = std::min(per_sm, std::max(1, (grid + sm_count_ - 1) / sm_count_));
  }
  const std::size_t ring = 96 * (sizeof(int32_t) + 16);
  const std::size_t smem_cap = std::min<std::size_t>(smem_optin_, (228 * 1024) / per_sm - 1024);
  int cache_bits = o.cache_bits;
  if (use_cache && cache_bits == 0) {
    cache_bits = 15;
    while (cache_bits > 8 &&
           plan_max + ring + (static_cast<std::size_t>(4) << cache_bits) > smem_cap) {
      --cache_bits;
    }
  }
  if (use_cache && (cache_bits < 4 || cache_bits > 20)) {
    return Fail(RDB_E_INVALID, "cache_bits must be 4..20 (0 = automatic)");
  }
  const std::size_t smem = SeqSmemBytes(plan_max, cache_bits, use_cache);
  if (smem > smem_optin_) return Fail(RDB_E_UNSUPPORTED, "palette plan does not fit in shared memory");

  if (use_cache && grid > memo_grid_[set]) {
    cudaDeviceSynchronize();  // earlier walks may still read the old slabs
    Release(&memo_[set]);
    Release(&memo_gen_[set]);
    memo_grid_[set] = 0;
    const std::size_t g = static_cast<std::size_t>(grid);
    if (int rc = Reserve(&memo_[set], g * static_cast<std::size_t>(entries) * sizeof(uint16_t), "memo slabs")) {
      return rc;
    }
    if (int rc = Reserve(&memo_gen_[set], g * sizeof(uint32_t), "memo generations")) return rc;
    cudaMemsetAsync(memo_[set].ptr, 0, memo_[set].bytes, s);
    cudaMemsetAsync(memo_gen_[set].ptr, 0, memo_gen_[set].bytes, s);
    memo_grid_[set] = grid;
  }
  if (int rc = Reserve(&seq_items_, items.size() * sizeof(SeqItem), "work items")) return rc;
  cudaError_t e = cudaMemcpyAsync(seq_items_.ptr, items.data(), items.size() * sizeof(SeqItem),
                                  cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return CudaFail(e, "work item upload");
  // The host vector must outlive the async copy.
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return CudaFail(e, "work item upload");
  cudaMemsetAsync(counter_.ptr, 0, sizeof(int), s);

  SeqLaunch L{};
  L.items = static_cast<const SeqItem*>(seq_items_.ptr);
  L.n_items = n;
  L.work_counter = static_cast<int*>(counter_.ptr);
  L.memo = static_cast<uint16_t*>(memo_[set].ptr);
  L.memo_gen = static_cast<uint32_t*>(memo_gen_[set].ptr);
  L.slab_entries = entries;
  L.cache_bits = use_cache ? cache_bits : 0;
  L.plan_smem_max = plan_max;
  L.use_cache = use_cache ? 1 : 0;
  scaled_weights(o.diffusion, L.sw);
  L.status = static_cast<int*>(status_.ptr);
  e = LaunchSeqWalk(L, grid, s);
  if (e != cudaSuccess) return CudaFail(e, "sequential walk launch");
  return RDB_OK;
}

int Context::Blocks(const rdb_job* jobs, int n, const rdb_options& o, cudaStream_t s) {
  const int pid = jobs[0].palette_id;
  const int layout = jobs[0].layout;
  for (int i = 1; i < n; ++i) {
    if (jobs[i].palette_id != pid || jobs[i].layout != layout) {
      return Fail(RDB_E_INVALID, "blocks engine: one palette and one layout per call");
    }
  }
  std::vector<BlockImage> imgs(static_cast<std::size_t>(n));
  for (int i = 0; i < n; ++i) {
    const rdb_job& j = jobs[i];
    BlockImage& b = imgs[static_cast<std::size_t>(i)];
    b.pixels = static_cast<const unsigned char*>(j.pixels);
    b.row_stride = static_cast<int64_t>(RowStride(j));
    b.width = j.width;
    b.height = j.height;
    b.layout = j.layout;
    b.indices = j.indices;
    // An RgbaF input dithered in place already holds its source values.
    b.rgba_out = reinterpret_cast<float4*>(j.rgba_out);
    if (j.rgba_out == j.pixels && BlockListLength(j.width, j.height) == 0) b.rgba_out = nullptr;
  }
  return RunBlocks(pid, layout, imgs, o, s);
}

// Shared by rdb_dither's blocks engine and the video-frame form: `imgs` hold
// everything but the walk bookkeeping, which is filled in here.
int Context::RunBlocks(int pid, int layout, std::vector<BlockImage>& all, const rdb_options& o,
                       cudaStream_t s, int sweeps) {
  if (o.block < kQueue) {
    return Fail(RDB_E_UNSUPPORTED, "--blocks must be at least 16 (the error queue is 16 entries deep)");
  }
  const DevPlan* p = Plan(pid);
  std::vector<BlockImage> imgs;
  std::vector<int64_t> offs;
  int64_t blocks = 0, positions = 0;
  int64_t longest = 0;
  for (BlockImage b : all) {
    const int64_t nb = BlockListLength(b.width, b.height);
    if (nb == 0) {
      // 1x1: BuildCurveIndex is empty and the pixel keeps its value.
      const cudaError_t e = LaunchSourceFill(b, s);
      if (e != cudaSuccess) return CudaFail(e, "source copy");
      continue;
    }
    if (int rc = Order(b.width, b.height, s, &b.order)) return rc;
    b.n = static_cast<int>(nb);
    b.first_block = blocks;
    b.nblocks = static_cast<int>((nb + o.block - 1) / o.block);
    blocks += b.nblocks;
    offs.push_back(positions);
    positions += nb;
    longest = std::max(longest, nb);
    imgs.push_back(b);
  }
  if (imgs.empty()) return RDB_OK;
  const bool packed = layout == RDB_RGB8 || layout == RDB_RGBA8;
  const std::size_t word = packed ? 4 : 16;
  // The walk's scratch (rdb_walk.h): groups of 32 blocks, bpad positions each.
  const int bpad = static_cast<int>((std::min<int64_t>(o.block, longest) + 15) & ~int64_t{15});
  const std::size_t cells = static_cast<std::size_t>((blocks + 31) / 32 * 32) * static_cast<std::size_t>(bpad);
  if (int rc = Reserve(&block_images_, imgs.size() * sizeof(BlockImage), "block images")) return rc;
  if (int rc = Reserve(&block_offsets_, offs.size() * sizeof(int64_t), "block offsets")) return rc;
  if (int rc = Reserve(&block_cx_, cells * word, "block samples")) return rc;
  if (int rc = Reserve(&block_chosen_, cells, "block indices")) return rc;
  const uint32_t* cand = nullptr;
  if (!p->assoc) {
    if (int rc = Candidates(pid, s, &cand)) return rc;
  }
  cudaMemcpyAsync(block_images_.ptr, imgs.data(), imgs.size() * sizeof(BlockImage),
                  cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(block_offsets_.ptr, offs.data(), offs.size() * sizeof(int64_t),
                  cudaMemcpyHostToDevice, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return CudaFail(e, "block descriptor upload");
  BlockLaunch L{};
  L.images = static_cast<const BlockImage*>(block_images_.ptr);
  L.n_images = static_cast<int>(imgs.size());
  L.block = o.block;
  L.total_blocks = blocks;
  L.cx = static_cast<uint32_t*>(block_cx_.ptr);
  L.chosen = static_cast<uint8_t*>(block_chosen_.ptr);
  L.pos_offset = static_cast<const int64_t*>(block_offsets_.ptr);
  L.cand = cand;
  L.bpad = bpad;
  L.plan = p->dev;
  L.plan_smem = p->smem;
  L.assoc = p->assoc ? 1 : 0;
  L.is_float = packed ? 0 : 1;
  scaled_weights(o.diffusion, L.sw);
  L.status = static_cast<int*>(status_.ptr);
  // Launch shape: the fastest measured for this workload class; its first
  // calls run each shape once, timed on the device (the very first untimed:
  // it pays module loading and table builds).
  int shape = 0, tune_slot = -1;
  SegTune* tune = nullptr;
  {
    int lb = 0, lp = 0;
    while ((int64_t{1} << (lb + 1)) <= blocks) ++lb;
    while ((1 << (lp + 1)) <= bpad) ++lp;
    std::lock_guard<std::mutex> lk(SegTuneLock());
    tune = &ShapeTuneTable()[std::make_tuple(device_, L.assoc, L.is_float, lb, lp)];
    if (tune->cand.empty()) {
      for (int c = 0; c < kBlockWalkShapes; ++c) tune->cand.push_back(c);
      tune->ms.assign(tune->cand.size(), -1.0);
    }
    if (!tune->warmed) {
      if (sweeps <= 1) tune->warmed = true;
    } else {
      for (std::size_t c = 0; c < tune->cand.size() && tune_slot < 0; ++c) {
        if (tune->ms[c] == -1.0) tune_slot = static_cast<int>(c);
      }
      if (sweeps > 1) tune_slot = -1;  // sweeps use what single walks measured
      if (tune_slot >= 0) {
        tune->ms[static_cast<std::size_t>(tune_slot)] = -2.0;
        shape = tune->cand[static_cast<std::size_t>(tune_slot)];
      } else {
        int best = 0;
        for (std::size_t c = 0; c < tune->cand.size(); ++c) {
          if (tune->ms[c] >= 0 && (tune->ms[static_cast<std::size_t>(best)] < 0 ||
                                   tune->ms[c] < tune->ms[static_cast<std::size_t>(best)])) {
            best = static_cast<int>(c);
          }
        }
        shape = tune->ms[static_cast<std::size_t>(best)] >= 0 ? tune->cand[static_cast<std::size_t>(best)] : 0;
      }
    }
  }
  BlockWalkShape(shape, L.assoc != 0, &stats_.block_threads, &stats_.block_min_ctas);
  if (sweeps <= 1) {
    if ((e = LaunchBlockGather(L, s)) != cudaSuccess) return CudaFail(e, "blocks engine launch");
    if (tune_slot >= 0) {
      for (cudaEvent_t& ev : tune_ev_) {
        if (!ev && (e = cudaEventCreate(&ev)) != cudaSuccess) return CudaFail(e, "tuner events");
      }
      cudaEventRecord(tune_ev_[0], s);
    }
    if ((e = LaunchBlockWalkOnly(L, s, shape)) != cudaSuccess) return CudaFail(e, "blocks engine launch");
    if (tune_slot >= 0) {
      float ms = 0.0f;
      cudaEventRecord(tune_ev_[1], s);
      cudaEventSynchronize(tune_ev_[1]);
      std::lock_guard<std::mutex> lk(SegTuneLock());
      tune->ms[static_cast<std::size_t>(tune_slot)] =
          cudaEventElapsedTime(&ms, tune_ev_[0], tune_ev_[1]) == cudaSuccess ? ms : -1.0;
    }
    if ((e = LaunchBlockScatter(L, positions, s)) != cudaSuccess) return CudaFail(e, "blocks engine launch");
    if (!dump_prefix_.empty()) return DumpBlockIndices(L, positions, s);
    return RDB_OK;
  }
  // Block sweeps: end queues ping-pong between two buffers; the counter of
  // changed blocks sits after them.
  const std::size_t qbytes = static_cast<std::size_t>(blocks) * 64 * sizeof(double);
  if (int rc = Reserve(&sweep_q_, 2 * qbytes + 256, "block sweep queues")) return rc;
  double* qbuf[2] = {static_cast<double*>(sweep_q_.ptr),
                     reinterpret_cast<double*>(static_cast<unsigned char*>(sweep_q_.ptr) + qbytes)};
  int* changed = reinterpret_cast<int*>(static_cast<unsigned char*>(sweep_q_.ptr) + 2 * qbytes);
  if ((e = LaunchBlockGather(L, s)) != cudaSuccess) return CudaFail(e, "block sweep gather");
  last_sweeps_ = 0;
  last_sweeps_converged_ = false;
  for (int k = 0; k < sweeps; ++k) {
    L.q_in = k == 0 ? nullptr : qbuf[(k - 1) & 1];
    L.q_out = qbuf[k & 1];
    L.changed = changed;
    if ((e = cudaMemsetAsync(changed, 0, sizeof(int), s)) != cudaSuccess ||
        (e = LaunchBlockWalkOnly(L, s, shape)) != cudaSuccess) {
      return CudaFail(e, "block sweep");
    }
    last_sweeps_ = k + 1;
    if (k == 0) continue;
    int n_changed = 0;
    if ((e = cudaMemcpyAsync(&n_changed, changed, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
      return CudaFail(e, "block sweep check");
    }
    if (n_changed == 0) {
      last_sweeps_converged_ = true;
      break;
    }
  }
  if (sweeps == 1 || blocks == static_cast<int64_t>(imgs.size())) last_sweeps_converged_ = true;
  if ((e = LaunchBlockScatter(L, positions, s)) != cudaSuccess) return CudaFail(e, "block sweep scatter");
  if (!dump_prefix_.empty()) return DumpBlockIndices(L, positions, s);
  return RDB_OK;
}

// The approximation's default form (rdb_options.jacobi_form 0): block sweeps
// over each image's block-mode list, blocks of 256, images of one palette and
// layout walked together.
int Context::JacobiSweeps(const rdb_job* jobs, int n, const rdb_options& o, cudaStream_t s) {
  if (o.jacobi_iters < 0) return Fail(RDB_E_INVALID, "negative Jacobi iteration count");
  rdb_options bo = o;
  bo.block = 256;
  const int sweeps = std::max(1, o.jacobi_iters);
  int most = 0;
  bool all_converged = true;
  int i = 0;
  while (i < n) {
    int k = i + 1;
    while (k < n && jobs[k].palette_id == jobs[i].palette_id && jobs[k].layout == jobs[i].layout) ++k;
    std::vector<BlockImage> imgs(static_cast<std::size_t>(k - i));
    for (int m = i; m < k; ++m) {
      const rdb_job& j = jobs[m];
      BlockImage& b = imgs[static_cast<std::size_t>(m - i)];
      b.pixels = static_cast<const unsigned char*>(j.pixels);
      b.row_stride = static_cast<int64_t>(RowStride(j));
      b.width = j.width;
      b.height = j.height;
      b.layout = j.layout;
      b.indices = j.indices;
      b.rgba_out = reinterpret_cast<float4*>(j.rgba_out);
      if (j.rgba_out == j.pixels && BlockListLength(j.width, j.height) == 0) b.rgba_out = nullptr;
    }
    last_sweeps_ = 0;
    last_sweeps_converged_ = true;  // an image with an empty list needs no sweep
    if (int rc = RunBlocks(jobs[i].palette_id, jobs[i].layout, imgs, bo, s, sweeps)) return rc;
    most = std::max(most, last_sweeps_);
    all_converged = all_converged && last_sweeps_converged_;
    i = k;
  }
  last_sweeps_ = most;
  last_sweeps_converged_ = all_converged;
  return RDB_OK;
}

int Context::BuildOctree(const void* pixels, int layout, int width, int height, std::size_t stride,
                         int max_colors, bool assoc, bool gray, cudaStream_t s, Octree* out,
                         int* device_rows, const void* host_pixels, std::size_t host_stride) {
  if (!s) s = stream_;
  cudaSetDevice(device_);
  *device_rows = 0;
  const std::size_t W = static_cast<std::size_t>(width);
  const std::size_t bpp = layout == RDB_RGBAF32 ? 16 : static_cast<std::size_t>(layout);
  // Rows for the host loops, copied back one at a time and widened to Q16.
  std::vector<unsigned char> raw(W * bpp);
  std::vector<float> widened(W * 4);
  cudaError_t fetch_error = cudaSuccess;
  const auto row_at = [&](std::size_t y) -> const float* {
    if (host_pixels) {
      // The same rows in host memory: no copy back.
      std::memcpy(raw.data(), static_cast<const unsigned char*>(host_pixels) + y * host_stride, raw.size());
    } else {
      const unsigned char* src = static_cast<const unsigned char*>(pixels) + y * stride;
      const cudaError_t e = cudaMemcpyAsync(raw.data(), src, raw.size(), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) {
        const cudaError_t e2 = cudaStreamSynchronize(s);
        if (e2 != cudaSuccess) fetch_error = e2;
      } else {
        fetch_error = e;
      }
    }
    if (layout == RDB_RGBAF32) {
      std::memcpy(widened.data(), raw.data(), raw.size());
    } else {
      for (std::size_t x = 0; x < W; ++x) {
        widened[4 * x + 0] = static_cast<float>(raw[bpp * x + 0]) * 257.0f;
        widened[4 * x + 1] = static_cast<float>(raw[bpp * x + 1]) * 257.0f;
        widened[4 * x + 2] = static_cast<float>(raw[bpp * x + 2]) * 257.0f;
        widened[4 * x + 3] = bpp == 4 ? static_cast<float>(raw[bpp * x + 3]) * 257.0f : 65535.0f;
      }
    }
    return widened.data();
  };
  const std::size_t H = static_cast<std::size_t>(height);
  using Clk = std::chrono::steady_clock;
  Clk::time_point tick = Clk::now();
  // Profiling: wall time of each part into stats_.octree_ms[part].
  const auto lap = [&](int part) {
    const Clk::time_point now = Clk::now();
    if (profiling_) stats_.octree_ms[part] += std::chrono::duration<double, std::milli>(now - tick).count();
    tick = now;
  };
  const std::size_t y0 = out->Begin(row_at, W, H, max_colors, assoc, gray);
  lap(0);
  if (fetch_error != cudaSuccess) return CudaFail(fetch_error, "octree row fetch");
  if (y0 < H) {
    // The first loop's live nodes, by key, to start the second from.
    std::vector<uint64_t> keys;
    std::vector<int32_t> index;
    out->LiveKeys(&keys, &index);
    std::vector<std::size_t> order(keys.size());
    for (std::size_t i = 0; i < order.size(); ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](std::size_t a, std::size_t b) { return keys[a] < keys[b]; });
    const std::size_t n = keys.size();
    std::vector<uint64_t> k_sorted(n), count(n);
    std::vector<double> qerr(n), total(4 * n);
    for (std::size_t i = 0; i < n; ++i) {
      const OctNode& node = out->nodes()[static_cast<std::size_t>(index[order[i]])];
      k_sorted[i] = keys[order[i]];
      qerr[i] = node.qerr;
      count[i] = node.number_unique;
      for (int c = 0; c < 4; ++c) total[4 * i + c] = node.total[c];
    }
    const std::size_t init_bytes = n * (8 + 8 + 8 + 32) + 256;
    if (int rc = Reserve(&octree_init_, init_bytes, "octree seed")) return rc;
    unsigned char* ib = static_cast<unsigned char*>(octree_init_.ptr);
    OctreeRowsLaunch L{};
    L.pixels = static_cast<const unsigned char*>(pixels);
    L.row_stride = static_cast<int64_t>(stride);
    L.width = width;
    L.y0 = static_cast<int64_t>(y0);
    L.pixels_n = static_cast<int64_t>(W * (H - y0));
    L.layout = layout;
    L.assoc = assoc ? 1 : 0;
    L.levels = out->depth();
    L.init_n = static_cast<int>(n);
    L.init_keys = reinterpret_cast<const uint64_t*>(ib);
    L.init_qerr = reinterpret_cast<const double*>(ib + n * 8);
    L.init_count = reinterpret_cast<const uint64_t*>(ib + n * 16);
    L.init_total = reinterpret_cast<const double*>(ib + n * 24);
    cudaError_t e = cudaSuccess;
    if (n && ((e = cudaMemcpyAsync(ib, k_sorted.data(), n * 8, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
              (e = cudaMemcpyAsync(ib + n * 8, qerr.data(), n * 8, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
              (e = cudaMemcpyAsync(ib + n * 16, count.data(), n * 8, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
              (e = cudaMemcpyAsync(ib + n * 24, total.data(), n * 32, cudaMemcpyHostToDevice, s)) != cudaSuccess)) {
      return CudaFail(e, "octree seed upload");
    }
    const std::size_t scratch = OctreeRowsScratch(L.pixels_n, L.levels, assoc);
    if (int rc = Reserve(&octree_scratch_, scratch, "octree classification")) return rc;
    OctreeRows rows;
    if ((e = ClassifyRowsDevice(L, octree_scratch_.ptr, scratch, s, &rows)) != cudaSuccess) {
      return CudaFail(e, "octree classification");
    }
    lap(1);
    if (out->Absorb(rows)) {
      *device_rows = static_cast<int>(H - y0);
    } else {
      out->ClassifyRows(row_at, W, y0, H);
      if (fetch_error != cudaSuccess) return CudaFail(fetch_error, "octree row fetch");
    }
    lap(2);
  }
  out->Finish();
  lap(3);
  return RDB_OK;
}

// The reference's `.idx.bin` debug dump (src/rd_opencl.cpp:2137-2147): the
// walk's index buffer as raw bytes, one per list position.  Synchronous.
int Context::DumpBlockIndices(const BlockLaunch& L, int64_t positions, cudaStream_t s) {
  if (int rc = Reserve(&dump_buf_, static_cast<std::size_t>(positions), "index dump")) return rc;
  uint8_t* d = static_cast<uint8_t*>(dump_buf_.ptr);
  std::vector<uint8_t> host(static_cast<std::size_t>(positions));
  cudaError_t e = LaunchBlockChosenLinear(L, positions, d, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(host.data(), d, host.size(), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return CudaFail(e, "index dump");
  const std::string path = dump_prefix_ + ".idx.bin";
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return Fail(RDB_E_INVALID, "cannot open " + path + " for writing");
  const bool ok = std::fwrite(host.data(), 1, host.size(), f) == host.size();
  if (std::fclose(f) != 0 || !ok) return Fail(RDB_E_INVALID, "cannot write " + path);
  return RDB_OK;
}

std::size_t FrameBytes(int format, int width, int height) {
  if (width < 1 || height < 1) return 0;
  const std::size_t px = static_cast<std::size_t>(width) * static_cast<std::size_t>(height);
  switch (format) {
    case RDB_RGB8: return px * 3;
    case RDB_RGBA8: return px * 4;
    case RDB_RGBAF32: return px * 16;
    case RDB_RGB16: return px * 6;
    case RDB_RGBA16: return px * 8;
    case RDB_YUV444P8: return px * 3;
    case RDB_YUV420P8: return (width % 2 || height % 2) ? 0 : px * 3 / 2;
    default: return 0;
  }
}

int Context::CheckFrames(const rdb_frames& f) const {
  if (f.width < 1 || f.height < 1 || f.frames < 1) {
    return Fail(RDB_E_INVALID, "frames must be at least 1x1 and at least one");
  }
  if (static_cast<int64_t>(f.width) * f.height >= (static_cast<int64_t>(1) << 31) - 1) {
    return Fail(RDB_E_UNSUPPORTED, "frame larger than 2^31 - 2 pixels");
  }
  if (!f.in || !f.out) return Fail(RDB_E_INVALID, "null frame buffer");
  const std::size_t in_bytes = FrameBytes(f.in_format, f.width, f.height);
  if (!in_bytes) {
    return Fail(RDB_E_INVALID, f.in_format == RDB_YUV420P8
                                   ? "4:2:0 frames must have even width and height"
                                   : "unknown input frame format");
  }
  if (f.out_format != RDB_RGBA16 && f.out_format != RDB_YUV444P8 && f.out_format != RDB_RGBAF32) {
    return Fail(RDB_E_INVALID, "output frame format must be RGBA16, YUV444P8 or RGBAF32");
  }
  const std::size_t out_bytes = FrameBytes(f.out_format, f.width, f.height);
  const std::size_t in_pitch = f.in_frame_bytes ? f.in_frame_bytes : in_bytes;
  const std::size_t out_pitch = f.out_frame_bytes ? f.out_frame_bytes : out_bytes;
  if (in_pitch < in_bytes || out_pitch < out_bytes) {
    return Fail(RDB_E_INVALID, "frame stride shorter than a frame");
  }
  // Vector loads and stores: float4 (16), ushort4 / RGBA8 words (8 / 4),
  // uint16 channels (2).
  const auto align = [](int fmt) -> std::size_t {
    switch (fmt) {
      case RDB_RGBAF32: return 16;
      case RDB_RGBA16: return 8;
      case RDB_RGBA8: return 4;
      case RDB_RGB16: return 2;
      default: return 1;
    }
  };
  const std::size_t ai = align(f.in_format), ao = align(f.out_format);
  if ((reinterpret_cast<uintptr_t>(f.in) | in_pitch) % ai ||
      (reinterpret_cast<uintptr_t>(f.out) | out_pitch) % ao) {
    return Fail(RDB_E_INVALID, "frame buffer or stride breaks the format's alignment");
  }
  if (f.in == f.out && !(f.in_format == RDB_RGBAF32 && f.out_format == RDB_RGBAF32 &&
                         in_pitch == out_pitch)) {
    return Fail(RDB_E_INVALID, "only RGBAF32 frames may be dithered in place");
  }
  const DevPlan* p = Plan(f.palette_id);
  if (!p) return Fail(RDB_E_INVALID, "unknown palette id");
  return RDB_OK;
}

int Context::Frames(const rdb_frames& f, const rdb_options& o, cudaStream_t s) {
  if (int rc = CheckFrames(f)) return rc;
  ++call_;
  if (!s) s = stream_;
  cudaSetDevice(device_);
  if (!scratch_ev_) {
    const cudaError_t e = cudaEventCreateWithFlags(&scratch_ev_, cudaEventDisableTiming);
    if (e != cudaSuccess) return CudaFail(e, "scratch event");
  } else if (scratch_stream_ != s) {
    cudaStreamWaitEvent(s, scratch_ev_, 0);
  }
  const std::size_t in_pitch =
      f.in_frame_bytes ? f.in_frame_bytes : FrameBytes(f.in_format, f.width, f.height);
  const std::size_t out_pitch =
      f.out_frame_bytes ? f.out_frame_bytes : FrameBytes(f.out_format, f.width, f.height);
  const std::size_t npx = static_cast<std::size_t>(f.width) * f.height;
  const bool planar = f.in_format == RDB_YUV444P8 || f.in_format == RDB_YUV420P8;
  std::vector<BlockImage> imgs(static_cast<std::size_t>(f.frames));
  for (int k = 0; k < f.frames; ++k) {
    BlockImage& b = imgs[static_cast<std::size_t>(k)];
    b.pixels = static_cast<const unsigned char*>(f.in) + static_cast<std::size_t>(k) * in_pitch;
    b.row_stride = planar ? f.width
                          : static_cast<int64_t>(FrameBytes(f.in_format, f.width, 1));
    b.width = f.width;
    b.height = f.height;
    b.layout = f.in_format;
    b.indices = f.indices ? f.indices + static_cast<std::size_t>(k) * npx : nullptr;
    unsigned char* out = static_cast<unsigned char*>(f.out) + static_cast<std::size_t>(k) * out_pitch;
    if (f.out_format == RDB_RGBAF32) {
      b.rgba_out = (out == b.pixels && BlockListLength(f.width, f.height) == 0)
                       ? nullptr
                       : reinterpret_cast<float4*>(out);
    } else {
      b.raw_out = out;
      b.out_format = f.out_format;
    }
  }
  const int rc = RunBlocks(f.palette_id, f.in_format, imgs, o, s);
  cudaEventRecord(scratch_ev_, s);
  scratch_stream_ = s;
  return rc;
}

int Context::FramesHost(const rdb_frames& f, const rdb_options& o) {
  if (int rc = CheckFrames(f)) return rc;
  const std::size_t in_bytes = FrameBytes(f.in_format, f.width, f.height);
  const std::size_t out_bytes = FrameBytes(f.out_format, f.width, f.height);
  const std::size_t in_pitch = f.in_frame_bytes ? f.in_frame_bytes : in_bytes;
  const std::size_t out_pitch = f.out_frame_bytes ? f.out_frame_bytes : out_bytes;
  const std::size_t frames = static_cast<std::size_t>(f.frames);
  const std::size_t npx = static_cast<std::size_t>(f.width) * f.height;
  // Device frames are packed; 16-byte multiples keep every format aligned.
  const std::size_t din_pitch = (in_bytes + 15) & ~std::size_t{15};
  const std::size_t dout_pitch = (out_bytes + 15) & ~std::size_t{15};
  if (int rc = Reserve(&host_in_, din_pitch * frames, "frame staging")) return rc;
  if (int rc = Reserve(&host_rgba_, dout_pitch * frames, "frame output staging")) return rc;
  if (f.indices && Reserve(&host_idx_, npx * frames, "index staging")) return RDB_E_NOMEM;
  cudaStream_t s = stream_;
  cudaSetDevice(device_);
  cudaError_t e;
  if (in_pitch == din_pitch) {
    e = cudaMemcpyAsync(host_in_.ptr, f.in, in_pitch * frames, cudaMemcpyHostToDevice, s);
  } else {
    e = cudaMemcpy2DAsync(host_in_.ptr, din_pitch, f.in, in_pitch, in_bytes, frames,
                          cudaMemcpyHostToDevice, s);
  }
  if (e != cudaSuccess) return CudaFail(e, "frame upload");
  if (f.indices) cudaMemsetAsync(host_idx_.ptr, 0, npx * frames, s);
  rdb_frames d = f;
  d.in = host_in_.ptr;
  d.in_frame_bytes = din_pitch;
  d.out = (f.out_format == RDB_RGBAF32 && f.in_format == RDB_RGBAF32 && f.out == f.in)
              ? host_in_.ptr
              : host_rgba_.ptr;
  d.out_frame_bytes = dout_pitch;
  d.indices = f.indices ? static_cast<uint8_t*>(host_idx_.ptr) : nullptr;
  if (int rc = Frames(d, o, s)) return rc;
  if (out_pitch == dout_pitch) {
    e = cudaMemcpyAsync(f.out, d.out, out_pitch * frames, cudaMemcpyDeviceToHost, s);
  } else {
    e = cudaMemcpy2DAsync(f.out, out_pitch, d.out, dout_pitch, out_bytes, frames,
                          cudaMemcpyDeviceToHost, s);
  }
  if (e != cudaSuccess) return CudaFail(e, "frame download");
  if (f.indices) {
    e = cudaMemcpyAsync(f.indices, d.indices, npx * frames, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return CudaFail(e, "index download");
  }
  return Synchronize(s);
}

int Context::Jacobi(const rdb_job* jobs, int n, const rdb_options& o, cudaStream_t s) {
  if (o.jacobi_taps < 1 || o.jacobi_taps > 4096) return Fail(RDB_E_UNSUPPORTED, "--approx-taps out of range");
  if (o.jacobi_form != 0 && o.jacobi_form != 1) return Fail(RDB_E_INVALID, "jacobi_form must be 0 or 1");
  if (o.jacobi_form == 0) return JacobiSweeps(jobs, n, o, s);
  if (o.jacobi_iters < 0) return Fail(RDB_E_INVALID, "negative Jacobi iteration count");
  // Impulse response of F = (I - H)^-1 for the walk's own feedback.  The walk
  // adds sw[i] * error[i] with error[15] the newest residual
  // (src/rd_riemersma_cpu.cpp:59-65, :104-112), so lag k carries sw[16 - k]:
  // the newest residual has the SMALLEST weight.  The reference's
  // BuildInverseFilter (src/rd_approx_cuda.cu:73-88) gives lag k w[k-1], the
  // reverse, so its fixed point is not the walk's; rdb_inverse_filter keeps
  // that formula for parity, the engine inverts the real feedback.
  std::vector<double> g(static_cast<std::size_t>(o.jacobi_taps) + 1);
  {
    double sw[kQueue];
    scaled_weights(o.diffusion, sw);
    g[0] = 1.0;
    for (int d = 1; d <= o.jacobi_taps; ++d) {
      double acc = 0.0;
      const int kmax = d < kQueue ? d : kQueue;
      for (int k = 1; k <= kmax; ++k) acc += sw[kQueue - k] * g[d - k];
      g[d] = acc;
    }
  }
  if (int rc = Reserve(&jac_g_, g.size() * sizeof(double), "filter")) return rc;
  cudaMemcpyAsync(jac_g_.ptr, g.data(), g.size() * sizeof(double), cudaMemcpyHostToDevice, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return CudaFail(e, "filter upload");
  for (int i = 0; i < n; ++i) {
    const rdb_job& j = jobs[i];
    const int64_t nb = BlockListLength(j.width, j.height);
    if (nb == 0) {
      if (j.rgba_out && j.rgba_out != j.pixels) {
        e = LaunchCopySource(static_cast<const unsigned char*>(j.pixels),
                             static_cast<int64_t>(RowStride(j)), j.width, j.height, j.layout,
                             reinterpret_cast<float4*>(j.rgba_out), s);
        if (e != cudaSuccess) return CudaFail(e, "source copy");
      }
      continue;
    }
    const DevPlan* p = Plan(j.palette_id);
    const int32_t* order = nullptr;
    if (int rc = Order(j.width, j.height, s, &order)) return rc;
    const std::size_t elem = o.jacobi_fp64 ? sizeof(double) : sizeof(float);
    if (int rc = Reserve(&jac_cx_, static_cast<std::size_t>(nb) * 4 * elem, "Jacobi samples")) return rc;
    if (int rc = Reserve(&jac_q_, static_cast<std::size_t>(nb) * 2 + 64, "Jacobi indices")) return rc;
    JacobiLaunch L{};
    L.pixels = static_cast<const unsigned char*>(j.pixels);
    L.row_stride = static_cast<int64_t>(RowStride(j));
    L.width = j.width;
    L.height = j.height;
    L.layout = j.layout;
    L.n = static_cast<int>(nb);
    L.order = order;
    L.indices = j.indices;
    L.rgba_out = reinterpret_cast<float4*>(j.rgba_out);
    L.plan = p->dev;
    L.plan_smem = p->smem;
    L.iterations = o.jacobi_iters;
    L.taps = o.jacobi_taps;
    L.fp64 = o.jacobi_fp64;
    L.cx = jac_cx_.ptr;
    L.q0 = static_cast<uint8_t*>(jac_q_.ptr);
    L.q1 = L.q0 + ((nb + 31) & ~int64_t{31});
    L.g = static_cast<const double*>(jac_g_.ptr);
    L.status = static_cast<int*>(status_.ptr);
    e = LaunchJacobi(L, s);
    if (e != cudaSuccess) return CudaFail(e, "Jacobi launch");
  }
  return RDB_OK;
}

int Context::Synchronize(cudaStream_t s) {
  if (!s) s = stream_;
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return CudaFail(e, "kernel execution");
  int status = 0;
  e = cudaMemcpy(&status, status_.ptr, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return CudaFail(e, "status readback");
  if (status != 0) {
    cudaMemset(status_.ptr, 0, sizeof(int));
    return Fail(RDB_E_DEVICE, "a kernel reported status " + std::to_string(status));
  }
  return RDB_OK;
}

// Host jobs staged back to back on the context's stream (256-byte aligned
// slices), as device jobs over the staging buffers.
int Context::StageHostJobs(const rdb_host_job* jobs, int n, std::vector<rdb_job>* out) {
  if (n <= 0) return n == 0 ? RDB_OK : Fail(RDB_E_INVALID, "bad job list");
  std::vector<std::size_t> in_off(static_cast<std::size_t>(n)), idx_off(static_cast<std::size_t>(n)),
      rgba_off(static_cast<std::size_t>(n));
  std::size_t in_total = 0, idx_total = 0, rgba_total = 0;
  const auto al = [](std::size_t v) { return (v + 255) & ~static_cast<std::size_t>(255); };
  for (int i = 0; i < n; ++i) {
    const rdb_host_job& j = jobs[i];
    if (j.width < 1 || j.height < 1 || !j.pixels || !j.indices) {
      return Fail(RDB_E_INVALID, "bad host job");
    }
    const std::size_t row = static_cast<std::size_t>(j.width) * BytesPerPixel(j.layout);
    in_off[i] = in_total;
    in_total = al(in_total + row * j.height);
    idx_off[i] = idx_total;
    idx_total = al(idx_total + static_cast<std::size_t>(j.width) * j.height);
    rgba_off[i] = rgba_total;
    if (j.rgba_out) rgba_total = al(rgba_total + static_cast<std::size_t>(j.width) * j.height * 16);
  }
  if (int rc = Reserve(&host_in_, in_total, "input staging")) return rc;
  if (int rc = Reserve(&host_idx_, idx_total, "index staging")) return rc;
  if (rgba_total && Reserve(&host_rgba_, rgba_total, "RgbaF staging")) return RDB_E_NOMEM;
  cudaStream_t s = stream_;
  cudaSetDevice(device_);
  std::vector<rdb_job>& dj = *out;
  dj.assign(static_cast<std::size_t>(n), rdb_job{});
  for (int i = 0; i < n; ++i) {
    const rdb_host_job& j = jobs[i];
    const std::size_t row = static_cast<std::size_t>(j.width) * BytesPerPixel(j.layout);
    unsigned char* din = static_cast<unsigned char*>(host_in_.ptr) + in_off[i];
    cudaError_t e;
    if (j.row_stride == 0 || j.row_stride == row) {
      e = cudaMemcpyAsync(din, j.pixels, row * j.height, cudaMemcpyHostToDevice, s);
    } else {
      e = cudaMemcpy2DAsync(din, row, j.pixels, j.row_stride, row, j.height,
                            cudaMemcpyHostToDevice, s);
    }
    if (e != cudaSuccess) return CudaFail(e, "input upload");
    rdb_job& d = dj[static_cast<std::size_t>(i)];
    d.pixels = din;
    d.row_stride = row;
    d.width = j.width;
    d.height = j.height;
    d.layout = j.layout;
    d.palette_id = j.palette_id;
    d.indices = static_cast<uint8_t*>(host_idx_.ptr) + idx_off[i];
    // RgbaF results follow the reference's in-place semantics: an RgbaF input
    // is dithered in place, so a pixel no engine writes keeps its source.
    d.rgba_out = !j.rgba_out ? nullptr
                 : j.layout == RDB_RGBAF32
                     ? reinterpret_cast<float*>(din)
                     : reinterpret_cast<float*>(static_cast<unsigned char*>(host_rgba_.ptr) +
                                                rgba_off[i]);
  }
  // Cells an engine leaves unwritten (the block list's gap) read back as 0.
  cudaMemsetAsync(host_idx_.ptr, 0, idx_total, s);
  return RDB_OK;
}

// Results of staged host jobs back to their host buffers; waits for them.
int Context::FinishHostJobs(const rdb_host_job* jobs, int n, const std::vector<rdb_job>& dj) {
  cudaStream_t s = stream_;
  for (int i = 0; i < n; ++i) {
    const rdb_host_job& j = jobs[i];
    const std::size_t npx = static_cast<std::size_t>(j.width) * j.height;
    cudaError_t e = cudaMemcpyAsync(j.indices, dj[i].indices, npx, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return CudaFail(e, "index download");
    if (j.rgba_out) {
      e = cudaMemcpyAsync(j.rgba_out, dj[i].rgba_out, npx * 16, cudaMemcpyDeviceToHost, s);
      if (e != cudaSuccess) return CudaFail(e, "RgbaF download");
    }
  }
  return Synchronize(s);
}

int Context::DitherHost(int engine, const rdb_host_job* jobs, int n, const rdb_options& o) {
  std::vector<rdb_job> dj;
  if (int rc = StageHostJobs(jobs, n, &dj)) return rc;
  if (n <= 0) return RDB_OK;
  if (int rc = Dither(engine, dj.data(), n, o, stream_)) return rc;
  return FinishHostJobs(jobs, n, dj);
}

int Context::CreatePaletteFromTree(const Octree& t, int* id) {
  const auto& nodes = t.nodes();
  const auto& cm = t.colormap();
  std::vector<double> colors(cm.size() * 4);
  for (std::size_t i = 0; i < cm.size(); ++i) {
    colors[4 * i] = cm[i].r;
    colors[4 * i + 1] = cm[i].g;
    colors[4 * i + 2] = cm[i].b;
    colors[4 * i + 3] = cm[i].a;
  }
  std::vector<int32_t> child(nodes.size() * 16), parent(nodes.size());
  std::vector<uint32_t> cn(nodes.size());
  std::vector<uint64_t> nu(nodes.size());
  for (std::size_t i = 0; i < nodes.size(); ++i) {
    for (int c = 0; c < 16; ++c) child[16 * i + c] = nodes[i].child[c];
    parent[i] = nodes[i].parent;
    cn[i] = nodes[i].color_number;
    nu[i] = nodes[i].number_unique;
  }
  PlanInput in;
  in.count = t.color_count();
  in.assoc = t.associate_alpha();
  in.colors = colors.data();
  in.node_count = static_cast<int>(nodes.size());
  in.root = 0;
  in.child = child.data();
  in.parent = parent.data();
  in.color_number = cn.data();
  in.number_unique = nu.data();
  return CreatePalette(in, id);
}

int Context::DitherHostBuilding(int engine, const rdb_host_job* jobs, const int* colors,
                                const int* assoc, int n, const rdb_options& o, double* build_ms) {
  std::vector<rdb_job> dj;
  if (int rc = StageHostJobs(jobs, n, &dj)) return rc;
  if (n <= 0) return RDB_OK;
  std::vector<int> pids;
  const auto release = [&] {
    for (int pid : pids) DestroyPalette(pid);
  };
  for (int i = 0; i < n; ++i) {
    const auto t0 = std::chrono::steady_clock::now();
    const rdb_host_job& j = jobs[i];
    const int gray = rdb_is_grayscale(j.pixels, j.layout, static_cast<std::size_t>(j.width),
                                      static_cast<std::size_t>(j.height), j.row_stride);
    Octree tree;
    int rows = 0;
    const std::size_t host_stride =
        j.row_stride ? j.row_stride : static_cast<std::size_t>(j.width) * BytesPerPixel(j.layout);
    int rc = BuildOctree(dj[i].pixels, j.layout, j.width, j.height, static_cast<std::size_t>(dj[i].row_stride),
                         colors[i], assoc[i] != 0, gray != 0, stream_, &tree, &rows, j.pixels, host_stride);
    int pid = 0;
    if (rc == RDB_OK) rc = CreatePaletteFromTree(tree, &pid);
    if (rc != RDB_OK) {
      release();
      return rc;
    }
    pids.push_back(pid);
    dj[static_cast<std::size_t>(i)].palette_id = pid;
    if (build_ms) {
      build_ms[i] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
  }
  int rc = Dither(engine, dj.data(), n, o, stream_);
  if (rc == RDB_OK) rc = FinishHostJobs(jobs, n, dj);
  release();
  return rc;
}

// The speculative segmented walk (rdb_ssw.h): every image is cut into
// segments, all segments of all images run as one persistent launch per pass,
// and passes repeat until each image's verified prefix covers it.
int Context::SeqSegmented(const rdb_job* jobs, int n, const rdb_options& o, cudaStream_t s) {
  const bool use_cache = o.use_cache != 0;
  const int seg_len = o.seg_len > 0 ? std::max(o.seg_len, 64) : 2048;
  const int warm_len = o.warm_len > 0 ? o.warm_len : 1024;
  std::vector<SswImage> imgs(static_cast<std::size_t>(n));
  std::vector<SswSeg> segs;
  int plan_max = 0;
  bool any_assoc = false;
  std::size_t g_bytes = 0;
  std::vector<std::size_t> g_off(static_cast<std::size_t>(n));
  std::vector<uint32_t> g_cap(static_cast<std::size_t>(n));
  int max_seg = 0;
  for (int i = 0; i < n; ++i) {
    const rdb_job& j = jobs[i];
    const DevPlan* p = Plan(j.palette_id);
    const int32_t* order = nullptr;
    if (int rc = Order(j.width, j.height, s, &order)) return rc;
    SswImage& im = imgs[static_cast<std::size_t>(i)];
    std::memset(&im, 0, sizeof(im));
    im.pixels = static_cast<const unsigned char*>(j.pixels);
    im.row_stride = static_cast<int64_t>(RowStride(j));
    im.width = j.width;
    im.height = j.height;
    im.layout = j.layout;
    im.n = j.width * j.height;
    im.order = order;
    im.indices = j.indices;
    im.rgba_out = reinterpret_cast<float4*>(j.rgba_out);
    im.plan = p->dev;
    im.plan_smem = p->smem;
    im.assoc = p->assoc ? 1 : 0;
    plan_max = std::max(plan_max, p->smem);
    any_assoc = any_assoc || p->assoc;
    // Segments of [seg_len, 2 seg_len) positions; a short image is one segment.
    const int k_count = std::max(1, im.n / seg_len);
    im.first_seg = static_cast<int>(segs.size());
    im.nsegs = k_count;
    for (int k = 0; k < k_count; ++k) {
      SswSeg sg{};
      sg.image = i;
      sg.k = k;
      sg.begin = k * seg_len;
      sg.end = (k == k_count - 1) ? im.n : (k + 1) * seg_len;
      sg.warm = k == 0 ? 0 : std::min(sg.begin, warm_len);
      sg.run_tag = 0;
      max_seg = std::max(max_seg, sg.end - sg.begin);
      segs.push_back(sg);
    }
    // G: a direct 2^18 table for RGB keys, a hash sized for the image otherwise.
    uint32_t cap = 1u << 18;
    if (p->assoc) {
      cap = 1024;
      const int64_t want = std::min<int64_t>(2 * static_cast<int64_t>(im.n), int64_t{1} << 25);
      while (static_cast<int64_t>(cap) < want) cap <<= 1;
    }
    g_cap[i] = cap;
    g_off[i] = g_bytes;
    g_bytes += static_cast<std::size_t>(cap) * (p->assoc ? 16 : 8);  // 2 buffers x (vals [+ keys])
  }
  const int total = static_cast<int>(segs.size());
  // L tables: room for twice the distinct keys a segment can touch.
  int ltab_bits = 6;
  const int64_t key_space = any_assoc ? (int64_t{1} << 24) : (int64_t{1} << 18);
  while ((int64_t{1} << ltab_bits) < std::min<int64_t>(2 * static_cast<int64_t>(max_seg), 2 * key_space)) {
    ++ltab_bits;
  }
  const std::size_t ltab_bytes = static_cast<std::size_t>(total) << (ltab_bits + 3);
  const std::size_t q_bytes = static_cast<std::size_t>(total) * 64 * sizeof(double);
  if (int rc = Reserve(&ssw_images_, imgs.size() * sizeof(SswImage), "segmented walk images")) return rc;
  if (int rc = Reserve(&ssw_segs_, segs.size() * sizeof(SswSeg), "segments")) return rc;
  if (int rc = Reserve(&ssw_work_, segs.size() * sizeof(int), "segment work list")) return rc;
  if (int rc = Reserve(&ssw_q_, 2 * q_bytes, "segment queues")) return rc;
  if (use_cache && Reserve(&ssw_ltab_, ltab_bytes, "segment memo tables")) return RDB_E_NOMEM;
  if (use_cache && Reserve(&ssw_g_, g_bytes, "first-touch maps")) return RDB_E_NOMEM;
  if (int rc = Reserve(&ssw_bad_, imgs.size() * sizeof(int), "verification flags")) return rc;
  unsigned char* gbase = static_cast<unsigned char*>(ssw_g_.ptr);
  for (int i = 0; i < n; ++i) {
    SswImage& im = imgs[static_cast<std::size_t>(i)];
    if (!use_cache) continue;
    const uint32_t cap = g_cap[i];
    uint32_t* base = reinterpret_cast<uint32_t*>(gbase + g_off[i]);
    im.g_vals[0] = base;
    im.g_vals[1] = base + cap;
    if (im.assoc) {
      im.g_keys[0] = base + 2 * static_cast<std::size_t>(cap);
      im.g_keys[1] = base + 3 * static_cast<std::size_t>(cap);
      im.g_mask = cap - 1;
    }
  }
  cudaError_t e;
  if ((e = cudaMemcpyAsync(ssw_images_.ptr, imgs.data(), imgs.size() * sizeof(SswImage),
                           cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(ssw_segs_.ptr, segs.data(), segs.size() * sizeof(SswSeg),
                           cudaMemcpyHostToDevice, s)) != cudaSuccess) {
    return CudaFail(e, "segment upload");
  }
  double* q_start = static_cast<double*>(ssw_q_.ptr);
  double* q_end = q_start + static_cast<std::size_t>(total) * 64;
  cudaMemsetAsync(q_start, 0, 2 * q_bytes, s);
  if (use_cache) {
    cudaMemsetAsync(ssw_ltab_.ptr, 0, ltab_bytes, s);
    // G buffer 0 (read by pass 0) empty: vals all ones, keys zero.
    for (int i = 0; i < n; ++i) {
      const SswImage& im = imgs[static_cast<std::size_t>(i)];
      cudaMemsetAsync(im.g_vals[0], 0xFF, static_cast<std::size_t>(g_cap[i]) * 4, s);
      if (im.assoc) cudaMemsetAsync(im.g_keys[0], 0, static_cast<std::size_t>(g_cap[i]) * 4, s);
    }
  }

  // Shared memory per warp: the largest plan, a memo cache, the pixel ring.
  int cache_bits = o.cache_bits > 0 ? o.cache_bits : 11;
  if (cache_bits < 4 || cache_bits > 20) return Fail(RDB_E_INVALID, "cache_bits must be 4..20 (0 = automatic)");
  const std::size_t smem = SswSmemBytes(plan_max, cache_bits);
  if (smem > smem_optin_) return Fail(RDB_E_UNSUPPORTED, "palette plan does not fit in shared memory");
  const int per_sm = std::max(1, std::min<int>(16, static_cast<int>((228 * 1024) / (smem + 1024))));

  SswLaunch L{};
  L.images = static_cast<const SswImage*>(ssw_images_.ptr);
  L.segs = static_cast<SswSeg*>(ssw_segs_.ptr);
  L.work = static_cast<const int*>(ssw_work_.ptr);
  L.q_start = q_start;
  L.q_end = q_end;
  L.ltab = static_cast<uint64_t*>(ssw_ltab_.ptr);
  L.ltab_bits = ltab_bits;
  L.use_cache = use_cache ? 1 : 0;
  L.cache_bits = cache_bits;
  L.plan_smem_max = plan_max;
  L.counter = static_cast<int*>(counter_.ptr);
  L.first_bad = static_cast<int*>(ssw_bad_.ptr);
  L.status = static_cast<int*>(status_.ptr);
  scaled_weights(o.diffusion, L.sw);

  std::vector<int> verified(static_cast<std::size_t>(n), 0);
  std::vector<int> bad(static_cast<std::size_t>(n));
  std::vector<int> work;
  const int max_passes = o.max_passes > 0 ? o.max_passes : 1 << 30;
  int pass = 0;
  for (;; ++pass) {
    if (pass >= max_passes || pass >= 255) {
      return Fail(RDB_E_DEVICE, "segmented walk did not converge within the pass limit");
    }
    work.clear();
    for (int i = 0; i < n; ++i) {
      for (int k = verified[i]; k < imgs[i].nsegs; ++k) work.push_back(imgs[i].first_seg + k);
    }
    if (work.empty()) break;
    L.pass = pass;
    L.tag = pass + 1;
    L.n_work = static_cast<int>(work.size());
    if ((e = cudaMemcpyAsync(ssw_work_.ptr, work.data(), work.size() * sizeof(int),
                             cudaMemcpyHostToDevice, s)) != cudaSuccess) {
      return CudaFail(e, "work list upload");
    }
    if (pass > 0 && (e = LaunchSswCarry(L, s)) != cudaSuccess) return CudaFail(e, "queue carry");
    cudaMemsetAsync(counter_.ptr, 0, sizeof(int), s);
    const int grid = std::min(L.n_work, sm_count_ * per_sm);
    if ((e = LaunchSswWalk(L, grid, s)) != cudaSuccess) return CudaFail(e, "segmented walk");
    if (use_cache) {
      for (int i = 0; i < n; ++i) {
        const SswImage& im = imgs[static_cast<std::size_t>(i)];
        const int wb = (pass & 1) ^ 1;
        cudaMemsetAsync(im.g_vals[wb], 0xFF, static_cast<std::size_t>(g_cap[i]) * 4, s);
        if (im.assoc) cudaMemsetAsync(im.g_keys[wb], 0, static_cast<std::size_t>(g_cap[i]) * 4, s);
      }
      if ((e = LaunchSswBuildG(L, total, s)) != cudaSuccess) return CudaFail(e, "first-touch map");
    }
    cudaMemsetAsync(ssw_bad_.ptr, 0x7F, static_cast<std::size_t>(n) * sizeof(int), s);
    if ((e = LaunchSswVerify(L, s)) != cudaSuccess) return CudaFail(e, "verification");
    if ((e = cudaMemcpyAsync(bad.data(), ssw_bad_.ptr, static_cast<std::size_t>(n) * sizeof(int),
                             cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
      return CudaFail(e, "verification readback");
    }
    int status = 0;
    cudaMemcpy(&status, status_.ptr, sizeof(int), cudaMemcpyDeviceToHost);
    if (status != 0) {
      cudaMemset(status_.ptr, 0, sizeof(int));
      return Fail(RDB_E_DEVICE, "segmented walk reported status " + std::to_string(status));
    }
    for (int i = 0; i < n; ++i) {
      verified[i] = std::min(bad[i], imgs[i].nsegs);
    }
  }
  last_passes_ = pass;
  loop_pending_ = false;  // this call's count, not an earlier device loop's
  if ((e = LaunchSswRgba(L, n, s)) != cudaSuccess) return CudaFail(e, "RgbaF output");
  return RDB_OK;
}

// Automatic sequential mode: short images walk whole on one warp each, long
// ones are segmented on thread walkers.
int Context::SeqAuto(const rdb_job* jobs, int n, const rdb_options& o, cudaStream_t s) {
  std::vector<rdb_job> plain, thread;
  for (int i = 0; i < n; ++i) {
    const rdb_job& j = jobs[i];
    const int64_t px = int64_t{j.width} * j.height;
    (px < 8192 ? plain : thread).push_back(j);
  }
  if (!plain.empty()) {
    if (int rc = Seq(plain.data(), static_cast<int>(plain.size()), o, s)) return rc;
  }
  if (!thread.empty()) {
    if (int rc = SeqThreadSegmented(thread.data(), static_cast<int>(thread.size()), o, s)) return rc;
  }
  return RDB_OK;
}

// The thread-walker segmented walk (rdb_tsw.h): every image's visit order is
// cut into segments of seg_len positions, one thread each; passes repeat
// until each image's verified prefix covers it.
int Context::SeqThreadSegmented(const rdb_job* jobs, int n, const rdb_options& o, cudaStream_t s) {
  // One launch walks palettes of one kind: three channels and direct key maps
  // without alpha, four channels and hashed maps with it.
  {
    std::vector<rdb_job> rgb, alpha;
    for (int i = 0; i < n; ++i) (Plan(jobs[i].palette_id)->assoc ? alpha : rgb).push_back(jobs[i]);
    if (!rgb.empty() && !alpha.empty()) {
      if (int rc = SeqThreadSegmented(rgb.data(), static_cast<int>(rgb.size()), o, s)) return rc;
      return SeqThreadSegmented(alpha.data(), static_cast<int>(alpha.size()), o, s);
    }
  }
  const bool assoc = Plan(jobs[0].palette_id)->assoc;
  const bool use_cache = o.use_cache != 0;
  const int warm_len = std::max(16, o.warm_len > 0 ? o.warm_len : 64);
  constexpr int kChunk = 128;
  constexpr int kKeys = 1 << 18;
  std::vector<TswImage> imgs(static_cast<std::size_t>(n));
  std::vector<TswChunk> chunks;
  int plan_max = 0;
  bool is_float = false;
  int total = 0;
  int64_t positions = 0;
  int64_t all_px = 0;
  for (int i = 0; i < n; ++i) {
    const DevPlan* p = Plan(jobs[i].palette_id);
    plan_max = std::max(plan_max, p->smem);
    all_px += int64_t{jobs[i].width} * jobs[i].height;
  }
  if (TswSmemBytes(plan_max) > smem_optin_) {
    return Fail(RDB_E_UNSUPPORTED, "palette plan does not fit in shared memory");
  }
  // Segment length: as given, else the shortest (at least 64) that keeps
  // every segment of the call on a resident thread -- one wave per pass.
  int seg_len = o.seg_len;
  SegTune* tune = nullptr;
  int tune_slot = -1;
  if (o.walk_form < 0 || o.walk_form > 2) return Fail(RDB_E_INVALID, "walk_form must be 0..2");
  // Paired warps unless their shared memory (the plan, the residual-side
  // colours and the mailboxes) leaves no room for a CTA.
  // Automatic: paired for one image without alpha; with alpha the four-channel
  // ring leaves one paired CTA per SM, and one thread per segment measured
  // faster (4K RGBA: 25.7 ms against 31.3).
  bool paired = o.walk_form == 1 || (o.walk_form == 0 && n == 1 && !assoc);
  if (paired && TswResidentThreads(plan_max, sm_count_, assoc ? 1 : 0, 1) <= 0) paired = false;
  const int64_t resident = std::max(1, TswResidentThreads(plan_max, sm_count_, assoc ? 1 : 0, paired ? 1 : 0));
  // Each image walks a window of segments beyond its front each pass
  // (rdb_tsw.h) -- one image the resident segments, several a share of them
  // each -- so segments can be shorter than "all of them resident" allows: a
  // pass costs seg_len steps, and the front advances about as far per pass in
  // positions, so shorter segments cost fewer steps in total, and no pass
  // walks segments far past a front only to walk them again.
  // Windows by default: one image the resident segments; several share
  // twice that (the 512-image batch: 290 ms without windows; 221 ms with a
  // shared window of twice the resident segments at 192-256 positions, 225 at
  // once them).
  const bool windowed = o.seg_window >= 0;
  if (seg_len <= 0) {
    const int rule = static_cast<int>(std::min<int64_t>(16384, (all_px + resident - 1) / resident));
    int bucket = 0;
    while ((int64_t{1} << (bucket + 1)) <= all_px) ++bucket;
    std::lock_guard<std::mutex> lk(SegTuneLock());
    tune = &SegTuneTable()[std::make_tuple(device_, bucket,
                                           (assoc ? 1 : 0) + (windowed ? 2 : 0) + (paired ? 4 : 0) +
                                               (n > 1 ? 8 : 0))];
    if (tune->cand.empty()) {
      const std::initializer_list<int> all = {rule, rule / 2, rule / 4, rule * 2};
      const std::initializer_list<int> win = {96, 64, 48, 128};
      const std::initializer_list<int> win_batch = {256, 192, 384, 128};
      for (int c : windowed ? (n > 1 ? win_batch : win) : all) {
        c = std::min(16384, (std::max(c, windowed ? 32 : 64) + 15) & ~15);
        if (std::find(tune->cand.begin(), tune->cand.end(), c) == tune->cand.end()) tune->cand.push_back(c);
      }
      tune->ms.assign(tune->cand.size(), -1.0);
    }
    for (std::size_t c = 0; c < tune->cand.size() && tune_slot < 0 && tune->warmed; ++c) {
      if (tune->ms[c] == -1.0) tune_slot = static_cast<int>(c);
    }
    if (!tune->warmed) {
      tune->warmed = true;
      seg_len = tune->cand[0];
    } else if (tune_slot >= 0) {
      tune->ms[static_cast<std::size_t>(tune_slot)] = -2.0;
      seg_len = tune->cand[static_cast<std::size_t>(tune_slot)];
    } else {
      // Fastest measured (others may still be under measurement).
      int best = 0;
      for (std::size_t c = 0; c < tune->cand.size(); ++c) {
        if (tune->ms[c] >= 0 && (tune->ms[static_cast<std::size_t>(best)] < 0 ||
                                 tune->ms[c] < tune->ms[static_cast<std::size_t>(best)])) {
          best = static_cast<int>(c);
        }
      }
      seg_len = tune->cand[static_cast<std::size_t>(best)];
    }
  }
  seg_len = (std::max(seg_len, windowed ? 16 : 64) + 15) & ~15;
  for (int i = 0; i < n; ++i) {
    const rdb_job& j = jobs[i];
    const DevPlan* p = Plan(j.palette_id);
    const int32_t* order = nullptr;
    if (int rc = Order(j.width, j.height, s, &order)) return rc;
    TswImage& im = imgs[static_cast<std::size_t>(i)];
    std::memset(&im, 0, sizeof(im));
    im.pixels = static_cast<const unsigned char*>(j.pixels);
    im.row_stride = static_cast<int64_t>(RowStride(j));
    im.width = j.width;
    im.height = j.height;
    im.layout = j.layout;
    im.n = j.width * j.height;
    im.order = order;
    im.indices = j.indices;
    im.rgba_out = reinterpret_cast<float4*>(j.rgba_out);
    im.plan = p->dev;
    im.plan_smem = p->smem;
    if (int rc = Uniform(j.palette_id, s, &im.uni)) {
      // An alpha palette's table is an accelerator: without room for it the
      // walk answers every key through the memo.
      if (!assoc) return rc;
      im.uni = nullptr;
    }
    im.first_seg = total;
    im.nsegs = (im.n + seg_len - 1) / seg_len;
    im.cx_offset = positions;
    for (int k0 = 0; k0 < im.nsegs; k0 += kChunk) {
      chunks.push_back(TswChunk{i, k0, std::min(kChunk, im.nsegs - k0), 0});
    }
    total += im.nsegs;
    positions += (im.n + 15) & ~15;
    is_float = is_float || j.layout == RDB_RGBAF32;
  }
  int own_bits = 4;
  while ((1 << own_bits) < 2 * seg_len) ++own_bits;
  const std::size_t own_entries = static_cast<std::size_t>(total) << own_bits;
  const std::size_t q_bytes = static_cast<std::size_t>(total) * 64 * sizeof(double);
  // Key maps: direct (3 x 2^18 words per image) without alpha; with alpha a
  // hashed map per image of 4 x n slots (at least 4096, at most 2^25 -- twice
  // the 2^24 possible keys): keys, two first-touch words, usemin, slot list.
  std::vector<uint32_t> hcap(static_cast<std::size_t>(n), 0);
  std::vector<std::size_t> g_off(static_cast<std::size_t>(n), 0);
  std::size_t g_words = 0;
  for (int i = 0; i < n; ++i) {
    const std::size_t si = static_cast<std::size_t>(i);
    g_off[si] = g_words;
    if (assoc) {
      uint32_t cap = 4096;
      const int64_t want = 4 * int64_t{jobs[i].width} * jobs[i].height;
      while (static_cast<int64_t>(cap) < want && cap < (1u << 25)) cap <<= 1;
      hcap[si] = cap;
      g_words += 5 * static_cast<std::size_t>(cap) + 4;
    } else {
      g_words += 3 * static_cast<std::size_t>(kKeys);
    }
  }
  if (int rc = Reserve(&tsw_images_, imgs.size() * sizeof(TswImage), "segmented walk images")) return rc;
  if (int rc = Reserve(&tsw_chunks_, chunks.size() * sizeof(TswChunk), "segment chunks")) return rc;
  if (int rc = Reserve(&tsw_bad_, 3 * static_cast<std::size_t>(n) * sizeof(int), "verification flags")) return rc;
  if (int rc = Reserve(&tsw_q_, 3 * q_bytes, "segment queues")) return rc;
  if (int rc = Reserve(&tsw_cx_, static_cast<std::size_t>(positions) * (is_float ? 16 : 4), "gathered samples")) return rc;
  if (int rc = Reserve(&tsw_chosen_, static_cast<std::size_t>(positions), "segment indices")) return rc;
  if (int rc = Reserve(&tsw_changed_, 4 * static_cast<std::size_t>(total), "segment flags")) return rc;
  if (use_cache) {
    if (int rc = Reserve(&tsw_own_, own_entries * sizeof(uint64_t), "segment memo tables")) return rc;
    if (int rc = Reserve(&tsw_list_, own_entries * sizeof(uint32_t), "segment memo lists")) return rc;
    if (int rc = Reserve(&tsw_count_, static_cast<std::size_t>(total) * sizeof(int), "segment memo counts")) return rc;
    if (int rc = Reserve(&tsw_g_, g_words * sizeof(uint32_t), "first-touch maps")) return rc;
    uint32_t* g = static_cast<uint32_t*>(tsw_g_.ptr);
    for (int i = 0; i < n; ++i) {
      const std::size_t si = static_cast<std::size_t>(i);
      TswImage& im = imgs[si];
      uint32_t* base = g + g_off[si];
      const std::size_t cap = assoc ? hcap[si] : static_cast<std::size_t>(kKeys);
      im.g[0] = base;
      im.g[1] = base + cap;
      im.usemin = base + 2 * cap;
      if (assoc) {
        im.hkeys = base + 3 * cap;
        im.hlist = base + 4 * cap;
        im.hcount = reinterpret_cast<int*>(base + 5 * cap);
        im.hmask = hcap[si] - 1;
      }
    }
  }
  cudaError_t e;
  if ((e = cudaMemcpyAsync(tsw_images_.ptr, imgs.data(), imgs.size() * sizeof(TswImage),
                           cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(tsw_chunks_.ptr, chunks.data(), chunks.size() * sizeof(TswChunk),
                           cudaMemcpyHostToDevice, s)) != cudaSuccess) {
    return CudaFail(e, "segment upload");
  }
  int* bad = static_cast<int*>(tsw_bad_.ptr);
  TswLaunch L{};
  L.images = static_cast<const TswImage*>(tsw_images_.ptr);
  L.n_images = n;
  L.chunks = static_cast<const TswChunk*>(tsw_chunks_.ptr);
  L.n_chunks = static_cast<int>(chunks.size());
  L.seg_len = seg_len;
  L.warm_len = warm_len;
  L.q_start = static_cast<double*>(tsw_q_.ptr);
  L.q_end[0] = L.q_start + static_cast<std::size_t>(total) * 64;
  L.q_end[1] = L.q_end[0] + static_cast<std::size_t>(total) * 64;
  L.own = static_cast<uint64_t*>(tsw_own_.ptr);
  L.own_list = static_cast<uint32_t*>(tsw_list_.ptr);
  L.own_count = static_cast<int*>(tsw_count_.ptr);
  L.own_bits = own_bits;
  L.cx = tsw_cx_.ptr;
  L.chosen = static_cast<uint8_t*>(tsw_chosen_.ptr);
  L.use_cache = use_cache ? 1 : 0;
  L.is_float = is_float ? 1 : 0;
  L.assoc = assoc ? 1 : 0;
  L.plan_smem_max = plan_max;
  L.chunk_threads = kChunk;
  L.bad[0] = bad;
  L.bad[1] = bad + n;
  L.changed = static_cast<uint8_t*>(tsw_changed_.ptr);
  L.walked[0] = L.changed + total;
  L.walked[1] = L.changed + 2 * static_cast<std::size_t>(total);
  L.warmed = L.changed + 3 * static_cast<std::size_t>(total);
  L.paired = paired ? 1 : 0;
  L.window = 0;
  L.win = nullptr;
  if (windowed) {
    // One image: the walk's grid covers the window's chunks plus one, since
    // the front need not sit on a chunk boundary; a window of the resident
    // segments less one chunk keeps that grid within one wave of resident
    // CTAs (with the full resident count, the extra CTA walked a second wave
    // of seg_len steps on its own after the first).
    const int64_t auto_w = n > 1 ? 2 * resident : std::max<int64_t>(1, resident - kChunk);
    const int w = o.seg_window > 0 ? o.seg_window
                                   : static_cast<int>(std::min<int64_t>(auto_w, total));
    if (w < total) {
      if (n == 1) {
        L.window = std::max(1, w);
      } else {
        L.win = bad + 2 * n;
        L.resident_segs = std::max(1, w);
        L.win_min = kBatchWindowMin;
      }
    }
  }
  // Segments dealt to the CTAs interleaved (rdb_tsw.h): one image with a
  // window or without, several with per-image windows.
  L.spread = (n == 1 || L.win) ? 1 : 0;
  if (L.window > 0 || L.win) cudaMemsetAsync(L.walked[0], 0, 2 * static_cast<std::size_t>(total), s);
  L.walk_count = nullptr;
  if (profiling_) {
    L.walk_count = reinterpret_cast<unsigned long long*>(static_cast<unsigned char*>(status_.ptr) + 64);
    cudaMemsetAsync(L.walk_count, 0, sizeof(unsigned long long), s);
  }
  L.status = static_cast<int*>(status_.ptr);
  scaled_weights(o.diffusion, L.sw);

  // Pass 0 reads bad[1] as "nothing verified" and g[1] as the empty map.
  cudaMemsetAsync(L.bad[1], 0, static_cast<std::size_t>(n) * sizeof(int), s);
  if (use_cache) {
    cudaMemsetAsync(tsw_own_.ptr, 0, own_entries * sizeof(uint64_t), s);
    for (int i = 0; i < n; ++i) {
      const TswImage& im = imgs[static_cast<std::size_t>(i)];
      if (assoc) {
        // Empty keys and counts; every first-touch and usemin word "none".
        const std::size_t cap = hcap[static_cast<std::size_t>(i)];
        cudaMemsetAsync(im.g[0], 0xFF, 3 * cap * sizeof(uint32_t), s);
        cudaMemsetAsync(im.hkeys, 0, cap * sizeof(uint32_t), s);
        cudaMemsetAsync(im.hcount, 0, 3 * sizeof(int), s);  // count, classified, to classify
      } else {
        cudaMemsetAsync(im.g[1], 0xFF, kKeys * sizeof(uint32_t), s);
      }
    }
  }
  if ((e = LaunchTswGather(L, positions, s)) != cudaSuccess) return CudaFail(e, "sample gather");
  if (L.win) {
    // Pass 0's windows, from every front at 0 (bad[1] as pass 0 reads it).
    TswLaunch first = L;
    first.pass = 1;
    if ((e = LaunchTswWindows(first, s)) != cudaSuccess) return CudaFail(e, "segment windows");
  }

  const int max_passes_opt = o.max_passes > 0 ? o.max_passes : 1 << 30;
  const bool device_loop = o.loop_mode == 2 || (o.loop_mode == 0 && !profiling_);
  if (o.loop_mode < 0 || o.loop_mode > 2) return Fail(RDB_E_INVALID, "loop_mode must be 0..2");
  if (device_loop) {
    if (int rc = Reserve(&tsw_ctl_, 64, "loop control")) return rc;
    static const int kCtlInit[8] = {0, 0, 0, 0, 3, 0, 0, 0};  // counters, then the tag of pass 2
    int* ctl = static_cast<int*>(tsw_ctl_.ptr);
    uint32_t* tag_dev = reinterpret_cast<uint32_t*>(ctl + 4);
    if ((e = cudaMemcpyAsync(ctl, kCtlInit, sizeof(kCtlInit), cudaMemcpyHostToDevice, s)) != cudaSuccess) {
      return CudaFail(e, "loop control");
    }
    TswLaunch even = L, odd = L;
    even.pass = 2;
    odd.pass = 3;
    even.tag_dev = odd.tag_dev = tag_dev;
    const int loop_max = std::max(1, max_passes_opt - 2);
    // The executable graph is rebuilt only when the launch parameters change.
    std::vector<unsigned char> key(sizeof(TswLaunch) + 2 * sizeof(int));
    std::memcpy(key.data(), &even, sizeof(TswLaunch));
    std::memcpy(key.data() + sizeof(TswLaunch), &total, sizeof(int));
    std::memcpy(key.data() + sizeof(TswLaunch) + sizeof(int), &loop_max, sizeof(int));
    if (!loop_exec_ || key != loop_key_) {
      if (loop_exec_) {
        cudaGraphExecDestroy(loop_exec_);
        loop_exec_ = nullptr;
      }
      cudaGraph_t g = nullptr;
      if ((e = BuildTswLoopGraph(even, odd, total, ctl, tag_dev, loop_max, &g)) != cudaSuccess) {
        return CudaFail(e, "pass-loop graph");
      }
      e = cudaGraphInstantiate(&loop_exec_, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        loop_exec_ = nullptr;
        return CudaFail(e, "pass-loop graph instantiation");
      }
      loop_key_ = key;
    }
  }
  // The tuner times the passes on the device: setup, uploads and the graph's
  // instantiation above are outside its events.
  const bool timing = tune && tune_slot >= 0;
  if (timing) {
    for (cudaEvent_t& ev : tune_ev_) {
      if (!ev && (e = cudaEventCreate(&ev)) != cudaSuccess) return CudaFail(e, "tuner events");
    }
    cudaEventRecord(tune_ev_[0], s);
  }
  if (device_loop) {
    // Passes 0 and 1 from the host (pass 0 is the warm-up pass), then the
    // rest as one graph launch: nothing here waits for the device.
    for (int pass = 0; pass < 2; ++pass) {
      L.pass = pass;
      L.tag = static_cast<uint32_t>(pass + 1);
      cudaMemsetAsync(L.bad[pass & 1], 0x7F, static_cast<std::size_t>(n) * sizeof(int), s);
      if ((e = LaunchTswPrepare(L, s)) != cudaSuccess) return CudaFail(e, "first-touch map");
      if ((e = LaunchTswWalk(L, s)) != cudaSuccess) return CudaFail(e, "segmented walk");
      if ((e = LaunchTswVerify(L, total, s)) != cudaSuccess) return CudaFail(e, "verification");
      if ((e = LaunchTswWindows(L, s)) != cudaSuccess) return CudaFail(e, "segment windows");
    }
    if ((e = cudaGraphLaunch(loop_exec_, s)) != cudaSuccess) return CudaFail(e, "pass-loop graph launch");
    if ((e = LaunchTswScatter(L, positions, s)) != cudaSuccess) return CudaFail(e, "index scatter");
    loop_pending_ = true;
    loop_stream_ = s;
    if (timing) {
      // The tuner still needs this length's time: wait for it here.
      cudaEventRecord(tune_ev_[1], s);
      cudaEventSynchronize(tune_ev_[1]);
      float ms = 0.0f;
      std::lock_guard<std::mutex> lk(SegTuneLock());
      tune->ms[static_cast<std::size_t>(tune_slot)] =
          cudaEventElapsedTime(&ms, tune_ev_[0], tune_ev_[1]) == cudaSuccess ? ms : -1.0;
    }
    return RDB_OK;
  }

  // Passes are enqueued up to kDepth ahead of the one the host is checking:
  // every kernel takes its verified prefix from the device's own result of
  // the previous pass, so the host only has to learn when to stop.  Each pass
  // copies its per-image first failure and the status word into a pinned
  // ring slot and records an event; passes enqueued past convergence find
  // every segment verified and walk nothing.
  constexpr int kDepth = 4;
  const std::size_t slot_ints = static_cast<std::size_t>(n) + 1;
  if (int rc = PinnedRing(kDepth * slot_ints)) return rc;
  if (int rc = PassEvents(kDepth)) return rc;
  std::vector<int> front(static_cast<std::size_t>(n), -1);
  const int max_passes = o.max_passes > 0 ? o.max_passes : 1 << 30;
  const auto drain = [&](int code, const std::string& msg) {
    cudaStreamSynchronize(s);
    cudaMemset(status_.ptr, 0, sizeof(int));
    return Fail(code, msg);
  };
  int issued = 0, checked = 0;
  bool done = false;
  while (!done) {
    while (issued < checked + kDepth && issued < max_passes) {
      const int k = issued % kDepth;
      L.pass = issued;
      L.tag = static_cast<uint32_t>(issued + 1);
      int* cur = L.bad[issued & 1];
      cudaMemsetAsync(cur, 0x7F, static_cast<std::size_t>(n) * sizeof(int), s);
      if ((e = LaunchTswPrepare(L, s)) != cudaSuccess) return drain(RDB_E_CUDA, CudaErr(e, "first-touch map"));
      if (profiling_) cudaEventRecord(walk_ev_[2 * k], s);
      if ((e = LaunchTswWalk(L, s)) != cudaSuccess) return drain(RDB_E_CUDA, CudaErr(e, "segmented walk"));
      if (profiling_) cudaEventRecord(walk_ev_[2 * k + 1], s);
      if ((e = LaunchTswVerify(L, total, s)) != cudaSuccess) return drain(RDB_E_CUDA, CudaErr(e, "verification"));
      if ((e = LaunchTswWindows(L, s)) != cudaSuccess) return drain(RDB_E_CUDA, CudaErr(e, "segment windows"));
      int* slot = ring_h_ + static_cast<std::size_t>(k) * slot_ints;
      if ((e = cudaMemcpyAsync(slot, cur, static_cast<std::size_t>(n) * sizeof(int),
                               cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
          (e = cudaMemcpyAsync(slot + n, status_.ptr, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
          (e = cudaEventRecord(pass_ev_[k], s)) != cudaSuccess) {
        return drain(RDB_E_CUDA, CudaErr(e, "verification readback"));
      }
      // walk, checks, [prepare, keys, alpha-key classification]
      if (profiling_) stats_.launches += 1 + 1 + (use_cache ? (assoc ? 3 : 2) : 0) + (L.win ? 1 : 0);
      ++issued;
    }
    if (checked == issued) return drain(RDB_E_DEVICE, "segmented walk did not converge within the pass limit");
    const int k = checked % kDepth;
    if ((e = cudaEventSynchronize(pass_ev_[k])) != cudaSuccess) return drain(RDB_E_CUDA, CudaErr(e, "pass wait"));
    const int* slot = ring_h_ + static_cast<std::size_t>(k) * slot_ints;
    if (slot[n] != 0) {
      return drain(RDB_E_DEVICE, "segmented walk reported status " + std::to_string(slot[n]));
    }
    if (profiling_) {
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, walk_ev_[2 * k], walk_ev_[2 * k + 1]);
      stats_.walk_ms += ms;
      stats_.walk_launches += 1;
      stats_.passes += 1;
    }
    // The verified prefix of every unfinished image grows by at least one
    // segment a pass (its first walked segment started from exact state);
    // anything else is an engine fault, reported rather than looped on.
    done = true;
    for (int i = 0; i < n; ++i) {
      const std::size_t si = static_cast<std::size_t>(i);
      const int nf = std::min(slot[i], imgs[si].nsegs);
      if (nf < imgs[si].nsegs && nf <= front[si]) {
        return drain(RDB_E_DEVICE, "segmented walk made no progress on an image");
      }
      front[si] = nf;
      done = done && nf >= imgs[si].nsegs;
    }
    ++checked;
  }
  const int pass = checked - 1;
  if (timing) {
    // The last checked pass's completion event was recorded after its
    // verification: time from the first pass's start to it.
    float ms = 0.0f;
    cudaEventRecord(tune_ev_[1], s);
    cudaEventSynchronize(tune_ev_[1]);
    std::lock_guard<std::mutex> lk(SegTuneLock());
    tune->ms[static_cast<std::size_t>(tune_slot)] =
        cudaEventElapsedTime(&ms, tune_ev_[0], tune_ev_[1]) == cudaSuccess ? ms : -1.0;
  }
  last_passes_ = pass + 1;
  loop_pending_ = false;  // this call's count, not an earlier device loop's
  if ((e = LaunchTswScatter(L, positions, s)) != cudaSuccess) return CudaFail(e, "index scatter");
  if (profiling_) {
    stats_.launches += 2 + (L.win ? 1 : 0);  // gather, scatter, first windows
    stats_.seg_len = seg_len;
    stats_.chains = total;
    unsigned long long walked = 0;
    if (cudaMemcpyAsync(&walked, L.walk_count, sizeof(walked), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
        cudaStreamSynchronize(s) == cudaSuccess) {
      stats_.walk_positions += static_cast<int64_t>(walked);
    }
  }
  return RDB_OK;
}

std::size_t ScratchBound(int engine, int width, int height, int layout, bool assoc, bool rgba_out,
                         const rdb_options& o) {
  using sz = std::size_t;
  const sz n = static_cast<sz>(std::max(width, 1)) * static_cast<sz>(std::max(height, 1));
  const bool is_float = layout == RDB_RGBAF32;
  // Staging (StageHostJobs, 256-byte aligned slices), the visit order and its
  // builder's scratch (Order), the palette's plan block (a shared-memory
  // image, so below the opt-in limit, in 16 KiB classes) and uniform-key table.
  sz b = n * BytesPerPixel(layout) + n + (rgba_out ? 16 * n : 0) + 3 * 256;
  b += 4 * n + CurveScratchBytes(CurveLevel(width, height));
  b += (sz{256} << 10) + (assoc ? sz{kUniformKeysAlpha} : sz{kUniformKeys});
  const auto blocks = [&](sz block, bool sweeps) {
    // RunBlocks: groups of 32 blocks of bpad <= block + 15 cells; the
    // candidate table without alpha; the sweeps' two end-queue buffers.
    const sz nb = (n + block - 1) / block;
    const sz cells = (nb + 31) / 32 * 32 * (block + 15);
    sz r = cells * ((is_float ? 16 : 4) + 1) + (assoc ? 0 : sz{kCandKeys} * 4) + 64 * nb;
    if (sweeps) r += 2 * nb * 64 * sizeof(double) + 256;
    return r;
  };
  if (engine == RDB_ENGINE_BLOCKS) return b + blocks(static_cast<sz>(std::max(o.block, 16)), false);
  if (engine == RDB_ENGINE_JACOBI) {
    if (o.jacobi_form == 0) return b + blocks(256, true);
    const sz elem = o.jacobi_fp64 ? 8 : 4;
    return b + n * 4 * elem + 2 * n + 64 + (static_cast<sz>(std::max(o.jacobi_taps, 0)) + 1) * 8;
  }
  const bool use_cache = o.use_cache != 0;
  int mode = o.seq_mode;
  if (mode == 0) mode = n < 8192 ? 1 : 3;  // SeqAuto's rule
  if (mode == 1) {
    // One memo slab (2^18 or 2^24 uint16 keys plus its generation) and a work
    // item; the walk's CTAs never outnumber its images.
    return b + (use_cache ? (assoc ? (sz{1} << 25) : (sz{1} << 19)) + 4 : 0) + 256;
  }
  if (mode == 2) {
    // SeqSegmented: segments of [seg, 2 seg) positions, memo tables of fewer
    // than 4 x 2 seg 8-byte entries, two queues each; first-touch maps.
    const sz seg = static_cast<sz>(o.seg_len > 0 ? std::max(o.seg_len, 64) : 2048);
    const sz segs = std::max<sz>(1, n / seg);
    sz r = segs * (2 * 64 * sizeof(double) + 64) + 64;
    if (use_cache) {
      r += segs * 8 * 8 * seg;
      sz cap = sz{1} << 18;
      if (assoc) {
        cap = 1024;
        while (cap < std::min<sz>(2 * n, sz{1} << 25)) cap <<= 1;
      }
      r += cap * (assoc ? 16 : 8);
    }
    return b + r;
  }
  // SeqThreadSegmented: segments of at least 16 positions (32 when the tuner
  // picks), three queue buffers and four flag bytes each; samples and
  // indices; memo tables below 4 entries per position (16 at least per
  // segment) of 8 + 4 bytes; first-touch maps (3 direct 2^18-word maps, or 5
  // words per slot of a hashed map of 4n..8n slots).
  const sz seg = static_cast<sz>(o.seg_len > 0 ? std::max(16, o.seg_len) : 32);
  const sz segs = n / seg + 1;
  sz r = (n + 16) * ((is_float ? 16 : 4) + 1) + segs * (3 * 64 * sizeof(double) + 4 + 4) +
         (segs / 128 + 1) * sizeof(TswChunk) + sizeof(TswImage) + 64;
  if (use_cache) {
    r += (4 * (n + 16384) + 16 * segs) * 12 + 4 * segs;  // the last segment may be partial
    if (assoc) {
      sz cap = 4096;
      while (cap < 4 * n && cap < (sz{1} << 25)) cap <<= 1;
      r += 5 * cap * 4 + 16;
    } else {
      r += 3 * (sz{1} << 18) * 4;
    }
  }
  return b + r;
}

}  // namespace rdb
