// rdb_serve.cpp -- the request loop declared in include/rdb.h (rdb_server_*).
//
// Stages joined by queues under one mutex:
//   build    the request's colour tree (the reference's ColorTree::Build
//            semantics, greyscale rule of src/rd_cli.cpp:2452-2456).  By
//            default host threads build it (rdb_octree_build) before
//            admission, parallel by request; with device_palettes the device
//            worker builds it from the uploaded pixels
//            (rdb_octree_build_device) at the start of the batch call;
//   admit    a request waits until the device-memory estimate of all
//            admitted requests plus its own fits the budget (first fit in
//            arrival order, so one large request does not block small ones
//            behind it forever: it is taken as soon as it fits);
//   device   each worker owns a context and its stream; when idle it takes
//            every admitted request that shares the oldest one's engine and
//            options (a block request alone: that engine walks one palette
//            per call) as one batched call, so arrivals during a batch form
//            the next batch on whichever worker frees first.
// A request's result does not depend on its batch: every engine treats the
// jobs of a call independently.
#include <sched.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/rdb.h"
#include "rdb_octree_dev.h"
#include "rdb_runtime.h"

namespace {

using Clock = std::chrono::steady_clock;

double Ms(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// CPUs this process may run on: its affinity mask, capped by a cgroup (v2 or
// v1) CPU quota when one is set.  hardware_concurrency() counts every CPU of
// the machine, which oversubscribes a container limited to a few of them.
int UsableCpus() {
  int n = 0;
  cpu_set_t set;
  CPU_ZERO(&set);
  if (sched_getaffinity(0, sizeof(set), &set) == 0) n = CPU_COUNT(&set);
  if (n <= 0) n = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
  double quota = -1.0;
  if (FILE* f = std::fopen("/sys/fs/cgroup/cpu.max", "r")) {
    char q[64] = {0};
    long long period = 0;
    if (std::fscanf(f, "%63s %lld", q, &period) == 2 && std::strcmp(q, "max") != 0 && period > 0) {
      quota = std::atof(q) / static_cast<double>(period);
    }
    std::fclose(f);
  } else if (FILE* f1 = std::fopen("/sys/fs/cgroup/cpu/cpu.cfs_quota_us", "r")) {
    long long qu = -1, period = 0;
    if (std::fscanf(f1, "%lld", &qu) == 1 && qu > 0) {
      if (FILE* f2 = std::fopen("/sys/fs/cgroup/cpu/cpu.cfs_period_us", "r")) {
        if (std::fscanf(f2, "%lld", &period) == 1 && period > 0) {
          quota = static_cast<double>(qu) / static_cast<double>(period);
        }
        std::fclose(f2);
      }
    }
    std::fclose(f1);
  }
  if (quota > 0.0) n = std::min(n, std::max(1, static_cast<int>(quota + 0.5)));
  return std::max(1, n);
}

struct Req {
  rdb_request r{};
  uint64_t ticket = 0;
  Clock::time_point t_submit, t_build_start, t_built, t_start, t_done;
  rdb_octree* tree = nullptr;
  std::size_t bytes = 0;
  int status = RDB_OK;
  bool done = false;
  int batch = 0;
  double device_ms = 0.0;
  std::string err;
};

// Device bytes an idle context keeps after releasing its buffers (its work
// counter, status word and loop control words).
constexpr std::size_t kContextFloor = 4096;

// The octree build's classification depth (rd_octree.cpp:255-275).
int TreeDepth(int colors, bool assoc, bool gray) {
  int depth = 1;
  for (std::size_t c = static_cast<std::size_t>(colors > 0 ? colors : 65536); c != 0; ++depth) c >>= 2;
  if (depth > 2) --depth;
  if (assoc && depth > 5) --depth;
  if (gray) depth = 8;
  return std::min(8, std::max(2, depth));
}

// Device bytes one request needs while admitted: the runtime's bound for its
// engine and path (rdb::ScratchBound: staging, visit order, palette tables,
// the walk's scratch) and, when its palette is built on the device, that
// build's classification scratch.
std::size_t EstimateBytes(const rdb_request& r, bool device_palette) {
  const std::size_t px = static_cast<std::size_t>(r.width) * r.height;
  std::size_t build = 0;
  if (device_palette) {
    const bool gray = rdb_is_grayscale(r.pixels, r.layout, static_cast<std::size_t>(r.width),
                                       static_cast<std::size_t>(r.height), r.row_stride) != 0;
    build = rdb::OctreeRowsScratch(static_cast<int64_t>(px),
                                   TreeDepth(r.colors, r.associate_alpha != 0, gray),
                                   r.associate_alpha != 0);
  }
  return rdb::ScratchBound(r.engine, r.width, r.height, r.layout, r.associate_alpha != 0,
                           r.rgba_out != nullptr, r.options) +
         build + (std::size_t{1} << 20);
}

bool SameOptions(const rdb_options& a, const rdb_options& b) {
  return std::memcmp(&a, &b, sizeof(rdb_options)) == 0;
}

}  // namespace

struct rdb_server {
  rdb_server_options o{};
  std::size_t budget = 0;
  std::mutex mu;
  std::condition_variable cv_build, cv_ready, cv_done;
  std::deque<Req*> incoming;
  std::deque<Req*> ready;
  std::unordered_map<uint64_t, Req*> all;
  uint64_t next_ticket = 1;
  std::size_t admitted = 0;
  bool stop = false;
  int pending = 0;  // submitted, not yet completed
  std::vector<std::thread> builders, workers;
  // statistics: per completed request, its stage durations (RDB_STAGE_*)
  std::vector<std::array<double, RDB_STAGES>> latencies;
  int64_t failed = 0, pixels = 0, batches = 0;
  bool any = false;
  Clock::time_point first_submit, last_done;
  std::size_t peak = 0;
  // Per worker: its context, the device bytes that context holds between
  // batches (counted against the budget like admitted requests), and whether
  // it is running a batch.
  std::vector<rdb_context*> ctxs;
  std::vector<std::size_t> cached;
  std::vector<char> busy;

  void Build();
  void Work(int index);
  std::vector<Req*> TakeBatch();
  std::size_t Held() const;
  bool TrimIdle();
};

std::size_t rdb_server::Held() const {
  std::size_t h = admitted;
  for (std::size_t c : cached) h += c;
  return h;
}

// Under the lock: idle workers' contexts release their cached buffers (the
// workers wait on the lock, so nothing uses those contexts meanwhile).
// False when none held anything to release.
bool rdb_server::TrimIdle() {
  bool any_freed = false;
  for (std::size_t w = 0; w < ctxs.size(); ++w) {
    if (!ctxs[w] || busy[w] || cached[w] == 0) continue;
    const std::size_t before = ctxs[w]->impl.bytes();
    ctxs[w]->impl.ReleaseScratch();
    cached[w] = ctxs[w]->impl.bytes();
    any_freed = any_freed || cached[w] < before;
  }
  return any_freed;
}

void rdb_server::Build() {
  for (;;) {
    Req* q = nullptr;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_build.wait(lk, [&] { return stop || !incoming.empty(); });
      if (incoming.empty()) return;
      q = incoming.front();
      incoming.pop_front();
      q->t_build_start = Clock::now();
    }
    const rdb_request& r = q->r;
    const int gray = rdb_is_grayscale(r.pixels, r.layout, r.width, r.height, r.row_stride);
    const int rc = rdb_octree_build(r.pixels, r.layout, r.width, r.height, r.row_stride, r.colors,
                                    r.associate_alpha, gray, &q->tree);
    std::lock_guard<std::mutex> lk(mu);
    q->t_built = Clock::now();
    if (rc != RDB_OK) {
      q->status = rc;
      q->err = std::string("palette build: ") + rdb_last_error();
      q->done = true;
      q->t_done = q->t_built;
      ++failed;
      --pending;
      cv_done.notify_all();
      continue;
    }
    ready.push_back(q);
    cv_ready.notify_all();
  }
}

// Under the lock: the oldest admissible request and every other admissible
// request compatible with it, admitted now.
std::vector<Req*> rdb_server::TakeBatch() {
  std::vector<Req*> batch;
  Req* head = nullptr;
  for (int attempt = 0; attempt < 2 && !head && !ready.empty(); ++attempt) {
    for (Req* q : ready) {
      if (Held() + q->bytes <= budget) {
        head = q;
        break;
      }
    }
    // Nothing fits: idle contexts give back their caches, then once more.
    // With no batch running every context is idle, so the oldest request
    // (never above the budget) then fits.
    if (!head && !TrimIdle()) break;
  }
  if (!head) return batch;
  const int max_batch = o.max_batch > 0 ? o.max_batch : 512;
  for (auto it = ready.begin(); it != ready.end() && static_cast<int>(batch.size()) < max_batch;) {
    Req* q = *it;
    const bool compatible = q == head ||
                            (q->r.engine == head->r.engine && SameOptions(q->r.options, head->r.options) &&
                             q->r.engine != RDB_ENGINE_BLOCKS);
    if (compatible && (q == head || Held() + q->bytes <= budget)) {
      admitted += q->bytes;
      batch.push_back(q);
      it = ready.erase(it);
    } else {
      ++it;
    }
  }
  peak = std::max(peak, Held());
  return batch;
}

void rdb_server::Work(int index) {
  rdb_context* ctx = nullptr;
  // Between batches a context keeps its buffers for the next one, up to an
  // equal share of the budget; past that it releases them.
  const std::size_t share = budget / static_cast<std::size_t>(std::max(1, o.workers));
  const std::size_t w = static_cast<std::size_t>(index);
  cudaSetDevice(o.device);
  const int crc = rdb_context_create(o.device, budget, &ctx);
  {
    std::lock_guard<std::mutex> lk(mu);
    ctxs[w] = crc == RDB_OK ? ctx : nullptr;
    cached[w] = crc == RDB_OK ? ctx->impl.bytes() : 0;
  }
  for (;;) {
    std::vector<Req*> batch;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_ready.wait(lk, [&] {
        if (stop && ready.empty() && incoming.empty() && pending == 0) return true;
        if (ready.empty()) return false;
        batch = TakeBatch();
        return !batch.empty();
      });
      if (batch.empty()) break;
      busy[w] = 1;
      // The batch may hold what the context already has plus its admitted
      // bytes, and no more.
      std::size_t want = cached[w];
      for (Req* q : batch) want += q->bytes;
      if (crc == RDB_OK) ctx->impl.SetBudget(want);
    }
    const Clock::time_point t0 = Clock::now();
    std::vector<int> pids(batch.size(), 0);
    std::vector<rdb_host_job> jobs(batch.size());
    std::vector<int> colors(batch.size()), assoc(batch.size());
    std::vector<double> build_ms(batch.size(), 0.0);
    const bool on_device = o.device_palettes != 0;
    int rc = crc;
    for (std::size_t i = 0; i < batch.size() && rc == RDB_OK; ++i) {
      if (!on_device) rc = rdb_palette_from_octree(ctx, batch[i]->tree, &pids[i]);
      const rdb_request& r = batch[i]->r;
      rdb_host_job& j = jobs[i];
      j.pixels = r.pixels;
      j.row_stride = r.row_stride;
      j.width = r.width;
      j.height = r.height;
      j.layout = r.layout;
      j.palette_id = pids[i];
      j.indices = r.indices;
      j.rgba_out = r.rgba_out;
      colors[i] = r.colors;
      assoc[i] = r.associate_alpha;
    }
    if (rc == RDB_OK) {
      if (on_device) {
        rc = ctx->impl.DitherHostBuilding(batch[0]->r.engine, jobs.data(), colors.data(), assoc.data(),
                                          static_cast<int>(jobs.size()), batch[0]->r.options,
                                          build_ms.data());
      } else {
        rc = rdb_dither_host(ctx, batch[0]->r.engine, jobs.data(), static_cast<int>(jobs.size()),
                             &batch[0]->r.options);
      }
    }
    const std::string err = rc == RDB_OK ? std::string() : std::string(rdb_last_error());
    for (int pid : pids) {
      if (pid) rdb_palette_destroy(ctx, pid);
    }
    const Clock::time_point t1 = Clock::now();
    if (crc == RDB_OK && ctx->impl.bytes() > share) ctx->impl.ReleaseScratch();
    // Built on the device: the builds ran one after another at the start of
    // the batch call, then the walk.
    Clock::time_point dither_start = t0;
    if (on_device) {
      double cum = 0.0;
      for (std::size_t i = 0; i < batch.size(); ++i) {
        const auto at = [&](double ms) {
          return t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double, std::milli>(ms));
        };
        batch[i]->t_build_start = at(cum);
        cum += build_ms[i];
        batch[i]->t_built = at(cum);
      }
      dither_start = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double, std::milli>(cum));
    }
    std::lock_guard<std::mutex> lk(mu);
    ++batches;
    busy[w] = 0;
    cached[w] = crc == RDB_OK ? ctx->impl.bytes() : 0;
    for (Req* q : batch) {
      rdb_octree_free(q->tree);
      q->tree = nullptr;
      q->status = rc;
      q->t_start = on_device ? dither_start : t0;
      q->t_done = t1;
      q->device_ms = Ms(q->t_start, t1);
      q->batch = static_cast<int>(batch.size());
      q->err = err;
      q->done = true;
      admitted -= q->bytes;
      --pending;
      if (rc == RDB_OK) {
        latencies.push_back({Ms(q->t_submit, q->t_build_start), Ms(q->t_build_start, q->t_built),
                             Ms(q->t_built, q->t_start), Ms(q->t_start, t1), Ms(q->t_submit, t1)});
        pixels += static_cast<int64_t>(q->r.width) * q->r.height;
        last_done = t1;
      } else {
        ++failed;
      }
    }
    cv_done.notify_all();
    cv_ready.notify_all();  // memory freed: other workers may admit now
  }
  {
    std::lock_guard<std::mutex> lk(mu);
    ctxs[w] = nullptr;
    cached[w] = 0;
  }
  if (ctx) rdb_context_destroy(ctx);
}

extern "C" {

int rdb_server_create(const rdb_server_options* opts, rdb_server** out) {
  if (!out) return rdb::Fail(RDB_E_INVALID, "rdb_server_create: null output");
  rdb_server* s = new rdb_server();
  if (opts) s->o = *opts;
  if (s->o.workers <= 0) s->o.workers = 4;
  if (s->o.host_threads <= 0) s->o.host_threads = UsableCpus();
  if (cudaSetDevice(s->o.device) != cudaSuccess) {
    delete s;
    return rdb::Fail(RDB_E_CUDA, "rdb_server_create: no such device");
  }
  std::size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
    delete s;
    return rdb::Fail(RDB_E_CUDA, "rdb_server_create: cudaMemGetInfo failed");
  }
  s->budget = s->o.memory_budget ? std::min(s->o.memory_budget, (free_b / 10) * 9) : (free_b / 10) * 9;
  if (!s->o.device_palettes) {
    for (int i = 0; i < s->o.host_threads; ++i) s->builders.emplace_back([s] { s->Build(); });
  }
  s->ctxs.assign(static_cast<std::size_t>(s->o.workers), nullptr);
  s->cached.assign(static_cast<std::size_t>(s->o.workers), 0);
  s->busy.assign(static_cast<std::size_t>(s->o.workers), 0);
  for (int i = 0; i < s->o.workers; ++i) s->workers.emplace_back([s, i] { s->Work(i); });
  *out = s;
  return RDB_OK;
}

size_t rdb_request_bytes(const rdb_request* req, int device_palettes) {
  if (!req || !req->pixels || req->width < 1 || req->height < 1) return 0;
  return EstimateBytes(*req, device_palettes != 0);
}

int rdb_server_submit(rdb_server* s, const rdb_request* req, uint64_t* ticket) {
  if (!s || !req || !ticket) return rdb::Fail(RDB_E_INVALID, "rdb_server_submit: null argument");
  if (!req->pixels || !req->indices || req->width < 1 || req->height < 1) {
    return rdb::Fail(RDB_E_INVALID, "rdb_server_submit: bad request");
  }
  if (req->engine < RDB_ENGINE_SEQ || req->engine > RDB_ENGINE_JACOBI) {
    return rdb::Fail(RDB_E_INVALID, "rdb_server_submit: unknown engine");
  }
  Req* q = new Req();
  q->r = *req;
  q->bytes = EstimateBytes(*req, s->o.device_palettes != 0);
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) {
    delete q;
    return rdb::Fail(RDB_E_INVALID, "rdb_server_submit: server is stopping");
  }
  if (q->bytes + static_cast<std::size_t>(s->o.workers) * kContextFloor > s->budget) {
    delete q;
    return rdb::Fail(RDB_E_NOMEM, "rdb_server_submit: request larger than the admission budget");
  }
  q->ticket = s->next_ticket++;
  q->t_submit = Clock::now();
  if (!s->any) {
    s->any = true;
    s->first_submit = q->t_submit;
  }
  s->all[q->ticket] = q;
  ++s->pending;
  *ticket = q->ticket;
  if (!s->o.device_palettes) {
    s->incoming.push_back(q);
    s->cv_build.notify_one();
  } else {
    // Straight to admission: the device worker builds the palette.
    q->t_build_start = q->t_built = q->t_submit;
    s->ready.push_back(q);
    s->cv_ready.notify_all();
  }
  return RDB_OK;
}

int rdb_server_wait(rdb_server* s, uint64_t ticket, int timeout_ms, rdb_request_result* out) {
  if (!s) return rdb::Fail(RDB_E_INVALID, "rdb_server_wait: null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(ticket);
  if (it == s->all.end()) return rdb::Fail(RDB_E_INVALID, "rdb_server_wait: unknown ticket");
  Req* q = it->second;
  const auto done = [&] { return q->done; };
  if (timeout_ms < 0) {
    s->cv_done.wait(lk, done);
  } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) {
    return rdb::Fail(RDB_E_TIMEOUT, "rdb_server_wait: not done yet");
  }
  if (out) {
    out->status = q->status;
    out->queue_ms = Ms(q->t_submit, q->t_built);
    out->admit_ms = q->t_start > q->t_built ? Ms(q->t_built, q->t_start) : 0.0;
    out->device_ms = q->device_ms;
    out->total_ms = Ms(q->t_submit, q->t_done);
    out->batch_size = q->batch;
  }
  s->all.erase(it);
  const int st = q->status;
  const std::string err = q->err;
  delete q;
  if (st != RDB_OK) return rdb::Fail(st, "rdb_server_wait: the request failed: " + err);
  return RDB_OK;
}

int rdb_server_stats_get(rdb_server* s, rdb_server_stats* out) {
  if (!s || !out) return rdb::Fail(RDB_E_INVALID, "rdb_server_stats_get: null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(out, 0, sizeof(*out));
  out->completed = static_cast<int64_t>(s->latencies.size());
  out->failed = s->failed;
  out->pixels = s->pixels;
  out->batches = s->batches;
  out->peak_admitted_bytes = s->peak;
  out->host_threads = s->o.host_threads;
  out->workers = s->o.workers;
  if (!s->latencies.empty()) {
    std::vector<double> v(s->latencies.size());
    const auto pct = [&](double p) {
      const std::size_t k = static_cast<std::size_t>(p * static_cast<double>(v.size() - 1) + 0.5);
      return v[std::min(k, v.size() - 1)];
    };
    for (int st = 0; st < RDB_STAGES; ++st) {
      for (std::size_t i = 0; i < v.size(); ++i) v[i] = s->latencies[i][static_cast<std::size_t>(st)];
      std::sort(v.begin(), v.end());
      out->stage_p50_ms[st] = pct(0.50);
      out->stage_p99_ms[st] = pct(0.99);
    }
    out->p50_ms = out->stage_p50_ms[RDB_STAGE_TOTAL];
    out->p99_ms = out->stage_p99_ms[RDB_STAGE_TOTAL];
    out->max_ms = v.back();
    const double span = Ms(s->first_submit, s->last_done);
    out->mpx_per_s = span > 0 ? static_cast<double>(s->pixels) / (span * 1e3) : 0.0;
  }
  return RDB_OK;
}

int rdb_server_stats_reset(rdb_server* s) {
  if (!s) return rdb::Fail(RDB_E_INVALID, "rdb_server_stats_reset: null server");
  std::lock_guard<std::mutex> lk(s->mu);
  s->latencies.clear();
  s->failed = 0;
  s->pixels = 0;
  s->batches = 0;
  s->any = false;
  s->peak = s->admitted;
  return RDB_OK;
}

void rdb_server_destroy(rdb_server* s) {
  if (!s) return;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait(lk, [&] { return s->pending == 0; });
    s->stop = true;
  }
  s->cv_build.notify_all();
  s->cv_ready.notify_all();
  for (std::thread& t : s->builders) t.join();
  for (std::thread& t : s->workers) t.join();
  for (auto& kv : s->all) {
    rdb_octree_free(kv.second->tree);
    delete kv.second;
  }
  delete s;
}

}  // extern "C"
