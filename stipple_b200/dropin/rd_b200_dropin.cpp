// rd_b200_dropin.cpp -- the reference's GPU engine entry points, implemented
// on the B200 engines through the C ABI (include/rdb.h).
//
// rdither links one of two providers of these seven symbols: its CUDA engines
// (src/rd_riemersma_cuda.cu, src/rd_blocks_cuda.cu, src/rd_approx_cuda.cu) or
// the stubs of src/rd_cuda_stub.cpp:50-95.  This file is a third provider with
// the same declarations (include/rd_riemersma.h:214-217, :284-288, :303-310,
// :450-464, :480-481), so a build that compiles it instead of those sources
// gets the B200 engines with no change to any caller (src/rd_cli.cpp:2613,
// 2628, 2674, 2718; src/rd_video.cpp:4414).  It is compiled against the
// reference's own headers and only translates: reference structs in, POD
// descriptors to the C ABI, a std::string out (empty = success, never empty
// without output, src/rd_cuda_stub.cpp:60-74).
//
// State: the reference's walk is stateless per call; its blocks engine keeps
// kGpuStateSlots device states, one mutex each (src/rd_blocks_cuda.cu:990-1002).
// Here every slot is an rdb_context guarded by its own mutex -- slot 0 and 1
// for the blocks engine, a third for the walk and the approximation -- and
// each context keeps the palettes it has seen, keyed by a hash of palette and
// tree, so a video's fixed palette is uploaded once.
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "rd_octree.h"
#include "rd_riemersma.h"
#include "rdb.h"

namespace {

constexpr int kSlots = rd::kGpuStateSlots + 1;  // blocks slots, then walk/approx
constexpr int kWalkSlot = rd::kGpuStateSlots;
constexpr std::size_t kMaxCachedPalettes = 64;

struct Slot {
  std::mutex mu;
  rdb_context* ctx = nullptr;
  std::map<uint64_t, int> palettes;  // palette+tree hash -> palette id
  std::vector<uint64_t> order;       // insertion order, for eviction
};

Slot g_slots[kSlots];

std::string Err(const char* what) {
  return std::string("riemersma-b200: ") + what + ": " + rdb_last_error();
}

void DeviceName(std::string* out) {
  if (!out) return;
  char buf[256];
  if (rdb_device_name(0, buf, sizeof buf) == RDB_OK) *out = buf;
}

// FNV-1a over the bytes that decide the plan.
struct Fnv {
  uint64_t h = 1469598103934665603ull;
  void add(const void* p, std::size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (std::size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
  }
};

uint64_t Hash(const rd::Palette& pal, const rd::ColorTree& tree) {
  Fnv f;
  f.add(&pal.count, sizeof pal.count);
  f.add(&pal.associate_alpha, sizeof pal.associate_alpha);
  f.add(pal.entries, sizeof(rd::PaletteEntry) * static_cast<std::size_t>(pal.count));
  const int tc = tree.color_count();
  f.add(&tc, sizeof tc);
  f.add(tree.colormap(), sizeof(rd::PaletteEntry) * static_cast<std::size_t>(tc));
  const int32_t root = tree.root();
  f.add(&root, sizeof root);
  for (const rd::QNode& q : tree.nodes()) {
    f.add(q.child, sizeof q.child);
    f.add(&q.parent, sizeof q.parent);
    f.add(&q.number_unique, sizeof q.number_unique);
    f.add(&q.color_number, sizeof q.color_number);
  }
  return f.h;
}

// Slot context and the palette id of (palette, tree), created on first use.
// The caller holds the slot's mutex.
std::string Prepare(Slot& s, const rd::Palette& pal, const rd::ColorTree& tree, int* pid) {
  if (!s.ctx && rdb_context_create(0, 0, &s.ctx) != RDB_OK) return Err("no device context");
  const uint64_t h = Hash(pal, tree);
  auto it = s.palettes.find(h);
  if (it != s.palettes.end()) {
    *pid = it->second;
    return {};
  }
  if (pal.count < 1 || pal.count > 256) {
    return "riemersma-b200: palettes of 1..256 colours only (one index byte per pixel)";
  }
  const std::vector<rd::QNode>& nodes = tree.nodes();
  const std::size_t nn = nodes.size();
  std::vector<double> colors(4 * static_cast<std::size_t>(pal.count));
  std::vector<double> search(4 * static_cast<std::size_t>(pal.count));
  for (int i = 0; i < pal.count; ++i) {
    const rd::PaletteEntry& e = pal.entries[i];
    colors[4 * i + 0] = e.r;
    colors[4 * i + 1] = e.g;
    colors[4 * i + 2] = e.b;
    colors[4 * i + 3] = e.a;
    const rd::PaletteEntry& c = i < tree.color_count() ? tree.colormap()[i] : e;
    search[4 * i + 0] = c.r;
    search[4 * i + 1] = c.g;
    search[4 * i + 2] = c.b;
    search[4 * i + 3] = c.a;
  }
  std::vector<int32_t> child(16 * nn), parent(nn);
  std::vector<uint32_t> cn(nn);
  std::vector<uint64_t> nu(nn);
  for (std::size_t i = 0; i < nn; ++i) {
    std::memcpy(&child[16 * i], nodes[i].child, sizeof nodes[i].child);
    parent[i] = nodes[i].parent;
    cn[i] = nodes[i].color_number;
    nu[i] = nodes[i].number_unique;
  }
  rdb_palette_desc d{};
  d.count = pal.count;
  d.associate_alpha = pal.associate_alpha ? 1 : 0;
  d.colors = colors.data();
  d.search_colors = search.data();
  d.node_count = static_cast<int>(nn);
  d.root = tree.root();
  d.child = child.data();
  d.parent = parent.data();
  d.color_number = cn.data();
  d.number_unique = nu.data();
  if (s.order.size() >= kMaxCachedPalettes) {
    const uint64_t old = s.order.front();
    s.order.erase(s.order.begin());
    rdb_palette_destroy(s.ctx, s.palettes[old]);
    s.palettes.erase(old);
  }
  if (rdb_palette_create(s.ctx, &d, pid) != RDB_OK) return Err("palette");
  s.palettes[h] = *pid;
  s.order.push_back(h);
  return {};
}

// `frames` RgbaF frames in place through one host-buffer call.
std::string DitherFrames(Slot& s, int engine, int pid, std::size_t width, std::size_t height,
                         rd::RgbaF* pixels, int frames, const rdb_options& o) {
  if (width == 0 || height == 0) return "riemersma-b200: empty image";
  if (!pixels) return "riemersma-b200: no pixels";
  if (frames < 1) return "riemersma-b200: frames must be >= 1";
  if (width > 0x7FFFFFFF || height > 0x7FFFFFFF) return "riemersma-b200: image too large";
  const std::size_t n = width * height;
  std::vector<uint8_t> idx(n * static_cast<std::size_t>(frames));
  std::vector<rdb_host_job> jobs(static_cast<std::size_t>(frames));
  for (int f = 0; f < frames; ++f) {
    rdb_host_job& j = jobs[static_cast<std::size_t>(f)];
    float* frame = reinterpret_cast<float*>(pixels + static_cast<std::size_t>(f) * n);
    j.pixels = frame;
    j.row_stride = 0;
    j.width = static_cast<int>(width);
    j.height = static_cast<int>(height);
    j.layout = RDB_RGBAF32;
    j.palette_id = pid;
    j.indices = idx.data() + static_cast<std::size_t>(f) * n;
    j.rgba_out = frame;  // in place, as the reference works
  }
  if (rdb_dither_host(s.ctx, engine, jobs.data(), frames, &o) != RDB_OK) return Err("dither");
  return {};
}

}  // namespace

namespace rd {

bool CudaAvailable() {
  int n = 0;
  return rdb_device_count(&n) == RDB_OK && n > 0;
}

int CudaMaxFrames(std::size_t width, std::size_t height, std::size_t vram_budget) {
  return rdb_max_frames(0, RDB_ENGINE_SEQ, width, height, vram_budget);
}

void* CudaAllocPinned(std::size_t bytes) { return rdb_alloc_pinned(bytes); }

void CudaFreePinned(void* p) { rdb_free_pinned(p); }

std::vector<double> ApproxInverseFilter(int taps, double diffusion) {
  if (taps < 1 || taps > 4096) return {};
  std::vector<double> g(static_cast<std::size_t>(taps) + 1);
  if (rdb_inverse_filter(taps, diffusion, g.data()) != RDB_OK) return {};
  return g;
}

std::string RiemersmaWalkCuda(const Palette& palette, const DitherParams& params,
                              const ColorTree& tree, std::size_t width, std::size_t height,
                              RgbaF* pixels, int frames, std::string* device_name) {
  Slot& s = g_slots[kWalkSlot];
  std::lock_guard<std::mutex> lock(s.mu);
  int pid = 0;
  std::string err = Prepare(s, palette, tree, &pid);
  if (!err.empty()) return err;
  rdb_options o;
  rdb_options_default(&o);
  o.diffusion = params.diffusion;
  o.use_cache = params.use_cache ? 1 : 0;
  err = DitherFrames(s, RDB_ENGINE_SEQ, pid, width, height, pixels, frames, o);
  if (err.empty()) DeviceName(device_name);
  return err;
}

std::string RiemersmaBlocksCuda(const Palette& palette, const DitherParams& params,
                                const ColorTree& tree, std::size_t width, std::size_t height,
                                RgbaF* batch, const BlockOptions& options,
                                std::string* device_name, std::uint16_t* out_u16,
                                int state_slot, const std::uint16_t* in_u16) {
  // The reference's refusals (src/rd_blocks_cuda.cu:1014-1041).
  if (palette.count > 256) return "riemersma-b200: the block engine takes at most 256 colours";
  if (options.block < 16) return "riemersma-b200: block must be >= 16";
  if (state_slot < 0 || state_slot >= kGpuStateSlots) return "riemersma-b200: bad state slot";
  // The fused forms are selected as the reference selects them
  // (src/rd_blocks_cuda.cu:1063-1071): a flag AND its buffer.
  const bool fused_out = options.emit_u16 && out_u16 != nullptr;
  const bool fused_in = options.upload_u16 && in_u16 != nullptr;
  Slot& s = g_slots[state_slot];
  std::lock_guard<std::mutex> lock(s.mu);
  int pid = 0;
  std::string err = Prepare(s, palette, tree, &pid);
  if (!err.empty()) return err;
  rdb_options o;
  rdb_options_default(&o);
  o.diffusion = params.diffusion;
  o.block = options.block;
  if (!fused_out && !fused_in) {
    err = DitherFrames(s, RDB_ENGINE_BLOCKS, pid, width, height, batch, options.frames, o);
    if (err.empty()) DeviceName(device_name);
    return err;
  }
  if (width == 0 || height == 0) return "riemersma-b200: empty image";
  if (width > 0x7FFFFFFF || height > 0x7FFFFFFF) return "riemersma-b200: image too large";
  if (options.frames < 1) return "riemersma-b200: frames must be >= 1";
  rdb_frames f{};
  f.width = static_cast<int>(width);
  f.height = static_cast<int>(height);
  f.frames = options.frames;
  f.palette_id = pid;
  if (fused_in) {
    // `in_u16` holds the decoder's bytes: uint16 samples, or planar 8-bit
    // YCbCr (the pointer type is the reference's, not the data's).  The
    // prepass variant converts the same planes through a uint16 RGB frame,
    // which is the same widening.
    switch (options.in_mode) {
      case BlockOptions::InMode::Interleaved16:
        f.in_format = options.in_channels == 3 ? RDB_RGB16 : RDB_RGBA16;
        break;
      case BlockOptions::InMode::PlanarYuv444:
      case BlockOptions::InMode::PlanarYuv444Prepass:
        f.in_format = RDB_YUV444P8;
        break;
      case BlockOptions::InMode::PlanarYuv420:
        f.in_format = RDB_YUV420P8;
        break;
      default:
        return "riemersma-b200: unknown input mode";
    }
    f.in = in_u16;
  } else {
    if (!batch) return "riemersma-b200: no pixels";
    f.in = batch;
    f.in_format = RDB_RGBAF32;
  }
  if (fused_out) {
    f.out = out_u16;
    f.out_format = options.emit_yuv444 ? RDB_YUV444P8 : RDB_RGBA16;
  } else {
    if (!batch) return "riemersma-b200: no output buffer";
    f.out = batch;
    f.out_format = RDB_RGBAF32;
  }
  if (rdb_dither_frames_host(s.ctx, &f, &o) != RDB_OK) return Err("dither");
  DeviceName(device_name);
  return {};
}

std::string RiemersmaApproxCuda(const Palette& palette, const DitherParams& params,
                                const ColorTree& tree, std::size_t width, std::size_t height,
                                RgbaF* pixels, const ApproxOptions& options,
                                std::string* device_name) {
  // The reference's refusals (src/rd_approx_cuda.cu:247-255).
  if (palette.count > 256) return "riemersma-b200: the approximation takes at most 256 colours";
  if (options.taps < 1 || options.taps > 4096) return "riemersma-b200: taps must be 1..4096";
  if (!options.use_tree) {
    return "riemersma-b200: the approximation implements the octree lookup only (use_tree)";
  }
  Slot& s = g_slots[kWalkSlot];
  std::lock_guard<std::mutex> lock(s.mu);
  int pid = 0;
  std::string err = Prepare(s, palette, tree, &pid);
  if (!err.empty()) return err;
  rdb_options o;
  rdb_options_default(&o);
  o.diffusion = params.diffusion;
  // The block-sweep form (rdb_options.jacobi_form 0): `iterations` caps the
  // sweeps; taps and fp64 shape only the point-iteration form.
  o.jacobi_iters = options.iterations;
  o.jacobi_taps = options.taps;
  o.jacobi_fp64 = options.fp64 ? 1 : 0;
  err = DitherFrames(s, RDB_ENGINE_JACOBI, pid, width, height, pixels, 1, o);
  if (err.empty()) DeviceName(device_name);
  return err;
}

}  // namespace rd
