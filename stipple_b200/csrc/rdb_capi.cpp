// rdb_capi.cpp -- the extern "C" surface declared in include/rdb.h.
#include <cuda_runtime.h>

#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/rdb.h"
#include "rdb_numeric.h"
#include "rdb_octree.h"
#include "rdb_runtime.h"
#include "rdb_uniform.h"

struct rdb_octree {
  rdb::Octree tree;
};

namespace {

int Guard(const char* what) {
  return rdb::Fail(RDB_E_INVALID, std::string(what) + ": null argument");
}

std::size_t LayoutBytes(int layout) {
  return layout == RDB_RGBAF32 ? 16u : static_cast<std::size_t>(layout);
}

bool LayoutOk(int layout) {
  return layout == RDB_RGB8 || layout == RDB_RGBA8 || layout == RDB_RGBAF32;
}

}  // namespace

extern "C" {

const char* rdb_last_error(void) { return rdb::LastError(); }

int rdb_device_count(int* count) {
  if (!count) return Guard("rdb_device_count");
  *count = 0;
  const cudaError_t e = cudaGetDeviceCount(count);
  if (e != cudaSuccess) {
    *count = 0;
    return rdb::CudaFail(e, "cudaGetDeviceCount");
  }
  return RDB_OK;
}

int rdb_device_name(int device, char* buf, size_t len) {
  if (!buf || len == 0) return Guard("rdb_device_name");
  cudaDeviceProp prop{};
  const cudaError_t e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) return rdb::CudaFail(e, "cudaGetDeviceProperties");
  const std::string s = std::string(prop.name) + " (sm_" + std::to_string(prop.major) +
                        std::to_string(prop.minor) + ")";
  std::strncpy(buf, s.c_str(), len - 1);
  buf[len - 1] = '\0';
  return RDB_OK;
}

void* rdb_alloc_pinned(size_t bytes) {
  void* p = nullptr;
  if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) return nullptr;
  return p;
}

void rdb_free_pinned(void* p) {
  if (p) cudaFreeHost(p);
}

int rdb_max_frames(int device, int engine, size_t width, size_t height, size_t vram_budget) {
  if (width == 0 || height == 0) return 0;
  if (cudaSetDevice(device) != cudaSuccess) return 0;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return 0;
  if (vram_budget != 0 && vram_budget < free_b) free_b = vram_budget;
  const size_t px = width * height;
  // Fixed per call: the visit order (4 B per position), the palette plan and
  // uniform-key table, the status and work words.
  const size_t fixed = 4 * px + (size_t{1} << 20);
  // Per frame: RgbaF staging in and out (16 + 16 B), the index map (1 B), and
  // the engine's scratch: the segmented walk's gathered samples, chosen
  // indices, memo tables and queues (~60 B) plus its 3 MB of key maps; the
  // block and Jacobi engines' curve-ordered copies (~20 B).
  size_t per_px = 33, per_frame_fixed = 0;
  if (engine == RDB_ENGINE_SEQ) {
    per_px += 60;
    per_frame_fixed = size_t{3} << 20;
  } else {
    per_px += 20;
  }
  const size_t per_frame = per_px * px + per_frame_fixed;
  if (free_b < fixed + per_frame) return 0;
  size_t frames = (free_b - fixed) / per_frame;
  if (frames > 4096) frames = 4096;
  return static_cast<int>(frames);
}

int rdb_octree_build(const void* pixels, int layout, size_t width, size_t height,
                     size_t row_stride, int max_colors, int associate_alpha, int grayscale,
                     rdb_octree** out) {
  if (!pixels || !out) return Guard("rdb_octree_build");
  if (!LayoutOk(layout)) return rdb::Fail(RDB_E_INVALID, "unknown pixel layout");
  if (width == 0 || height == 0) return rdb::Fail(RDB_E_INVALID, "empty image");
  rdb_octree* t = new (std::nothrow) rdb_octree();
  if (!t) return rdb::Fail(RDB_E_NOMEM, "octree allocation");
  const std::size_t stride = row_stride ? row_stride : width * LayoutBytes(layout);
  t->tree.Build(pixels, static_cast<rdb::PixelLayout>(layout), width, height, stride, max_colors,
                associate_alpha != 0, grayscale != 0);
  *out = t;
  return RDB_OK;
}

int rdb_octree_build_device(rdb_context* ctx, const void* pixels, int layout, size_t width,
                            size_t height, size_t row_stride, int max_colors, int associate_alpha,
                            int grayscale, void* stream, rdb_octree** out, int* device_rows) {
  if (!ctx || !pixels || !out) return Guard("rdb_octree_build_device");
  *out = nullptr;
  if (!LayoutOk(layout)) return rdb::Fail(RDB_E_INVALID, "unknown pixel layout");
  if (width == 0 || height == 0) return rdb::Fail(RDB_E_INVALID, "empty image");
  if (width * height >= (std::size_t{1} << 31) / 8) {
    return rdb::Fail(RDB_E_UNSUPPORTED, "rdb_octree_build_device takes images below 2^28 pixels");
  }
  rdb_octree* t = new (std::nothrow) rdb_octree();
  if (!t) return rdb::Fail(RDB_E_NOMEM, "octree allocation");
  const std::size_t stride = row_stride ? row_stride : width * LayoutBytes(layout);
  int rows = 0;
  const int rc = ctx->impl.BuildOctree(pixels, layout, static_cast<int>(width), static_cast<int>(height),
                                       stride, max_colors, associate_alpha != 0, grayscale != 0,
                                       static_cast<cudaStream_t>(stream), &t->tree, &rows);
  if (rc != RDB_OK) {
    delete t;
    return rc;
  }
  if (device_rows) *device_rows = rows;
  *out = t;
  return RDB_OK;
}

int rdb_octree_color_count(const rdb_octree* t) { return t ? t->tree.color_count() : 0; }
int rdb_octree_node_count(const rdb_octree* t) {
  return t ? static_cast<int>(t->tree.nodes().size()) : 0;
}
int rdb_octree_depth(const rdb_octree* t) { return t ? t->tree.depth() : 0; }

void rdb_octree_colormap(const rdb_octree* t, double* out) {
  if (!t || !out) return;
  const auto& cm = t->tree.colormap();
  for (std::size_t i = 0; i < cm.size(); ++i) {
    out[4 * i + 0] = cm[i].r;
    out[4 * i + 1] = cm[i].g;
    out[4 * i + 2] = cm[i].b;
    out[4 * i + 3] = cm[i].a;
  }
}

void rdb_octree_nodes(const rdb_octree* t, int32_t* child, int32_t* parent,
                      uint32_t* color_number, uint64_t* number_unique) {
  if (!t) return;
  const auto& nodes = t->tree.nodes();
  for (std::size_t i = 0; i < nodes.size(); ++i) {
    if (child) std::memcpy(child + 16 * i, nodes[i].child, sizeof(nodes[i].child));
    if (parent) parent[i] = nodes[i].parent;
    if (color_number) color_number[i] = nodes[i].color_number;
    if (number_unique) number_unique[i] = nodes[i].number_unique;
  }
}

void rdb_octree_free(rdb_octree* t) { delete t; }

int rdb_palette_write_text(const double* colors, int count, const char* path) {
  if (!colors || !path) return Guard("rdb_palette_write_text");
  return rdb::WritePaletteText(colors, count, path);
}

int rdb_palette_read_text(const char* path, int expect_colors, rdb_octree** out,
                          int* associate_alpha) {
  if (!path || !out) return Guard("rdb_palette_read_text");
  *out = nullptr;
  std::vector<float> strip;
  int count = 0;
  bool assoc = false, gray = false;
  if (int rc = rdb::ReadPaletteText(path, expect_colors, &strip, &count, &assoc, &gray)) return rc;
  rdb_octree* t = new (std::nothrow) rdb_octree();
  if (!t) return rdb::Fail(RDB_E_NOMEM, "octree allocation");
  t->tree.Build(strip.data(), rdb::PixelLayout::kRgbaF32, static_cast<std::size_t>(count), 1,
                static_cast<std::size_t>(count) * 16, count, false, gray);
  if (t->tree.color_count() != count) {
    const int kept = t->tree.color_count();
    delete t;
    return rdb::Fail(RDB_E_INVALID, std::string(path) + ": the tree reduced " +
                                        std::to_string(count) + " colours to " +
                                        std::to_string(kept) +
                                        "; the palette holds duplicate or unreachable entries");
  }
  if (associate_alpha) *associate_alpha = assoc ? 1 : 0;
  *out = t;
  return RDB_OK;
}

int rdb_palette_write_png(const double* colors, int count, const char* path) {
  if (!colors || !path) return Guard("rdb_palette_write_png");
  return rdb::WritePalettePng(colors, count, path);
}

int rdb_palette_read_png(const char* path, int expect_colors, rdb_octree** out) {
  if (!path || !out) return Guard("rdb_palette_read_png");
  *out = nullptr;
  std::vector<float> swatch;
  std::size_t w = 0, h = 0;
  int count = 0;
  bool gray = false;
  if (int rc = rdb::ReadPalettePng(path, expect_colors, &swatch, &w, &h, &count, &gray)) return rc;
  rdb_octree* t = new (std::nothrow) rdb_octree();
  if (!t) return rdb::Fail(RDB_E_NOMEM, "octree allocation");
  t->tree.Build(swatch.data(), rdb::PixelLayout::kRgbaF32, w, h, w * 16, count, false, gray);
  *out = t;
  return RDB_OK;
}

int rdb_is_grayscale(const void* pixels, int layout, size_t width, size_t height,
                     size_t row_stride) {
  if (!pixels || !LayoutOk(layout)) return 0;
  const std::size_t stride = row_stride ? row_stride : width * LayoutBytes(layout);
  for (std::size_t y = 0; y < height; ++y) {
    const unsigned char* row = static_cast<const unsigned char*>(pixels) + y * stride;
    for (std::size_t x = 0; x < width; ++x) {
      if (layout == RDB_RGBAF32) {
        const float* p = reinterpret_cast<const float*>(row) + 4 * x;
        if (!(p[0] == p[1] && p[1] == p[2])) return 0;
      } else {
        const unsigned char* p = row + static_cast<std::size_t>(layout) * x;
        if (!(p[0] == p[1] && p[1] == p[2])) return 0;
      }
    }
  }
  return 1;
}

int rdb_context_create(int device, size_t memory_budget, rdb_context** out) {
  if (!out) return Guard("rdb_context_create");
  *out = nullptr;
  rdb_context* c = new (std::nothrow) rdb_context();
  if (!c) return rdb::Fail(RDB_E_NOMEM, "context allocation");
  const int rc = c->impl.Init(device, memory_budget);
  if (rc != RDB_OK) {
    delete c;
    return rc;
  }
  *out = c;
  return RDB_OK;
}

void rdb_context_destroy(rdb_context* ctx) { delete ctx; }

size_t rdb_context_bytes(const rdb_context* ctx) { return ctx ? ctx->impl.bytes() : 0; }

int rdb_context_last_sweeps(const rdb_context* ctx, int* converged) {
  if (!ctx) return 0;
  if (converged) *converged = ctx->impl.last_sweeps_converged() ? 1 : 0;
  return ctx->impl.last_sweeps();
}

int rdb_context_last_passes(const rdb_context* ctx) {
  return ctx ? const_cast<rdb_context*>(ctx)->impl.last_passes() : 0;
}

int rdb_context_profile(rdb_context* ctx, int enable) {
  if (!ctx) return Guard("rdb_context_profile");
  return ctx->impl.Profile(enable != 0);
}

int rdb_context_dump_indices(rdb_context* ctx, const char* prefix) {
  if (!ctx) return Guard("rdb_context_dump_indices");
  ctx->impl.DumpIndices(prefix ? prefix : "");
  return RDB_OK;
}

int rdb_context_stats(const rdb_context* ctx, rdb_kernel_stats* out) {
  if (!ctx || !out) return Guard("rdb_context_stats");
  *out = ctx->impl.stats();
  return RDB_OK;
}

int rdb_palette_create(rdb_context* ctx, const rdb_palette_desc* d, int* palette_id) {
  if (!ctx || !d || !palette_id || !d->colors || !d->child || !d->color_number ||
      !d->number_unique) {
    return Guard("rdb_palette_create");
  }
  rdb::PlanInput in;
  in.count = d->count;
  in.assoc = d->associate_alpha != 0;
  in.colors = d->colors;
  in.search_colors = d->search_colors;
  in.node_count = d->node_count;
  in.root = d->root;
  in.child = d->child;
  in.parent = d->parent;
  in.color_number = d->color_number;
  in.number_unique = d->number_unique;
  return ctx->impl.CreatePalette(in, palette_id);
}

int rdb_plan_build(const rdb_palette_desc* d, void* out, size_t cap, size_t* size) {
  if (!d || !size || !d->colors || !d->child || !d->color_number || !d->number_unique) {
    return Guard("rdb_plan_build");
  }
  rdb::PlanInput in;
  in.count = d->count;
  in.assoc = d->associate_alpha != 0;
  in.colors = d->colors;
  in.search_colors = d->search_colors;
  in.node_count = d->node_count;
  in.root = d->root;
  in.child = d->child;
  in.parent = d->parent;
  in.color_number = d->color_number;
  in.number_unique = d->number_unique;
  std::vector<uint8_t> blob;
  const std::string err = rdb::BuildPlan(in, &blob);
  if (!err.empty()) return rdb::Fail(RDB_E_UNSUPPORTED, err);
  *size = blob.size();
  if (out) std::memcpy(out, blob.data(), blob.size() < cap ? blob.size() : cap);
  return RDB_OK;
}

int rdb_palette_from_octree(rdb_context* ctx, const rdb_octree* t, int* palette_id) {
  if (!ctx || !t || !palette_id) return Guard("rdb_palette_from_octree");
  return ctx->impl.CreatePaletteFromTree(t->tree, palette_id);
}

int rdb_palette_destroy(rdb_context* ctx, int palette_id) {
  if (!ctx) return Guard("rdb_palette_destroy");
  return ctx->impl.DestroyPalette(palette_id);
}

int rdb_palette_uniform(rdb_context* ctx, int palette_id, uint8_t* out, size_t cap) {
  if (!ctx || !out) return Guard("rdb_palette_uniform");
  const rdb::DevPlan* p = ctx->impl.Plan(palette_id);
  if (!p) return rdb::Fail(RDB_E_INVALID, "unknown palette id");
  const size_t keys = p->assoc ? rdb::kUniformKeysAlpha : rdb::kUniformKeys;
  if (cap < keys) {
    return rdb::Fail(RDB_E_INVALID, p->assoc ? "rdb_palette_uniform: buffer shorter than 2^24 bytes"
                                             : "rdb_palette_uniform: buffer shorter than 2^18 bytes");
  }
  cudaSetDevice(ctx->impl.device());
  cudaStream_t s = ctx->impl.stream();
  const uint8_t* dev = nullptr;
  if (int rc = ctx->impl.Uniform(palette_id, s, &dev)) return rc;
  cudaError_t e = cudaSuccess;
  if (p->assoc) {
    // Classify every key the walks have not met yet.
    e = rdb::LaunchUniformTableAlpha(p->dev, const_cast<uint8_t*>(dev), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dev, keys, cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? RDB_OK : rdb::CudaFail(e, "rdb_palette_uniform");
}

void rdb_options_default(rdb_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->diffusion = 1.0;
  o->use_cache = 1;
  o->block = 512;
  o->jacobi_iters = 20;
  o->jacobi_taps = 96;
  o->jacobi_fp64 = 0;
  o->cache_bits = 0;
  o->seq_mode = 0;
  o->seg_len = 0;
  o->warm_len = 0;
  o->max_passes = 0;
  o->loop_mode = 0;
}

int rdb_dither(rdb_context* ctx, int engine, const rdb_job* jobs, int n_jobs,
               const rdb_options* opts, void* stream) {
  if (!ctx) return Guard("rdb_dither");
  rdb_options o;
  if (opts) o = *opts; else rdb_options_default(&o);
  return ctx->impl.Dither(engine, jobs, n_jobs, o, static_cast<cudaStream_t>(stream));
}

int rdb_synchronize(rdb_context* ctx, void* stream) {
  if (!ctx) return Guard("rdb_synchronize");
  return ctx->impl.Synchronize(static_cast<cudaStream_t>(stream));
}

int rdb_dither_host(rdb_context* ctx, int engine, const rdb_host_job* jobs, int n_jobs,
                    const rdb_options* opts) {
  if (!ctx) return Guard("rdb_dither_host");
  rdb_options o;
  if (opts) o = *opts; else rdb_options_default(&o);
  return ctx->impl.DitherHost(engine, jobs, n_jobs, o);
}

size_t rdb_frame_bytes(int format, int width, int height) {
  return rdb::FrameBytes(format, width, height);
}

int rdb_dither_frames(rdb_context* ctx, const rdb_frames* f, const rdb_options* opts,
                      void* stream) {
  if (!ctx || !f) return Guard("rdb_dither_frames");
  rdb_options o;
  if (opts) o = *opts; else rdb_options_default(&o);
  return ctx->impl.Frames(*f, o, static_cast<cudaStream_t>(stream));
}

int rdb_dither_frames_host(rdb_context* ctx, const rdb_frames* f, const rdb_options* opts) {
  if (!ctx || !f) return Guard("rdb_dither_frames_host");
  rdb_options o;
  if (opts) o = *opts; else rdb_options_default(&o);
  return ctx->impl.FramesHost(*f, o);
}

void rdb_error_weights(double out[16]) {
  if (out) rdb::error_weights(out);
}

int rdb_inverse_filter(int taps, double diffusion, double* out) {
  if (!out) return Guard("rdb_inverse_filter");
  if (taps < 1 || taps > 4096) return rdb::Fail(RDB_E_UNSUPPORTED, "taps out of range");
  double w[16];
  rdb::error_weights(w);
  out[0] = 1.0;
  for (int d = 1; d <= taps; ++d) {
    double acc = 0.0;
    const int kmax = d < 16 ? d : 16;
    for (int k = 1; k <= kmax; ++k) acc += (diffusion / 16.0) * w[k - 1] * out[d - k];
    out[d] = acc;
  }
  return RDB_OK;
}

int64_t rdb_block_gap(int width, int height) {
  if (width < 1 || height < 1) return -1;
  int level = 0;
  const int extent = width > height ? width : height;
  while ((1 << level) < extent) ++level;
  if (level == 0) return -1;
  return width == (1 << level) ? static_cast<int64_t>(width - 1) : -1;
}

}  // extern "C"
