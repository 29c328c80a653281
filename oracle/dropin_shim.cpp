// dropin_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Drives the reference-facing C++ layer (stipple_b200/dropin: the seven engine
// symbols of include/rd_riemersma.h and the "riemersma-b200" registry entry)
// the way rdither's own callers do: the palette and tree come from the
// reference's ColorTree::Build (src/rd_octree.cpp, compiled unmodified from
// the reference tree by oracle/Makefile), the frames are RgbaF in place.
// The tests compare the results with the reference's CPU walks run on the same
// inputs through oracle/_ref/librdref.so.  Nothing here is shipped.
#include <cstring>
#include <string>
#include <vector>

#include "rd_octree.h"
#include "rd_plugin.h"
#include "rd_riemersma.h"

namespace {

void Copy(const std::string& s, char* out, std::size_t len) {
  if (!out || len == 0) return;
  std::strncpy(out, s.c_str(), len - 1);
  out[len - 1] = '\0';
}

}  // namespace

extern "C" {

int dropin_available() { return rd::CudaAvailable() ? 1 : 0; }

int dropin_max_frames(std::size_t w, std::size_t h, std::size_t budget) {
  return rd::CudaMaxFrames(w, h, budget);
}

int dropin_inverse_filter(int taps, double diffusion, double* out) {
  const std::vector<double> g = rd::ApproxInverseFilter(taps, diffusion);
  for (std::size_t i = 0; i < g.size(); ++i) out[i] = g[i];
  return static_cast<int>(g.size());
}

void* dropin_alloc_pinned(std::size_t bytes) { return rd::CudaAllocPinned(bytes); }
void dropin_free_pinned(void* p) { rd::CudaFreePinned(p); }

// engine: 0 RiemersmaWalkCuda, 1 RiemersmaBlocksCuda, 2 RiemersmaApproxCuda,
// 3 the "riemersma-b200" registry entry.  The tree is built from `tree_src`
// (one frame, w x h RgbaF) with the CLI's palette copy; `pixels` holds
// `frames` frames and is dithered in place.  Returns 0, or -1 with `err`.
int dropin_run(int engine, const float* tree_src, std::size_t w, std::size_t h, int colors,
               int assoc, int gray, float* pixels, int frames, double diffusion, int use_cache,
               int block, int iterations, int taps, int slot, char* err, std::size_t errlen,
               char* device, std::size_t devlen) {
  rd::ColorTree tree;
  tree.Build(reinterpret_cast<const rd::RgbaF*>(tree_src), w, h, colors, assoc != 0, gray != 0);
  static rd::Palette pal;  // 2 MiB: not on the stack
  pal = rd::Palette();
  pal.count = tree.color_count();
  pal.associate_alpha = assoc != 0;
  for (int i = 0; i < pal.count; ++i) pal.entries[i] = tree.colormap()[i];
  rd::DitherParams p;
  p.colors = colors;
  p.diffusion = diffusion;
  p.use_cache = use_cache != 0;
  rd::RgbaF* px = reinterpret_cast<rd::RgbaF*>(pixels);
  std::string name, e;
  if (engine == 0) {
    e = rd::RiemersmaWalkCuda(pal, p, tree, w, h, px, frames, &name);
  } else if (engine == 1) {
    rd::BlockOptions o;
    o.block = block;
    o.frames = frames;
    e = rd::RiemersmaBlocksCuda(pal, p, tree, w, h, px, o, &name, nullptr, slot, nullptr);
  } else if (engine == 2) {
    rd::ApproxOptions o;
    o.iterations = iterations;
    o.taps = taps;
    e = rd::RiemersmaApproxCuda(pal, p, tree, w, h, px, o, &name);
  } else {
    const rd::DitherAlgorithm* a = rd::FindDither("riemersma-b200");
    if (!a) {
      e = "riemersma-b200 is not registered";
    } else {
      rd::DitherJob job;
      job.palette = &pal;
      job.width = w;
      job.height = h;
      job.frames = frames;
      job.diffusion = diffusion;
      e = a->run(job, px).error;
    }
  }
  Copy(name, device, devlen);
  if (!e.empty()) {
    Copy(e, err, errlen);
    return -1;
  }
  return 0;
}

// RiemersmaBlocksCuda's fused forms: `in_raw` (the decoder's frames, used
// when upload) read per in_mode / in_channels, `batch` RgbaF (used when not
// upload, and as the output when not emit), `out_raw` rgba64 or planar 4:4:4.
int dropin_blocks_fused(const float* tree_src, std::size_t w, std::size_t h, int colors,
                        int assoc, float* batch, int frames, int block, int upload, int in_mode,
                        int in_channels, const void* in_raw, int emit, int emit_yuv444,
                        void* out_raw, char* err, std::size_t errlen) {
  rd::ColorTree tree;
  tree.Build(reinterpret_cast<const rd::RgbaF*>(tree_src), w, h, colors, assoc != 0, false);
  static rd::Palette pal;
  pal = rd::Palette();
  pal.count = tree.color_count();
  pal.associate_alpha = assoc != 0;
  for (int i = 0; i < pal.count; ++i) pal.entries[i] = tree.colormap()[i];
  rd::DitherParams p;
  p.colors = colors;
  rd::BlockOptions o;
  o.block = block;
  o.frames = frames;
  o.upload_u16 = upload != 0;
  o.in_mode = static_cast<rd::BlockOptions::InMode>(in_mode);
  o.in_channels = in_channels;
  o.emit_u16 = emit != 0;
  o.emit_yuv444 = emit_yuv444 != 0;
  std::string name;
  const std::string e = rd::RiemersmaBlocksCuda(
      pal, p, tree, w, h, reinterpret_cast<rd::RgbaF*>(batch), o, &name,
      static_cast<std::uint16_t*>(out_raw), 0, static_cast<const std::uint16_t*>(in_raw));
  if (!e.empty()) {
    Copy(e, err, errlen);
    return -1;
  }
  return 0;
}

}  // extern "C"
