// rd_b200_plugin.cpp -- registers the B200 sequential-exact walk with
// rdither's dither registry (include/rd_plugin.h:86-148) as "riemersma-b200".
//
// The registry's contract hands an algorithm the palette and the frames, not
// the colour tree the Riemersma lookup needs (DitherJob, rd_plugin.h:86-103).
// This plugin rebuilds the tree the CLI would build for the first frame
// (ColorTree::Build with the CLI's greyscale rule, src/rd_cli.cpp:2452-2456)
// and uses it only when that tree's colormap reproduces the palette it was
// handed (the CLI's own check, src/rd_cli.cpp:2506-2530); otherwise it reports
// an error rather than dither against a different tree.  Each frame keeps its
// own error queue (frames are independent jobs of one call).
#include <cstring>
#include <string>

#include "rd_octree.h"
#include "rd_plugin.h"
#include "rd_riemersma.h"

namespace {

bool Grey(const rd::RgbaF* px, std::size_t n) {
  for (std::size_t i = 0; i < n; ++i) {
    if (px[i].r != px[i].g || px[i].g != px[i].b) return false;
  }
  return true;
}

bool SameColormap(const rd::ColorTree& tree, const rd::Palette& pal) {
  if (tree.color_count() != pal.count) return false;
  return std::memcmp(tree.colormap(), pal.entries,
                     sizeof(rd::PaletteEntry) * static_cast<std::size_t>(pal.count)) == 0;
}

rd::DitherResult RunB200(rd::DitherJob& job, rd::RgbaF* pixels) {
  rd::DitherResult r;
  if (!job.palette || !pixels || job.width == 0 || job.height == 0) {
    r.error = "riemersma-b200: empty job";
    return r;
  }
  const rd::Palette& pal = *job.palette;
  const std::size_t n = job.width * job.height;
  const bool grey = Grey(pixels, n);
  // The requested colour count is not part of the job; the tree's colour count
  // can fall below it, so try the palette's own count, then the usual sizes.
  static const int kCounts[] = {0, 2, 4, 8, 16, 32, 64, 128, 256};
  rd::ColorTree tree;
  bool found = false;
  for (int c : kCounts) {
    const int want = c == 0 ? pal.count : c;
    if (want < pal.count) continue;
    tree.Build(pixels, job.width, job.height, want, pal.associate_alpha, grey);
    if (SameColormap(tree, pal)) {
      found = true;
      break;
    }
  }
  if (!found) {
    r.error = "riemersma-b200: the palette is not this image's octree colormap";
    return r;
  }
  rd::DitherParams params;
  params.colors = pal.count;
  params.diffusion = job.diffusion;
  params.use_cache = true;
  r.error = rd::RiemersmaWalkCuda(pal, params, tree, job.width, job.height, pixels, job.frames,
                                  nullptr);
  return r;
}

const bool kRegistered = [] {
  return rd::RegisterDither({"riemersma-b200",
                             "Riemersma (Hilbert) error diffusion, bit-exact, on the B200 engines",
                             RunB200});
}();

}  // namespace
