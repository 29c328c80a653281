// rdb_octree.h -- host-side palette builder with ImageMagick 7 octree semantics.
//
// Reference: src/rd_octree.cpp (ColorTree::Build, :219-409) and
// include/rd_octree.h.  The Riemersma lookup searches a SUBTREE of this tree
// (the descent's stopping node's parent), so the tree itself -- not only the
// colormap -- is part of the observable output; both must match the reference
// bit for bit.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

namespace rdb {

struct OctNode {
  int32_t child[16];
  int32_t parent;
  uint32_t id;
  uint32_t level;
  uint32_t color_number;
  uint64_t number_unique;
  double total[4];
  double qerr;
};

struct PaletteColor {
  double r, g, b, a;
};

// Input pixel layouts the builder reads.
enum class PixelLayout { kRgb8 = 3, kRgba8 = 4, kRgbaF32 = 16 };

class Octree {
 public:
  // Builds, reduces to at most `max_colors` and defines the colormap exactly as
  // ColorTree::Build does.  Pixels are row-major; 8-bit samples are widened to
  // the Q16 range as v * 257.
  void Build(const void* pixels, PixelLayout layout, std::size_t width, std::size_t height,
             std::size_t row_stride_bytes, int max_colors, bool associate_alpha, bool grayscale);

  int color_count() const { return static_cast<int>(colormap_.size()); }
  const std::vector<PaletteColor>& colormap() const { return colormap_; }
  const std::vector<OctNode>& nodes() const { return nodes_; }
  int32_t root() const { return 0; }
  bool associate_alpha() const { return assoc_; }
  int depth() const { return depth_; }

 private:
  int32_t Add(uint32_t id, uint32_t level, int32_t parent);
  int Fan() const { return assoc_ ? 16 : 8; }
  void Classify(const float* rgba, std::size_t width, int level_limit, int colors_level);
  void Merge(int32_t node);
  void PruneAtDepth(int32_t node);
  void PruneBelowDepth(int32_t node);
  void ReducePass(int32_t node);
  std::size_t FlattenErrors(int32_t node, std::size_t offset, double* out) const;
  void Colormap(int32_t node);

  std::vector<OctNode> nodes_;
  std::vector<PaletteColor> colormap_;
  bool assoc_ = false;
  int depth_ = 2;
  int max_colors_ = 0;
  int colors_ = 0;
  std::size_t live_ = 0;
  double prune_below_ = 0.0;
  double next_prune_ = 0.0;
};

}  // namespace rdb
