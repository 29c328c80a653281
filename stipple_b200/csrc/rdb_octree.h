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

// 128 bytes on a 64-byte boundary: the error and the child table share the
// first cache line, so a level of the classification descent (child lookup,
// error update) touches one line; counts and totals (leaves only) the second.
struct alignas(64) OctNode {
  double qerr;
  int32_t child[16];
  int32_t parent;
  uint32_t id;
  uint32_t level;
  uint32_t color_number;
  uint64_t number_unique;
  double total[4];
};
static_assert(sizeof(OctNode) == 128, "OctNode is two cache lines");

struct PaletteColor {
  double r, g, b, a;
};

// Input pixel layouts the builder reads.
enum class PixelLayout { kRgb8 = 3, kRgba8 = 4, kRgbaF32 = 16 };

// What the device classification of the rows after the first phase returns
// (rdb_octree_dev.cu): per node visited, its path key (NodeKey) and final
// quantization error; per leaf reached, its pixel count and colour totals; and
// the sum of the visited nodes' running errors, which the root accumulates.
struct OctreeRows {
  std::vector<uint64_t> keys;       // ascending
  std::vector<double> qerr;
  std::vector<uint64_t> leaf_keys;  // ascending
  std::vector<uint64_t> leaf_count;
  std::vector<double> leaf_total;   // 4 per leaf
  double root_gain = 0.0;
};

// A node's path from the root as a key: level in bits 32..35, the child ids
// of levels 1..level packed most significant first (3 or 4 bits each).
inline uint64_t NodeKey(int level, uint32_t path) {
  return (static_cast<uint64_t>(level) << 32) | path;
}

class Octree {
 public:
  // Builds, reduces to at most `max_colors` and defines the colormap exactly as
  // ColorTree::Build does.  Pixels are row-major; 8-bit samples are widened to
  // the Q16 range as v * 257.
  void Build(const void* pixels, PixelLayout layout, std::size_t width, std::size_t height,
             std::size_t row_stride_bytes, int max_colors, bool associate_alpha, bool grayscale);

  // The same build in three steps, so that the rows after the first phase can
  // be classified elsewhere (rdb_octree_dev.cu):
  //   Begin    the set-up and the first classification loop (full depth,
  //            src/rd_octree.cpp:364-376) over rows fetched by `row_at`;
  //            returns the first row of the second loop (height when the first
  //            loop consumed the image);
  //   Absorb   the second loop's result for rows [that row, height), limited
  //            to depth() levels: creates the nodes it reached, sets their
  //            errors, counts and totals; false when the result cannot stand in
  //            for the sequential loop (see rdb_octree_dev.cu), in which case
  //            the tree is unchanged;
  //   ClassifyRows  the second loop on the host instead;
  //   Finish   the reduction and the colormap (:387-409).
  template <class RowAt>
  std::size_t Begin(RowAt row_at, std::size_t width, std::size_t height, int max_colors,
                    bool associate_alpha, bool grayscale);
  bool Absorb(const OctreeRows& rows);
  template <class RowAt>
  void ClassifyRows(RowAt row_at, std::size_t width, std::size_t y0, std::size_t height);
  void Finish();
  // The live nodes by key and their errors, counts and totals, for the device
  // classification to continue from (levels 1..depth()).
  void LiveKeys(std::vector<uint64_t>* keys, std::vector<int32_t>* index) const;
  std::size_t live() const { return live_; }
  static constexpr std::size_t kMaxNodes = 266817;  // quantize.c MaxQNodes (rd_octree.h:39)

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
  template <bool kAssoc>
  void ClassifyAs(const float* rgba, std::size_t width, int level_limit, int colors_level);
  void Merge(int32_t node);
  void PruneAtDepth(int32_t node);
  void PruneBelowDepth(int32_t node);
  void ReducePass(int32_t node);
  std::size_t FlattenErrors(int32_t node, std::size_t offset, double* out) const;
  void Colormap(int32_t node);

  void Setup(int max_colors, bool associate_alpha, bool grayscale);
  void KeysBelow(int32_t node, uint32_t path, std::vector<uint64_t>* keys,
                 std::vector<int32_t>* index) const;

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

template <class RowAt>
std::size_t Octree::Begin(RowAt row_at, std::size_t width, std::size_t height, int max_colors,
                          bool associate_alpha, bool grayscale) {
  Setup(max_colors, associate_alpha, grayscale);
  // rd_octree.cpp:364-376: the first loop at full depth, until the colours
  // first exceed the target (then nodes below the depth are folded up).
  for (std::size_t y = 0; y < height; ++y) {
    if (live_ > kMaxNodes) {
      PruneAtDepth(0);
      --depth_;
    }
    Classify(row_at(y), width, 8, 8);
    if (colors_ > max_colors_) {
      PruneBelowDepth(0);
      return y + 1;
    }
  }
  return height;
}

template <class RowAt>
void Octree::ClassifyRows(RowAt row_at, std::size_t width, std::size_t y0, std::size_t height) {
  // rd_octree.cpp:377-385: the second loop, at the (possibly lowered) depth.
  for (std::size_t y = y0; y < height; ++y) {
    if (live_ > kMaxNodes) {
      PruneAtDepth(0);
      --depth_;
    }
    Classify(row_at(y), width, depth_, depth_);
  }
}

}  // namespace rdb
