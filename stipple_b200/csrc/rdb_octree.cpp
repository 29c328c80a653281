// rdb_octree.cpp -- ImageMagick 7 octree classification, reduction and colormap.
//
// Reference: src/rd_octree.cpp.  The order of every floating-point operation
// follows the reference (compile with -ffp-contract=off), and so do its
// deliberate quirks: the live-node counter that includes pruned-then-recreated
// nodes, the root-parent self link, the per-level root error accumulation and
// the glibc qsort with a tolerance comparator for the reduction threshold.
#include "rdb_octree.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "rdb_numeric.h"

namespace rdb {
namespace {

// rd_octree.cpp:23-29: returns 0 for values within 1e-12, so the sort is
// deterministic only for this exact comparator and qsort implementation.
int CompareErrors(const void* a, const void* b) {
  const double p = *static_cast<const double*>(a);
  const double q = *static_cast<const double*>(b);
  if (p > q) return 1;
  if (std::fabs(q - p) <= kEpsilon) return 0;
  return -1;
}

struct Sample {
  float v[4];
};

// rd_types.h:179-192 (AssociateAlphaPixel) on a float sample.
inline void Associate(bool assoc, const Sample& s, double out[4]) {
  out[3] = static_cast<double>(s.v[3]);
  if (!assoc || s.v[3] == 65535.0f) {
    out[0] = static_cast<double>(s.v[0]);
    out[1] = static_cast<double>(s.v[1]);
    out[2] = static_cast<double>(s.v[2]);
    return;
  }
  const double alpha = kQuantumScale * static_cast<double>(s.v[3]);
  out[0] = alpha * static_cast<double>(s.v[0]);
  out[1] = alpha * static_cast<double>(s.v[1]);
  out[2] = alpha * static_cast<double>(s.v[2]);
}

}  // namespace

int32_t Octree::Add(uint32_t id, uint32_t level, int32_t parent) {
  OctNode n;
  std::memset(&n, 0, sizeof(n));
  for (int i = 0; i < 16; ++i) n.child[i] = -1;
  n.id = id;
  n.level = level;
  n.parent = parent;
  nodes_.push_back(n);
  return static_cast<int32_t>(nodes_.size() - 1);
}

// rd_octree.cpp:69-93 (PruneChild): fold a node into its parent while the live
// count exceeds the target.  The root's parent is the root itself, and the
// fold then doubles the root's counts, as in the reference.
void Octree::Merge(int32_t node) {
  for (int i = 0; i < Fan(); ++i) {
    const int32_t c = nodes_[node].child[i];
    if (c >= 0) Merge(c);
  }
  if (live_ > static_cast<std::size_t>(max_colors_)) {
    const int32_t parent = nodes_[node].parent;
    if (parent >= 0) {
      OctNode& p = nodes_[parent];
      OctNode& n = nodes_[node];
      p.number_unique += n.number_unique;
      for (int c = 0; c < 4; ++c) p.total[c] += n.total[c];
      p.child[n.id] = -1;
    }
    --live_;
  }
}

// rd_octree.cpp:95-102 (PruneLevel).
void Octree::PruneAtDepth(int32_t node) {
  for (int i = 0; i < Fan(); ++i) {
    const int32_t c = nodes_[node].child[i];
    if (c >= 0) PruneAtDepth(c);
  }
  if (static_cast<int>(nodes_[node].level) == depth_) Merge(node);
}

// rd_octree.cpp:104-111 (PruneToCubeDepth).
void Octree::PruneBelowDepth(int32_t node) {
  for (int i = 0; i < Fan(); ++i) {
    const int32_t c = nodes_[node].child[i];
    if (c >= 0) PruneBelowDepth(c);
  }
  if (static_cast<int>(nodes_[node].level) > depth_) Merge(node);
}

// rd_octree.cpp:113-127 (Reduce).
void Octree::ReducePass(int32_t node) {
  for (int i = 0; i < Fan(); ++i) {
    const int32_t c = nodes_[node].child[i];
    if (c >= 0) ReducePass(c);
  }
  const double e = nodes_[node].qerr;
  if (e <= prune_below_) {
    Merge(node);
  } else {
    if (nodes_[node].number_unique > 0) ++colors_;
    if (e < next_prune_) next_prune_ = e;
  }
}

// rd_octree.cpp:129-140 (QuantizeErrorFlatten).
std::size_t Octree::FlattenErrors(int32_t node, std::size_t offset, double* out) const {
  if (offset >= live_) return 0;
  out[offset] = nodes_[node].qerr;
  std::size_t n = 1;
  for (int i = 0; i < Fan(); ++i) {
    const int32_t c = nodes_[node].child[i];
    if (c >= 0) n += FlattenErrors(c, offset + n, out);
  }
  return n;
}

// rd_octree.cpp:142-176 (DefineImageColormap): colour numbers in post-order.
void Octree::Colormap(int32_t node) {
  for (int i = 0; i < Fan(); ++i) {
    const int32_t c = nodes_[node].child[i];
    if (c >= 0) Colormap(c);
  }
  OctNode& n = nodes_[node];
  if (n.number_unique == 0) return;
  PaletteColor q;
  const double alpha = safe_reciprocal(static_cast<double>(n.number_unique));
  if (!assoc_) {
    q.r = static_cast<float>(alpha * kQuantumRange * n.total[0]);
    q.g = static_cast<float>(alpha * kQuantumRange * n.total[1]);
    q.b = static_cast<float>(alpha * kQuantumRange * n.total[2]);
    q.a = kOpaqueAlpha;
  } else {
    const double opacity = alpha * kQuantumRange * n.total[3];
    q.a = static_cast<float>(opacity);
    if (q.a == kOpaqueAlpha) {
      q.r = static_cast<float>(alpha * kQuantumRange * n.total[0]);
      q.g = static_cast<float>(alpha * kQuantumRange * n.total[1]);
      q.b = static_cast<float>(alpha * kQuantumRange * n.total[2]);
    } else {
      const double gamma = safe_reciprocal(kQuantumScale * q.a);
      q.r = static_cast<float>(alpha * gamma * kQuantumRange * n.total[0]);
      q.g = static_cast<float>(alpha * gamma * kQuantumRange * n.total[1]);
      q.b = static_cast<float>(alpha * gamma * kQuantumRange * n.total[2]);
    }
  }
  n.color_number = static_cast<uint32_t>(colormap_.size());
  colormap_.push_back(q);
}

// rd_octree.cpp:305-362: one row, run-length collapsed, each run descending to
// `level_limit` and counting new nodes at `colors_level` as colours.  The
// alpha channel is a compile-time choice: without it the fourth midpoint and
// the fourth (zero) term of the distance are not computed, which changes no
// sum (a sum of squares plus +0.0 is itself).
void Octree::Classify(const float* rgba, std::size_t width, int level_limit, int colors_level) {
  if (assoc_) {
    ClassifyAs<true>(rgba, width, level_limit, colors_level);
  } else {
    ClassifyAs<false>(rgba, width, level_limit, colors_level);
  }
}

template <bool kAssoc>
void Octree::ClassifyAs(const float* rgba, std::size_t width, int level_limit, int colors_level) {
  const Sample* row = reinterpret_cast<const Sample*>(rgba);
  const double midpoint = kQuantumRange / 2.0;
  // The root's running error, which every visited node's error is added to
  // in visit order: kept in a register for the row (the descent never
  // visits the root itself, so no other read sees it meanwhile) instead of
  // a store and reload through the node array at every level.
  double root = nodes_[0].qerr;
  std::size_t x = 0;
  while (x < width) {
    std::size_t run = 1;
    while (x + run < width && row[x + run].v[0] == row[x].v[0] &&
           row[x + run].v[1] == row[x].v[1] && row[x + run].v[2] == row[x].v[2] &&
           row[x + run].v[3] == row[x].v[3]) {
      ++run;
    }
    double px[4];
    Associate(kAssoc, row[x], px);
    unsigned byte[4];
    for (int c = 0; c < 4; ++c) byte[c] = scale_char(clamp_pixel(px[c]));
    double half = (kQuantumRange + 1.0) / 2.0;
    double mid[4] = {midpoint, midpoint, midpoint, midpoint};
    int32_t node = 0;
    int bit = kMaxTreeDepth - 1;
    const double weight = static_cast<double>(run);
    for (int level = 1; level <= level_limit; ++level, --bit) {
      half *= 0.5;
      unsigned id = ((byte[0] >> bit) & 1u) | (((byte[1] >> bit) & 1u) << 1) |
                    (((byte[2] >> bit) & 1u) << 2);
      if (kAssoc) id |= ((byte[3] >> bit) & 1u) << 3;
      mid[0] += (id & 1u) ? half : -half;
      mid[1] += (id & 2u) ? half : -half;
      mid[2] += (id & 4u) ? half : -half;
      if (kAssoc) mid[3] += (id & 8u) ? half : -half;
      if (nodes_[node].child[id] < 0) {
        const int32_t made = Add(id, static_cast<uint32_t>(level), node);
        nodes_[node].child[id] = made;
        ++live_;
        if (level == colors_level) ++colors_;
      }
      node = nodes_[node].child[id];
      const double e0 = kQuantumScale * (px[0] - mid[0]);
      const double e1 = kQuantumScale * (px[1] - mid[1]);
      const double e2 = kQuantumScale * (px[2] - mid[2]);
      double dist = e0 * e0 + e1 * e1 + e2 * e2;
      if (kAssoc) {
        const double e3 = kQuantumScale * (px[3] - mid[3]);
        dist = dist + e3 * e3;
      }
      if (std::isnan(dist)) dist = 0.0;
      nodes_[node].qerr += weight * std::sqrt(dist);
      root += nodes_[node].qerr;
    }
    OctNode& leaf = nodes_[node];
    leaf.number_unique += run;
    leaf.total[0] += weight * kQuantumScale * static_cast<double>(clamp_pixel(px[0]));
    leaf.total[1] += weight * kQuantumScale * static_cast<double>(clamp_pixel(px[1]));
    leaf.total[2] += weight * kQuantumScale * static_cast<double>(clamp_pixel(px[2]));
    leaf.total[3] += weight * kQuantumScale *
                     static_cast<double>(clamp_pixel(kAssoc ? px[3] : kOpaqueAlpha));
    x += run;
  }
  nodes_[0].qerr = root;
}

void Octree::Setup(int max_colors, bool associate_alpha, bool grayscale) {
  nodes_.clear();
  colormap_.clear();
  assoc_ = associate_alpha;
  max_colors_ = (max_colors <= 0) ? kMaxColormap : max_colors;
  if (max_colors_ > kMaxColormap) max_colors_ = kMaxColormap;
  live_ = 0;
  colors_ = 0;
  prune_below_ = 0.0;
  next_prune_ = 0.0;

  // rd_octree.cpp:255-275: Log4(colours)+2, minus one for the dither, minus one
  // more with alpha above 5, forced to 8 for greyscale, clamped to [2, 8].
  int depth = 1;
  for (std::size_t c = static_cast<std::size_t>(max_colors_); c != 0; ++depth) c >>= 2;
  if (depth > 2) --depth;
  if (assoc_ && depth > 5) --depth;
  if (grayscale) depth = kMaxTreeDepth;
  if (depth > kMaxTreeDepth) depth = kMaxTreeDepth;
  if (depth < 2) depth = 2;
  depth_ = depth;

  Add(0, 0, -1);
  live_ = 1;
  nodes_[0].parent = 0;  // GetQCubeInfo's root->parent = root (rd_octree.cpp:285)
}

void Octree::Finish() {
  // rd_octree.cpp:387-404 (ReduceImageColors).
  if (colors_ > max_colors_) {
    next_prune_ = 0.0;
    if (live_ > 0) {
      const std::size_t n = live_;
      std::vector<double> errors(n, 0.0);
      (void)FlattenErrors(0, 0, errors.data());
      std::qsort(errors.data(), n, sizeof(double), CompareErrors);
      const std::size_t aggressive =
          (110u * (static_cast<std::size_t>(max_colors_) + 1u)) / 100u;
      if (n > aggressive) next_prune_ = errors[n - aggressive];
    }
  }
  while (colors_ > max_colors_) {
    prune_below_ = next_prune_;
    next_prune_ = nodes_[0].qerr - 1.0;
    colors_ = 0;
    ReducePass(0);
  }
  Colormap(0);
}

void Octree::KeysBelow(int32_t node, uint32_t path, std::vector<uint64_t>* keys,
                       std::vector<int32_t>* index) const {
  const int bits = assoc_ ? 4 : 3;
  for (int i = 0; i < Fan(); ++i) {
    const int32_t c = nodes_[node].child[i];
    if (c < 0) continue;
    const uint32_t p = (path << bits) | static_cast<uint32_t>(i);
    keys->push_back(NodeKey(static_cast<int>(nodes_[c].level), p));
    index->push_back(c);
    KeysBelow(c, p, keys, index);
  }
}

void Octree::LiveKeys(std::vector<uint64_t>* keys, std::vector<int32_t>* index) const {
  keys->clear();
  index->clear();
  KeysBelow(0, 0u, keys, index);
}

bool Octree::Absorb(const OctreeRows& r) {
  const int bits = assoc_ ? 4 : 3;
  // The root accumulates every visited node's running error; its exact bits
  // decide nothing as long as it exceeds every other node's error by more than
  // the reduction's one-unit step (it then sorts last, is never merged and
  // never becomes the next threshold), so a sum in another order stands in.
  double max_other = 0.0;
  for (const OctNode& n : nodes_) max_other = std::max(max_other, n.qerr);
  for (double q : r.qerr) max_other = std::max(max_other, q);
  const double root = nodes_[0].qerr + r.root_gain;
  if (!(root > max_other * (1.0 + 1e-9) + 2.0)) return false;
  if (live_ + r.keys.size() > kMaxNodes) return false;  // the loop would have pruned
  std::vector<uint64_t> keys;
  std::vector<int32_t> index;
  LiveKeys(&keys, &index);
  // Existing nodes by key (sorted for lookup).
  std::vector<std::pair<uint64_t, int32_t>> have(keys.size());
  for (std::size_t i = 0; i < keys.size(); ++i) have[i] = {keys[i], index[i]};
  std::sort(have.begin(), have.end());
  const auto find = [&](uint64_t k) -> int32_t {
    auto it = std::lower_bound(have.begin(), have.end(), std::make_pair(k, INT32_MIN));
    return (it != have.end() && it->first == k) ? it->second : -1;
  };
  // Keys ascend by level, so every parent exists before its children.
  std::vector<std::pair<uint64_t, int32_t>> made;
  const auto node_of = [&](uint64_t k) -> int32_t {
    const int32_t n = find(k);
    if (n >= 0) return n;
    auto it = std::lower_bound(made.begin(), made.end(), std::make_pair(k, INT32_MIN));
    return (it != made.end() && it->first == k) ? it->second : -1;
  };
  for (std::size_t i = 0; i < r.keys.size(); ++i) {
    const uint64_t k = r.keys[i];
    const int level = static_cast<int>(k >> 32);
    const uint32_t path = static_cast<uint32_t>(k);
    int32_t node = node_of(k);
    if (node < 0) {
      const int32_t parent = level == 1 ? 0 : node_of(NodeKey(level - 1, path >> bits));
      if (parent < 0) return false;
      const uint32_t id = path & ((1u << bits) - 1u);
      node = Add(id, static_cast<uint32_t>(level), parent);
      nodes_[parent].child[id] = node;
      ++live_;
      if (level == depth_) ++colors_;
      made.insert(std::upper_bound(made.begin(), made.end(), std::make_pair(k, node)), {k, node});
    }
    nodes_[node].qerr = r.qerr[i];
  }
  for (std::size_t i = 0; i < r.leaf_keys.size(); ++i) {
    const int32_t node = node_of(r.leaf_keys[i]);
    if (node < 0) return false;
    nodes_[node].number_unique = r.leaf_count[i];
    for (int c = 0; c < 4; ++c) nodes_[node].total[c] = r.leaf_total[4 * i + c];
  }
  nodes_[0].qerr = root;
  return true;
}

void Octree::Build(const void* pixels, PixelLayout layout, std::size_t width,
                   std::size_t height, std::size_t row_stride_bytes, int max_colors,
                   bool associate_alpha, bool grayscale) {
  // Rows are widened to Q16 floats one at a time.
  std::vector<float> widened(width * 4);
  const auto row_at = [&](std::size_t y) -> const float* {
    const unsigned char* base = static_cast<const unsigned char*>(pixels) + y * row_stride_bytes;
    if (layout == PixelLayout::kRgbaF32) return reinterpret_cast<const float*>(base);
    const int ch = static_cast<int>(layout);
    for (std::size_t x = 0; x < width; ++x) {
      widened[4 * x + 0] = static_cast<float>(base[ch * x + 0]) * 257.0f;
      widened[4 * x + 1] = static_cast<float>(base[ch * x + 1]) * 257.0f;
      widened[4 * x + 2] = static_cast<float>(base[ch * x + 2]) * 257.0f;
      widened[4 * x + 3] = ch == 4 ? static_cast<float>(base[ch * x + 3]) * 257.0f : 65535.0f;
    }
    return widened.data();
  };
  const std::size_t y0 = Begin(row_at, width, height, max_colors, associate_alpha, grayscale);
  ClassifyRows(row_at, width, y0, height);
  Finish();
}

void error_weights(double w[kQueue]) {
  double weight = 1.0;
  for (int i = 0; i < kQueue; ++i) {
    w[i] = safe_reciprocal(weight);
    weight *= std::exp(std::log(1.0 / (1.0 / 16.0)) / (kQueue - 1.0));
  }
}

void scaled_weights(double diffusion, double out[kQueue]) {
  double w[kQueue];
  error_weights(w);
  for (int k = 0; k < kQueue; ++k) out[k] = (1.0 / 16.0) * diffusion * w[k];
}

}  // namespace rdb
