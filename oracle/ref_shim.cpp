// ref_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C-ABI shim over the reference's own CPU code (rdither's rd_octree.cpp and
// rd_riemersma_cpu.cpp, compiled unmodified from the reference tree by
// oracle/Makefile into oracle/_ref/librdref.so).  It lets the tests run the
// reference itself beside the C restatement in oracle.c.  Nothing here is
// shipped; the library it builds is git-ignored.
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "rd_octree.h"
#include "rd_riemersma.h"

namespace {

struct RefTree {
  rd::ColorTree tree;
  std::unique_ptr<rd::Palette> palette{new rd::Palette()};
};

}  // namespace

extern "C" {

// ColorTree::Build (src/rd_octree.cpp:219) followed by the palette copy the CLI
// performs (palette.entries = tree.colormap(), count = color_count()).
void* ref_tree_build(const float* rgba, std::size_t w, std::size_t h, int max_colors,
                     int assoc, int gray) {
  RefTree* t = new RefTree();
  t->tree.Build(reinterpret_cast<const rd::RgbaF*>(rgba), w, h, max_colors, assoc != 0,
                gray != 0);
  t->palette->count = t->tree.color_count();
  t->palette->associate_alpha = assoc != 0;
  for (int i = 0; i < t->palette->count; ++i) t->palette->entries[i] = t->tree.colormap()[i];
  return t;
}

void ref_tree_free(void* h) { delete static_cast<RefTree*>(h); }

int ref_tree_color_count(void* h) { return static_cast<RefTree*>(h)->tree.color_count(); }
int ref_tree_depth(void* h) { return static_cast<RefTree*>(h)->tree.depth(); }
std::size_t ref_tree_node_count(void* h) {
  return static_cast<RefTree*>(h)->tree.nodes().size();
}

void ref_tree_colormap(void* h, double* out) {
  RefTree* t = static_cast<RefTree*>(h);
  for (int i = 0; i < t->palette->count; ++i) {
    out[4 * i + 0] = t->palette->entries[i].r;
    out[4 * i + 1] = t->palette->entries[i].g;
    out[4 * i + 2] = t->palette->entries[i].b;
    out[4 * i + 3] = t->palette->entries[i].a;
  }
}

// Node fields: child[16], parent, color_number, number_unique (as int64), level.
void ref_tree_nodes(void* h, int32_t* child, int32_t* parent, uint32_t* color_number,
                    uint64_t* number_unique, uint32_t* level) {
  const std::vector<rd::QNode>& n = static_cast<RefTree*>(h)->tree.nodes();
  for (std::size_t i = 0; i < n.size(); ++i) {
    for (int c = 0; c < 16; ++c) child[16 * i + c] = n[i].child[c];
    parent[i] = n[i].parent;
    color_number[i] = n[i].color_number;
    number_unique[i] = n[i].number_unique;
    level[i] = n[i].level;
  }
}

// RiemersmaWalkCpu (src/rd_riemersma_cpu.cpp:359), stack-walk form.
void ref_walk_seq(void* h, double diffusion, int use_cache, std::size_t w, std::size_t hgt,
                  float* rgba) {
  RefTree* t = static_cast<RefTree*>(h);
  rd::DitherParams p;
  p.diffusion = diffusion;
  p.use_cache = use_cache != 0;
  rd::RiemersmaWalkCpu(*t->palette, p, t->tree, w, hgt, reinterpret_cast<rd::RgbaF*>(rgba),
                       nullptr);
}

// RiemersmaBlocksCpu (src/rd_riemersma_cpu.cpp:477), RgbaF path.  Returns 0 on
// success, else copies the refusal into err.
int ref_walk_blocks(void* h, double diffusion, int block, std::size_t w, std::size_t hgt,
                    float* rgba, int frames, char* err, std::size_t errlen) {
  RefTree* t = static_cast<RefTree*>(h);
  rd::DitherParams p;
  p.diffusion = diffusion;
  p.use_cache = false;
  std::string e;
  rd::RiemersmaBlocksCpu(*t->palette, p, t->tree, w, hgt, reinterpret_cast<rd::RgbaF*>(rgba),
                         frames, block, nullptr, 0, true, &e);
  if (!e.empty()) {
    if (err && errlen) {
      std::strncpy(err, e.c_str(), errlen - 1);
      err[errlen - 1] = '\0';
    }
    return -1;
  }
  return 0;
}

// RiemersmaBlocksCpu with its fused gather and output (src/rd_riemersma_cpu.cpp:
// 224-268, 489-516, 711-801).  `rgba` is read when gather_layout is 0 (and is
// then left unwritten); gather_layout 3 = planar 8-bit 4:4:4, 4 = interleaved
// uint16 with gather_channels 3 or 4.  raw_out receives rgba64 (out_yuv444 0)
// or planar 4:4:4 bytes per frame.
int ref_walk_blocks_raw(void* h, double diffusion, int block, std::size_t w, std::size_t hgt,
                        float* rgba, int frames, unsigned char* raw_out, int out_yuv444,
                        const unsigned char* gather_raw, std::size_t gather_frame_bytes,
                        int gather_layout, int gather_channels, char* err, std::size_t errlen) {
  RefTree* t = static_cast<RefTree*>(h);
  rd::DitherParams p;
  p.diffusion = diffusion;
  p.use_cache = false;
  std::string e;
  rd::RiemersmaBlocksCpu(*t->palette, p, t->tree, w, hgt, reinterpret_cast<rd::RgbaF*>(rgba),
                         frames, block, raw_out, w * hgt, out_yuv444 != 0, &e, gather_raw,
                         gather_frame_bytes, gather_layout, gather_channels);
  if (!e.empty()) {
    if (err && errlen) {
      std::strncpy(err, e.c_str(), errlen - 1);
      err[errlen - 1] = '\0';
    }
    return -1;
  }
  return 0;
}

void ref_hilbert_point(int64_t n, int level, int* x, int* y) { rd::HilbertPoint(n, level, x, y); }

int ref_curve_level(std::size_t w, std::size_t h) { return rd::ComputeCurveLevel(w, h); }

// BuildCurveIndex (src/rd_riemersma_cpu.cpp:269): returns the count.
std::size_t ref_block_curve(std::size_t w, std::size_t h, int32_t* out, int32_t* owner) {
  std::vector<int> c, o;
  const std::size_t n = rd::BuildCurveIndex(rd::ComputeCurveLevel(w, h), w, h, &c, &o);
  for (std::size_t i = 0; i < c.size(); ++i) out[i] = c[i];
  for (std::size_t i = 0; i < o.size(); ++i) owner[i] = o[i];
  return n;
}

// The recursion's leaves (WalkCurve via BuildCurveSequence), x/y interleaved.
// Returns CurveEntryCount(level); the trailing entry is the reference's own.
std::size_t ref_curve_sequence(int level, int32_t* xy) {
  const std::size_t n = rd::CurveEntryCount(level);
  if (n == 0) return 0;
  std::vector<rd::CurveStepEntry> seq(n);
  rd::BuildCurveSequence(level, 0, 0, seq.data());
  for (std::size_t i = 0; i < n; ++i) {
    xy[2 * i] = seq[i].x;
    xy[2 * i + 1] = seq[i].y;
  }
  return n;
}

std::size_t ref_curve_mismatches(int level) { return rd::SelfTestCurveMatchesRecursion(level); }

void ref_error_weights(double* out) {
  double w[rd::kErrorQueueLength];
  rd::build_error_weights(w);
  for (int i = 0; i < rd::kErrorQueueLength; ++i) out[i] = w[i];
}

unsigned ref_scale_char(float q) { return rd::scale_quantum_to_char(q); }

}  // extern "C"
