// rdb_plan.cpp -- flattening a palette + colour tree into the device plan.
#include "rdb_plan.h"

#include <cstring>
#include <utility>

#include "rdb_numeric.h"

namespace rdb {
namespace {

std::size_t Align16(std::size_t v) { return (v + 15u) & ~static_cast<std::size_t>(15u); }

}  // namespace

std::string BuildPlan(const PlanInput& in, std::vector<uint8_t>* blob) {
  if (in.count < 1) return "empty palette";
  if (in.count > kMaxPaletteColors) {
    return "the palette has " + std::to_string(in.count) +
           " colours; the device engines carry one palette index per byte (at most 256)";
  }
  if (in.node_count < 1 || in.root < 0 || in.root >= in.node_count) return "empty colour tree";
  const int fan = in.assoc ? 16 : 8;
  const double* search = in.search_colors ? in.search_colors : in.colors;

  // Live nodes: reachable from the root through child links, children in
  // index order (rd_octree.cpp:180-185).  Pre-order numbering, root = 0.
  std::vector<int32_t> live_of(static_cast<std::size_t>(in.node_count), -1);
  std::vector<int32_t> orig;       // live id -> original index
  std::vector<int32_t> up;         // live id -> live parent (root: itself)
  std::vector<std::pair<int32_t, int32_t>> stack;
  live_of[in.root] = 0;
  orig.push_back(in.root);
  up.push_back(0);
  stack.emplace_back(in.root, 0);
  while (!stack.empty()) {
    const int32_t node = stack.back().first;
    const int32_t next = stack.back().second;
    if (next >= fan) {
      stack.pop_back();
      continue;
    }
    stack.back().second = next + 1;
    const int32_t c = in.child[16 * static_cast<std::size_t>(node) + next];
    if (c < 0) continue;
    if (c >= in.node_count) return "colour tree child index out of range";
    if (live_of[c] >= 0) return "colour tree is not a tree (a node is reached twice)";
    if (static_cast<int>(orig.size()) >= kMaxPlanNodes) return "colour tree too large";
    if (stack.size() > 64) return "colour tree too deep";
    live_of[c] = static_cast<int32_t>(orig.size());
    orig.push_back(c);
    up.push_back(live_of[node]);
    stack.emplace_back(c, 0);
  }
  const int nodes = static_cast<int>(orig.size());
  // The reference reads node->parent (include/rd_octree.h:98); for a tree
  // built by the octree it is the node the child link hangs from, and the
  // root's parent is the root.  Refuse a tree where the two disagree.
  if (in.parent) {
    for (int i = 0; i < nodes; ++i) {
      const int32_t p = in.parent[orig[i]];
      const int32_t expect = orig[up[i]];
      if (p != expect) return "colour tree parent links disagree with its child links";
    }
  }

  // Post-order slots and per-node subtree runs.
  std::vector<uint8_t> seq;
  std::vector<int32_t> first(static_cast<std::size_t>(nodes), 0);
  std::vector<int32_t> span(static_cast<std::size_t>(nodes), 0);
  {
    std::vector<std::pair<int32_t, int32_t>> st;  // (live id, next child)
    st.emplace_back(0, 0);
    first[0] = 0;
    while (!st.empty()) {
      const int32_t l = st.back().first;
      const int32_t next = st.back().second;
      if (next < fan) {
        st.back().second = next + 1;
        const int32_t c = in.child[16 * static_cast<std::size_t>(orig[l]) + next];
        if (c >= 0) {
          first[live_of[c]] = static_cast<int32_t>(seq.size());
          st.emplace_back(live_of[c], 0);
        }
        continue;
      }
      st.pop_back();
      const int32_t o = orig[l];
      if (in.number_unique[o] != 0) {
        const uint32_t cn = in.color_number[o];
        if (cn >= static_cast<uint32_t>(in.count)) return "colour number outside the palette";
        if (seq.size() >= static_cast<std::size_t>(kMaxPaletteColors)) {
          return "colour tree has more coloured nodes than a byte index can carry";
        }
        seq.push_back(static_cast<uint8_t>(cn));
      }
      span[l] = static_cast<int32_t>(seq.size()) - first[l];
    }
  }
  const int slots = static_cast<int>(seq.size());

  const int pal_stride = in.assoc ? 64 : 32;
  PlanHeader h;
  std::memset(&h, 0, sizeof(h));
  h.count = in.count;
  h.assoc = in.assoc ? 1 : 0;
  h.nodes = nodes;
  h.fan = fan;
  h.slots = slots;
  h.pal_stride = pal_stride;
  std::size_t off = sizeof(PlanHeader);
  h.off_pal = static_cast<int32_t>(off);
  off = Align16(off + static_cast<std::size_t>(in.count) * pal_stride);
  h.off_child = static_cast<int32_t>(off);
  off = Align16(off + static_cast<std::size_t>(nodes) * fan * sizeof(int16_t));
  h.off_range = static_cast<int32_t>(off);
  off = Align16(off + static_cast<std::size_t>(nodes) * 2 * sizeof(uint16_t));
  h.off_seq = static_cast<int32_t>(off);
  off = Align16(off + static_cast<std::size_t>(slots > 0 ? slots : 1));
  h.slot_stride = (slots + 1) & ~1;
  h.off_slotpal = static_cast<int32_t>(off);
  off = Align16(off + static_cast<std::size_t>(4) * h.slot_stride * sizeof(double));
  const int jump_entries = 1 << (kJumpLevels * (in.assoc ? 4 : 3));
  h.off_jump = static_cast<int32_t>(off);
  off = Align16(off + static_cast<std::size_t>(jump_entries) * sizeof(uint16_t));
  h.smem_bytes = static_cast<int32_t>(off);
  h.off_out = static_cast<int32_t>(off);
  off = Align16(off + static_cast<std::size_t>(in.count) * 4 * sizeof(float));
  h.total_bytes = static_cast<int32_t>(off);

  blob->assign(off, 0);
  uint8_t* b = blob->data();
  std::memcpy(b, &h, sizeof(h));

  for (int i = 0; i < in.count; ++i) {
    double* e = reinterpret_cast<double*>(b + h.off_pal + static_cast<std::size_t>(i) * pal_stride);
    const double* c = in.colors + 4 * i;
    const double* s = search + 4 * i;
    if (!in.assoc) {
      // Without alpha ClosestColor's alpha and beta are 1.0 and 1.0 * c == c.
      // The distance uses the tree's colormap, the residual the palette; the
      // reference asserts them equal (src/rd_cli.cpp:2516-2530) and so must a
      // plan without alpha, which keeps one table.
      if (s[0] != c[0] || s[1] != c[1] || s[2] != c[2]) {
        return "the tree's colormap differs from the palette";
      }
      e[0] = c[0];
      e[1] = c[1];
      e[2] = c[2];
      e[3] = c[3];
    } else {
      const double alpha = kQuantumScale * s[3];  // rd_octree.cpp:193
      e[0] = alpha * s[0];
      e[1] = alpha * s[1];
      e[2] = alpha * s[2];
      e[3] = s[3];
      // AssociateAlphaPixelInfo of the palette entry (rd_types.h:195-208).
      if (c[3] == kOpaqueAlpha) {
        e[4] = c[0];
        e[5] = c[1];
        e[6] = c[2];
      } else {
        const double ca = kQuantumScale * c[3];
        e[4] = ca * c[0];
        e[5] = ca * c[1];
        e[6] = ca * c[2];
      }
      e[7] = c[3];
    }
    float* o = reinterpret_cast<float*>(b + h.off_out) + 4 * i;
    o[0] = static_cast<float>(c[0]);
    o[1] = static_cast<float>(c[1]);
    o[2] = static_cast<float>(c[2]);
    o[3] = static_cast<float>(c[3]);
  }
  int16_t* child = reinterpret_cast<int16_t*>(b + h.off_child);
  uint16_t* range = reinterpret_cast<uint16_t*>(b + h.off_range);
  for (int l = 0; l < nodes; ++l) {
    for (int k = 0; k < fan; ++k) {
      const int32_t c = in.child[16 * static_cast<std::size_t>(orig[l]) + k];
      child[l * fan + k] = static_cast<int16_t>(c >= 0 ? live_of[c] : -1);
    }
    // The search runs over the subtree of the stopping node's parent.
    const int32_t p = up[l];
    range[2 * l] = static_cast<uint16_t>(first[p]);
    range[2 * l + 1] = static_cast<uint16_t>(span[p]);
  }
  std::memcpy(b + h.off_seq, seq.data(), seq.size());

  // Distance-side colours in slot order, one row per channel, so a search
  // over a run of slots reads consecutive doubles.
  double* slotpal = reinterpret_cast<double*>(b + h.off_slotpal);
  for (int s = 0; s < slots; ++s) {
    const double* e = reinterpret_cast<const double*>(b + h.off_pal +
                                                      static_cast<std::size_t>(seq[s]) * pal_stride);
    for (int c = 0; c < 4; ++c) slotpal[static_cast<std::size_t>(c) * h.slot_stride + s] = e[c];
  }

  // The first kJumpLevels levels of the descent (src/rd_riemersma_cpu.cpp:84-89)
  // for every combination of the top bits.
  uint16_t* jump = reinterpret_cast<uint16_t*>(b + h.off_jump);
  const int bits = in.assoc ? 4 : 3;
  for (int idx = 0; idx < jump_entries; ++idx) {
    int node = 0;
    bool stopped = false;
    for (int level = 0; level < kJumpLevels && !stopped; ++level) {
      const int bit = kJumpLevels - 1 - level;  // top bit first
      int id = 0;
      for (int c = 0; c < bits; ++c) {
        const int top = (idx >> (kJumpLevels * c)) & ((1 << kJumpLevels) - 1);
        id |= ((top >> bit) & 1) << c;
      }
      const int16_t next = child[node * fan + id];
      if (next < 0) {
        stopped = true;
      } else {
        node = next;
      }
    }
    jump[idx] = static_cast<uint16_t>(node | (stopped ? 0x8000 : 0));
  }
  return std::string();
}

}  // namespace rdb
