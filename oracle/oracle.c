/*
 * oracle.c -- TEST INFRASTRUCTURE ONLY: the CPU checker for the CUDA engines.
 *
 * A restatement in plain C of the reference's CPU path (rdither, files cited
 * per function).  It must be compiled with -O2 -ffp-contract=off and without
 * -ffast-math/-march=native, exactly as the reference's CPU oracle is, so
 * that every double operation rounds once in the written order.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define QRANGE 65535.0
#define QSCALE (1.0 / 65535.0)
#define OPAQUE 65535.0
#define EPS 1.0e-12
#define MAX_QNODES 266817
#define MAX_COLORMAP 65536
#define QUEUE 16

/* ---------------------------------------------------------------- rd_types.h */

/* include/rd_types.h:30-33 */
static double safe_reciprocal(double x) {
  const double sign = (x < 0.0) ? -1.0 : 1.0;
  return ((sign * x) >= EPS) ? 1.0 / x : sign * (1.0 / EPS);
}

/* include/rd_types.h:39-43 */
float orc_clamp_pixel(double v) {
  if (v < 0.0) return 0.0f;
  if (v >= QRANGE) return (float)QRANGE;
  return (float)v;
}

/* include/rd_types.h:133-138 */
unsigned char orc_scale_quantum_to_char(float q) {
  if (isnan(q) || q <= 0.0f) return 0;
  const float scaled = q / 257.0f;
  if (scaled >= 255.0f) return 255;
  return (unsigned char)(scaled + 0.5f);
}

/* include/rd_types.h:141-153 */
int orc_cache_offset(int assoc, double r, double g, double b, double a) {
  const unsigned rr = orc_scale_quantum_to_char(orc_clamp_pixel(r)) >> 2;
  const unsigned gg = orc_scale_quantum_to_char(orc_clamp_pixel(g)) >> 2;
  const unsigned bb = orc_scale_quantum_to_char(orc_clamp_pixel(b)) >> 2;
  int off = (int)rr | ((int)gg << 6) | ((int)bb << 12);
  if (assoc) off |= (int)(orc_scale_quantum_to_char(orc_clamp_pixel(a)) >> 2) << 18;
  return off;
}

/* include/rd_types.h:169-176 */
void orc_build_error_weights(double w[16]) {
  double weight = 1.0;
  for (int i = 0; i < QUEUE; ++i) {
    w[i] = safe_reciprocal(weight);
    weight *= exp(log(1.0 / (1.0 / 16.0)) / (QUEUE - 1.0));
  }
}

typedef struct {
  double r, g, b, a;
} dpix;

/* include/rd_types.h:179-192 */
static dpix assoc_pixel(int assoc, const float* px) {
  dpix o;
  o.a = (double)px[3];
  if (!assoc || px[3] == (float)OPAQUE) {
    o.r = (double)px[0];
    o.g = (double)px[1];
    o.b = (double)px[2];
    return o;
  }
  const double alpha = QSCALE * (double)px[3];
  o.r = alpha * (double)px[0];
  o.g = alpha * (double)px[1];
  o.b = alpha * (double)px[2];
  return o;
}

/* include/rd_types.h:195-208 */
static dpix assoc_info(int assoc, const orc_entry* e) {
  dpix o;
  o.a = e->a;
  if (!assoc || e->a == OPAQUE) {
    o.r = e->r;
    o.g = e->g;
    o.b = e->b;
    return o;
  }
  const double alpha = QSCALE * e->a;
  o.r = alpha * e->r;
  o.g = alpha * e->g;
  o.b = alpha * e->b;
  return o;
}

/* ------------------------------------------------------------ Hilbert curve */

/* include/rd_riemersma.h:88-94 */
int orc_curve_level(size_t width, size_t height) {
  const size_t extent = width > height ? width : height;
  if (extent == 0) return 0;
  int level = (int)log2((double)extent);
  if (((size_t)1 << level) < extent) ++level;
  return level;
}

/* src/rd_riemersma_cpu.cpp:167-189 */
void orc_hilbert_point(int64_t n, int level, int* out_x, int* out_y) {
  int x = 0, y = 0;
  const int64_t span = (int64_t)1 << level;
  for (int64_t side = 1; side < span; side <<= 1) {
    const int rx = (int)(1 & (n / 2));
    const int ry = (int)(1 & (n ^ rx));
    if (ry == 0) {
      if (rx == 1) {
        x = (int)(side - 1 - x);
        y = (int)(side - 1 - y);
      }
      const int t = x;
      x = y;
      y = t;
    }
    x += (int)(side * rx);
    y += (int)(side * ry);
    n /= 4;
  }
  *out_x = x;
  *out_y = y;
}

/* The order RiemersmaWalkCpu visits (src/rd_riemersma_cpu.cpp:403-416): the
 * recursion's 4^L-1 leaves followed by the trailing visit at the resting cursor.
 * The leaves equal the closed form for n in [0, 4^L-1) and the resting cursor is
 * HilbertPoint(4^L-1) = (2^L-1, 0), so the walk is the closed form over the whole
 * [0, 4^L), clipped to the image (level 0: the single pixel (0,0)). */
size_t orc_seq_order(size_t width, size_t height, int32_t* out) {
  const int level = orc_curve_level(width, height);
  const int64_t cells = (int64_t)1 << (2 * level);
  size_t k = 0;
  for (int64_t n = 0; n < cells; ++n) {
    int x, y;
    orc_hilbert_point(n, level, &x, &y);
    if (x < 0 || y < 0 || (size_t)x >= width || (size_t)y >= height) continue;
    out[k++] = (int32_t)((size_t)y * width + (size_t)x);
  }
  return k;
}

/* src/rd_riemersma_cpu.cpp:269-356 (BuildCurveIndex) */
size_t orc_block_order(size_t width, size_t height, int32_t* out, int32_t* owner) {
  for (size_t p = 0; p < width * height; ++p) owner[p] = -1;
  const int level = orc_curve_level(width, height);
  if (level <= 0) return 0;
  const int64_t leaves = ((int64_t)1 << (2 * level)) - 1;
  size_t k = 0;
  for (int64_t n = 0; n < leaves; ++n) {
    int x, y;
    orc_hilbert_point(n, level, &x, &y);
    if (x < 0 || y < 0 || (size_t)x >= width || (size_t)y >= height) continue;
    out[k++] = (int32_t)((size_t)y * width + (size_t)x);
  }
  out[k++] = 0; /* :349 the appended origin */
  for (size_t i = 0; i < k; ++i) owner[out[i]] = (int32_t)i; /* :352-354 */
  return k;
}

/* ------------------------------------------------------------------- octree */

static int32_t new_node(orc_tree* t, uint32_t id, uint32_t level, int32_t parent) {
  if (t->node_count == t->node_cap) {
    t->node_cap = t->node_cap ? t->node_cap * 2 : 1024;
    t->nodes = (orc_node*)realloc(t->nodes, t->node_cap * sizeof(orc_node));
  }
  orc_node* n = &t->nodes[t->node_count];
  memset(n, 0, sizeof(*n));
  for (int i = 0; i < 16; ++i) n->child[i] = -1;
  n->id = id;
  n->level = level;
  n->parent = parent;
  return (int32_t)(t->node_count++);
}

static int children_of(const orc_tree* t) { return t->associate_alpha ? 16 : 8; }

typedef struct {
  unsigned c[4];
} packed4;

/* src/rd_octree.cpp:50-57 */
static packed4 pack_channels(double r, double g, double b, double a) {
  packed4 p;
  p.c[0] = orc_scale_quantum_to_char(orc_clamp_pixel(r));
  p.c[1] = orc_scale_quantum_to_char(orc_clamp_pixel(g));
  p.c[2] = orc_scale_quantum_to_char(orc_clamp_pixel(b));
  p.c[3] = orc_scale_quantum_to_char(orc_clamp_pixel(a));
  return p;
}

/* src/rd_octree.cpp:59-67 */
static size_t node_id(const orc_tree* t, const packed4* p, int index) {
  size_t id = (size_t)((p->c[0] >> index) & 1u);
  id |= (size_t)((p->c[1] >> index) & 1u) << 1;
  id |= (size_t)((p->c[2] >> index) & 1u) << 2;
  if (t->associate_alpha) id |= (size_t)((p->c[3] >> index) & 1u) << 3;
  return id;
}

/* src/rd_octree.cpp:69-93 */
static void prune_child(orc_tree* t, int32_t node) {
  const int ch = children_of(t);
  for (int i = 0; i < ch; ++i) {
    const int32_t c = t->nodes[node].child[i];
    if (c >= 0) prune_child(t, c);
  }
  if (t->node_live_count > (size_t)t->maximum_colors) {
    const int32_t parent = t->nodes[node].parent;
    if (parent >= 0) {
      orc_node* p = &t->nodes[parent];
      orc_node* n = &t->nodes[node];
      p->number_unique += n->number_unique;
      for (int c = 0; c < 4; ++c) p->total_color[c] += n->total_color[c];
      p->child[n->id] = -1;
    }
    --t->node_live_count;
  }
}

/* src/rd_octree.cpp:95-102 */
static void prune_level(orc_tree* t, int32_t node) {
  const int ch = children_of(t);
  for (int i = 0; i < ch; ++i) {
    const int32_t c = t->nodes[node].child[i];
    if (c >= 0) prune_level(t, c);
  }
  if ((int)t->nodes[node].level == t->depth) prune_child(t, node);
}

/* src/rd_octree.cpp:104-111 */
static void prune_to_cube_depth(orc_tree* t, int32_t node) {
  const int ch = children_of(t);
  for (int i = 0; i < ch; ++i) {
    const int32_t c = t->nodes[node].child[i];
    if (c >= 0) prune_to_cube_depth(t, c);
  }
  if ((int)t->nodes[node].level > t->depth) prune_child(t, node);
}

/* src/rd_octree.cpp:113-127 */
static void reduce(orc_tree* t, int32_t node) {
  const int ch = children_of(t);
  for (int i = 0; i < ch; ++i) {
    const int32_t c = t->nodes[node].child[i];
    if (c >= 0) reduce(t, c);
  }
  if (t->nodes[node].quantize_error <= t->pruning_threshold) {
    prune_child(t, node);
  } else {
    if (t->nodes[node].number_unique > 0) ++t->color_count;
    if (t->nodes[node].quantize_error < t->next_threshold)
      t->next_threshold = t->nodes[node].quantize_error;
  }
}

/* src/rd_octree.cpp:129-140 */
static size_t qerr_flatten(const orc_tree* t, int32_t node, size_t offset, double* out) {
  if (offset >= t->node_live_count) return 0;
  out[offset] = t->nodes[node].quantize_error;
  size_t n = 1;
  const int ch = children_of(t);
  for (int i = 0; i < ch; ++i) {
    const int32_t c = t->nodes[node].child[i];
    if (c >= 0) n += qerr_flatten(t, c, offset + n, out);
  }
  return n;
}

/* src/rd_octree.cpp:23-29 */
static int qerr_compare(const void* a, const void* b) {
  const double* p = (const double*)a;
  const double* q = (const double*)b;
  if (*p > *q) return 1;
  if (fabs(*q - *p) <= EPS) return 0;
  return -1;
}

/* src/rd_octree.cpp:142-176 */
static void define_colormap(orc_tree* t, int32_t node) {
  const int ch = children_of(t);
  for (int i = 0; i < ch; ++i) {
    const int32_t c = t->nodes[node].child[i];
    if (c >= 0) define_colormap(t, c);
  }
  orc_node* n = &t->nodes[node];
  if (n->number_unique == 0) return;
  orc_entry* q = &t->colormap[t->color_count];
  const double alpha = safe_reciprocal((double)n->number_unique);
  if (!t->associate_alpha) {
    q->r = (double)(float)(alpha * QRANGE * n->total_color[0]);
    q->g = (double)(float)(alpha * QRANGE * n->total_color[1]);
    q->b = (double)(float)(alpha * QRANGE * n->total_color[2]);
    q->a = OPAQUE;
  } else {
    const double opacity = alpha * QRANGE * n->total_color[3];
    q->a = (double)(float)opacity;
    if (q->a == OPAQUE) {
      q->r = (double)(float)(alpha * QRANGE * n->total_color[0]);
      q->g = (double)(float)(alpha * QRANGE * n->total_color[1]);
      q->b = (double)(float)(alpha * QRANGE * n->total_color[2]);
    } else {
      const double gamma = safe_reciprocal(QSCALE * q->a);
      q->r = (double)(float)(alpha * gamma * QRANGE * n->total_color[0]);
      q->g = (double)(float)(alpha * gamma * QRANGE * n->total_color[1]);
      q->b = (double)(float)(alpha * gamma * QRANGE * n->total_color[2]);
    }
  }
  n->color_number = (uint32_t)t->color_count;
  ++t->color_count;
}

static int pixels_equal(const float* a, const float* b) {
  return a[0] == b[0] && a[1] == b[1] && a[2] == b[2] && a[3] == b[3];
}

/* src/rd_octree.cpp:305-362 (process_row) */
static void process_row(orc_tree* t, const float* row, size_t width, int level_limit,
                        int colors_level) {
  const double midpoint = QRANGE / 2.0;
  size_t x = 0;
  while (x < width) {
    size_t count = 1;
    while (x + count < width && pixels_equal(row + 4 * x, row + 4 * (x + count))) ++count;
    const dpix pixel = assoc_pixel(t->associate_alpha, row + 4 * x);
    int index = 7;
    double bisect = (QRANGE + 1.0) / 2.0;
    double mid[4] = {midpoint, midpoint, midpoint, midpoint};
    int32_t node = t->root;
    const packed4 packed = pack_channels(pixel.r, pixel.g, pixel.b, pixel.a);
    for (int level = 1; level <= level_limit; ++level) {
      bisect *= 0.5;
      const size_t id = node_id(t, &packed, index);
      mid[0] += (id & 1) ? bisect : -bisect;
      mid[1] += (id & 2) ? bisect : -bisect;
      mid[2] += (id & 4) ? bisect : -bisect;
      mid[3] += (id & 8) ? bisect : -bisect;
      if (t->nodes[node].child[id] < 0) {
        const int32_t created = new_node(t, (uint32_t)id, (uint32_t)level, node);
        t->nodes[node].child[id] = created;
        ++t->node_live_count;
        if (level == colors_level) ++t->color_count;
      }
      node = t->nodes[node].child[id];
      const double e0 = QSCALE * (pixel.r - mid[0]);
      const double e1 = QSCALE * (pixel.g - mid[1]);
      const double e2 = QSCALE * (pixel.b - mid[2]);
      const double e3 = t->associate_alpha ? (QSCALE * (pixel.a - mid[3])) : 0.0;
      double distance = e0 * e0 + e1 * e1 + e2 * e2 + e3 * e3;
      if (isnan(distance)) distance = 0.0;
      t->nodes[node].quantize_error += (double)count * sqrt(distance);
      t->nodes[t->root].quantize_error += t->nodes[node].quantize_error;
      --index;
    }
    orc_node* leaf = &t->nodes[node];
    leaf->number_unique += count;
    leaf->total_color[0] += (double)count * QSCALE * (double)orc_clamp_pixel(pixel.r);
    leaf->total_color[1] += (double)count * QSCALE * (double)orc_clamp_pixel(pixel.g);
    leaf->total_color[2] += (double)count * QSCALE * (double)orc_clamp_pixel(pixel.b);
    leaf->total_color[3] += (double)count * QSCALE *
                            (double)orc_clamp_pixel(t->associate_alpha ? pixel.a : OPAQUE);
    x += count;
  }
}

/* src/rd_octree.cpp:219-409 (ColorTree::Build) */
int orc_tree_build(orc_tree* t, const float* pixels, size_t width, size_t height,
                   int max_colors, int associate_alpha, int grayscale) {
  memset(t, 0, sizeof(*t));
  t->colormap = (orc_entry*)malloc(sizeof(orc_entry) * MAX_COLORMAP);
  if (!t->colormap) return -1;
  for (int i = 0; i < MAX_COLORMAP; ++i) {
    t->colormap[i].r = t->colormap[i].g = t->colormap[i].b = 0.0;
    t->colormap[i].a = OPAQUE;
  }
  t->associate_alpha = associate_alpha ? 1 : 0;
  t->maximum_colors = (max_colors <= 0) ? MAX_COLORMAP : max_colors;
  if (t->maximum_colors > MAX_COLORMAP) t->maximum_colors = MAX_COLORMAP;
  int depth = 1;
  for (size_t colors = (size_t)t->maximum_colors; colors != 0; ++depth) colors >>= 2;
  if (depth > 2) --depth;
  if (t->associate_alpha && depth > 5) --depth;
  if (grayscale) depth = 8;
  if (depth > 8) depth = 8;
  if (depth < 2) depth = 2;
  t->depth = depth;

  t->root = new_node(t, 0, 0, -1);
  t->node_live_count = 1;
  t->nodes[t->root].parent = t->root;

  size_t y = 0;
  for (; y < height; ++y) {
    if (t->node_live_count > (size_t)MAX_QNODES) {
      prune_level(t, t->root);
      --t->depth;
    }
    process_row(t, pixels + 4 * y * width, width, 8, 8);
    if (t->color_count > t->maximum_colors) {
      prune_to_cube_depth(t, t->root);
      break;
    }
  }
  ++y;
  for (; y < height; ++y) {
    if (t->node_live_count > (size_t)MAX_QNODES) {
      prune_level(t, t->root);
      --t->depth;
    }
    process_row(t, pixels + 4 * y * width, width, t->depth, t->depth);
  }

  if (t->color_count > t->maximum_colors) {
    t->next_threshold = 0.0;
    if (t->node_live_count > 0) {
      const size_t n = t->node_live_count;
      double* errors = (double*)calloc(n, sizeof(double));
      (void)qerr_flatten(t, t->root, 0, errors);
      qsort(errors, n, sizeof(double), qerr_compare);
      const size_t aggressive = (110u * ((size_t)t->maximum_colors + 1u)) / 100u;
      if (n > aggressive) t->next_threshold = errors[n - aggressive];
      free(errors);
    }
  }
  while (t->color_count > t->maximum_colors) {
    t->pruning_threshold = t->next_threshold;
    t->next_threshold = t->nodes[t->root].quantize_error - 1.0;
    t->color_count = 0;
    reduce(t, t->root);
  }
  t->color_count = 0;
  define_colormap(t, t->root);
  return 0;
}

void orc_tree_free(orc_tree* t) {
  free(t->nodes);
  free(t->colormap);
  memset(t, 0, sizeof(*t));
}

/* src/rd_octree.cpp:178-217 (ClosestColor) */
static void closest_color(const orc_tree* t, int32_t node, const dpix* target,
                          double* distance, int* color_number) {
  const int ch = children_of(t);
  for (int i = 0; i < ch; ++i) {
    const int32_t c = t->nodes[node].child[i];
    if (c >= 0) closest_color(t, c, target, distance, color_number);
  }
  const orc_node* n = &t->nodes[node];
  if (n->number_unique == 0) return;
  const orc_entry* p = &t->colormap[n->color_number];
  double alpha = 1.0, beta = 1.0;
  if (t->associate_alpha) {
    alpha = QSCALE * p->a;
    beta = QSCALE * target->a;
  }
  double pixel = alpha * p->r - beta * target->r;
  double d = pixel * pixel;
  if (d <= *distance) {
    pixel = alpha * p->g - beta * target->g;
    d += pixel * pixel;
    if (d <= *distance) {
      pixel = alpha * p->b - beta * target->b;
      d += pixel * pixel;
      if (d <= *distance) {
        if (t->associate_alpha) {
          pixel = p->a - target->a;
          d += pixel * pixel;
        }
        if (d <= *distance) {
          *distance = d;
          *color_number = (int)n->color_number;
        }
      }
    }
  }
}

/* src/rd_riemersma_cpu.cpp:82-92: descent from the root, then search the
 * subtree of node->parent. */
int orc_tree_lookup(const orc_tree* t, double r, double g, double b, double a) {
  const packed4 packed = pack_channels(r, g, b, a);
  int32_t node = t->root;
  for (int i = 7; i > 0; --i) {
    const size_t id = node_id(t, &packed, i);
    const int32_t c = t->nodes[node].child[id];
    if (c < 0) break;
    node = c;
  }
  double distance = 4.0 * ((QRANGE + 1.0) * (QRANGE + 1.0)) + 1.0;
  int index = 0;
  dpix target = {r, g, b, a};
  closest_color(t, t->nodes[node].parent, &target, &distance, &index);
  return index;
}

/* ------------------------------------------------------------------ walks */

/* src/rd_riemersma_cpu.cpp:39-113 (Visit) with the scaled weights of :370-373. */
static void visit(const orc_tree* t, const orc_entry* palette, int assoc,
                  const double sw[16], dpix err[16], int* cache, float* px,
                  uint8_t* idx_slot) {
  dpix pixel = assoc_pixel(assoc, px);
  for (int i = 0; i < QUEUE; ++i) {
    const double w = sw[i];
    pixel.r += w * err[i].r;
    pixel.g += w * err[i].g;
    pixel.b += w * err[i].b;
    if (assoc) pixel.a += w * err[i].a;
  }
  pixel.r = (double)orc_clamp_pixel(pixel.r);
  pixel.g = (double)orc_clamp_pixel(pixel.g);
  pixel.b = (double)orc_clamp_pixel(pixel.b);
  if (assoc) pixel.a = (double)orc_clamp_pixel(pixel.a);
  const int key = orc_cache_offset(assoc, pixel.r, pixel.g, pixel.b, pixel.a);
  int index = cache ? cache[key] : -1;
  if (index < 0) {
    index = orc_tree_lookup(t, pixel.r, pixel.g, pixel.b, pixel.a);
    if (cache) cache[key] = index;
  }
  px[0] = (float)palette[index].r;
  px[1] = (float)palette[index].g;
  px[2] = (float)palette[index].b;
  if (assoc) px[3] = (float)palette[index].a;
  if (idx_slot) *idx_slot = (uint8_t)index;
  for (int i = 0; i < QUEUE - 1; ++i) err[i] = err[i + 1];
  const dpix color = assoc_info(assoc, &palette[index]);
  err[QUEUE - 1].r = pixel.r - color.r;
  err[QUEUE - 1].g = pixel.g - color.g;
  err[QUEUE - 1].b = pixel.b - color.b;
  if (assoc) err[QUEUE - 1].a = pixel.a - color.a;
}

static void scaled_weights(double diffusion, double sw[16]) {
  double w[16];
  orc_build_error_weights(w);
  for (int k = 0; k < QUEUE; ++k) sw[k] = (1.0 / 16.0) * diffusion * w[k];
}

/* src/rd_riemersma_cpu.cpp:359-417 (RiemersmaWalkCpu) */
void orc_walk_seq(const orc_tree* t, const orc_entry* palette, int count,
                  int assoc, double diffusion, int use_cache, size_t width,
                  size_t height, float* pixels, uint8_t* idx_out) {
  (void)count;
  double sw[16];
  scaled_weights(diffusion, sw);
  dpix err[16];
  memset(err, 0, sizeof(err));
  int* cache = NULL;
  if (use_cache) {
    const size_t entries = assoc ? ((size_t)1 << 24) : ((size_t)1 << 18);
    cache = (int*)malloc(entries * sizeof(int));
    for (size_t i = 0; i < entries; ++i) cache[i] = -1;
  }
  int32_t* order = (int32_t*)malloc((width * height + 1) * sizeof(int32_t));
  const size_t n = orc_seq_order(width, height, order);
  for (size_t i = 0; i < n; ++i) {
    const size_t p = (size_t)order[i];
    visit(t, palette, assoc, sw, err, cache, pixels + 4 * p, idx_out ? idx_out + p : NULL);
  }
  free(order);
  free(cache);
}

/* The walk of RiemersmaBlocksCpu (src/rd_riemersma_cpu.cpp:640-696): every
 * block of the list from a zeroed queue, no memo; chosen[i] per position. */
static void block_walk_chosen(const orc_tree* t, const orc_entry* palette, int assoc,
                              const double sw[16], int block, const int32_t* curve, int n,
                              const float* pixels, uint8_t* chosen) {
  const int nblocks = (n + block - 1) / block;
  for (int b = 0; b < nblocks; ++b) {
    dpix err[16];
    memset(err, 0, sizeof(err));
    const int begin = b * block;
    const int end = (begin + block < n) ? (begin + block) : n;
    for (int i = begin; i < end; ++i) {
      dpix pixel = assoc_pixel(assoc, pixels + 4 * (size_t)curve[i]);
      for (int k = 0; k < QUEUE; ++k) {
        const double w = sw[k];
        pixel.r += w * err[k].r;
        pixel.g += w * err[k].g;
        pixel.b += w * err[k].b;
        if (assoc) pixel.a += w * err[k].a;
      }
      pixel.r = (double)orc_clamp_pixel(pixel.r);
      pixel.g = (double)orc_clamp_pixel(pixel.g);
      pixel.b = (double)orc_clamp_pixel(pixel.b);
      if (assoc) pixel.a = (double)orc_clamp_pixel(pixel.a);
      const int index = orc_tree_lookup(t, pixel.r, pixel.g, pixel.b, pixel.a);
      chosen[i] = (uint8_t)index;
      for (int k = 0; k < QUEUE - 1; ++k) err[k] = err[k + 1];
      const dpix color = assoc_info(assoc, &palette[index]);
      err[QUEUE - 1].r = pixel.r - color.r;
      err[QUEUE - 1].g = pixel.g - color.g;
      err[QUEUE - 1].b = pixel.b - color.b;
      if (assoc) err[QUEUE - 1].a = pixel.a - color.a;
    }
  }
}

/* src/rd_riemersma_cpu.cpp:477-805 (RiemersmaBlocksCpu), RgbaF path, 1 frame. */
int orc_walk_blocks(const orc_tree* t, const orc_entry* palette, int count,
                    int assoc, double diffusion, int block, size_t width,
                    size_t height, float* pixels, uint8_t* idx_out) {
  if (count > 256) return -1;
  if (block < QUEUE) return -1;
  double sw[16];
  scaled_weights(diffusion, sw);
  const size_t pixels_n = width * height;
  int32_t* curve = (int32_t*)malloc((pixels_n + 1) * sizeof(int32_t));
  int32_t* owner = (int32_t*)malloc((pixels_n ? pixels_n : 1) * sizeof(int32_t));
  const int n = (int)orc_block_order(width, height, curve, owner);
  uint8_t* chosen = (uint8_t*)malloc((size_t)(n > 0 ? n : 1));
  block_walk_chosen(t, palette, assoc, sw, block, curve, n, pixels, chosen);
  for (int i = 0; i < n; ++i) {
    const int p = curve[i];
    if (owner[p] != i) continue;
    const orc_entry* e = &palette[chosen[i]];
    float* out = pixels + 4 * (size_t)p;
    out[0] = (float)e->r;
    out[1] = (float)e->g;
    out[2] = (float)e->b;
    if (assoc) out[3] = (float)e->a;
    if (idx_out) idx_out[p] = chosen[i];
  }
  free(chosen);
  free(owner);
  free(curve);
  return 0;
}

/* The chosen index at every position of the block-mode list, in list order
 * (the array src/rd_riemersma_cpu.cpp:640-696 fills before its owner
 * scatter).  Returns the list length, or -1 for the refusals. */
int orc_block_chosen(const orc_tree* t, const orc_entry* palette, int count, int assoc,
                     double diffusion, int block, size_t width, size_t height,
                     const float* pixels, uint8_t* chosen_out) {
  if (count > 256) return -1;
  if (block < QUEUE) return -1;
  double sw[16];
  scaled_weights(diffusion, sw);
  const size_t pixels_n = width * height;
  int32_t* curve = (int32_t*)malloc((pixels_n + 1) * sizeof(int32_t));
  int32_t* owner = (int32_t*)malloc((pixels_n ? pixels_n : 1) * sizeof(int32_t));
  const int n = (int)orc_block_order(width, height, curve, owner);
  block_walk_chosen(t, palette, assoc, sw, block, curve, n, pixels, chosen_out);
  free(owner);
  free(curve);
  return n;
}

/* src/rd_approx_cuda.cu:73-88 (BuildInverseFilter) */
void orc_inverse_filter(int taps, double diffusion, double* g) {
  double w[16];
  orc_build_error_weights(w);
  for (int d = 0; d <= taps; ++d) g[d] = 0.0;
  g[0] = 1.0;
  for (int d = 1; d <= taps; ++d) {
    double acc = 0.0;
    const int kmax = (d < QUEUE) ? d : QUEUE;
    for (int k = 1; k <= kmax; ++k) acc += (diffusion / 16.0) * w[k - 1] * g[d - k];
    g[d] = acc;
  }
}

/* ---- video frame formats on either side of the block walk ----------------
 * RiemersmaBlocksCpu's fused gather widens the decoder's bytes to the RgbaF a
 * reader would have produced, and its fused output is the convert pass's
 * arithmetic applied to the RgbaF the non-fused walk leaves behind
 * (src/rd_riemersma_cpu.cpp:711-753 says so and reproduces it byte for byte),
 * so the checker is widen -> orc_walk_blocks -> narrow. */

/* include/rd_types.h:75-97 (SwsClip16, SwsYuvToRgb16), in the reference's
 * own order of operations: unsigned wrap of (c - 128) * 512, the 0x10000 and
 * -8192 luma offsets, the 9539 scale, the (1 << 13) - (1 << 29) rounding
 * offset, >> 14, clip around 1 << 15. */
static uint16_t sws_clip(int x) {
  const int v = x + 32768;
  return (uint16_t)(v < 0 ? 0 : (v > 65535 ? 65535 : v));
}
static void sws_yuv_to_rgb16(unsigned y, unsigned u, unsigned v, uint16_t out[3]) {
  int yy = (int)((y - 128u) * 512u);
  const int uu = (int)((u - 128u) * 512u);
  const int vv = (int)((v - 128u) * 512u);
  yy += 0x10000;
  yy -= 8192;
  yy *= 9539;
  yy += (1 << 13) - (1 << 29);
  out[0] = sws_clip((vv * 13075 + yy) >> 14);
  out[1] = sws_clip((vv * -6660 + uu * -3209 + yy) >> 14);
  out[2] = sws_clip((uu * 16525 + yy) >> 14);
}

/* src/rd_blocks_cuda.cu:660-676 (d_chroma_bilinear) as the 4:2:0 gather calls
 * it (:677-706): chroma plane w2 x h2, sample (x >> 1, y >> 1), phase (x & 1,
 * y & 1).  The reference has no CPU form of this mode. */
static unsigned chroma_bilinear(const unsigned char* plane, int w2, int h2, int x, int y) {
  const int cx = x >> 1, cy = y >> 1, ox = x & 1, oy = y & 1;
  const int x1 = (cx + 1 < w2) ? cx + 1 : cx;
  const int y1 = (cy + 1 < h2) ? cy + 1 : cy;
  const int a = plane[(size_t)cy * w2 + cx];
  const int b = plane[(size_t)cy * w2 + x1];
  const int c = plane[(size_t)y1 * w2 + cx];
  const int d = plane[(size_t)y1 * w2 + x1];
  const int top = a * (2 - ox) + b * ox;
  const int bot = c * (2 - ox) + d * ox;
  return (unsigned)((top * (2 - oy) + bot * oy + 2) >> 2);
}

/* src/rd_riemersma_cpu.cpp:496-516 (gather_pixel) for formats 6 (rgb48),
 * 8 (rgba64) and 444 (planar 4:4:4); 420 (planar 4:2:0) per the CUDA gather
 * above; 3 / 4 / 16 as the reader gives them (8-bit samples x 257, RgbaF as
 * is).  Writes W*H RgbaF. Returns -1 for an unknown format or odd 4:2:0. */
int orc_widen_frame(int format, const void* in, size_t width, size_t height, float* rgba) {
  const size_t n = width * height;
  const unsigned char* b = (const unsigned char*)in;
  const uint16_t* q = (const uint16_t*)in;
  if (format == 420 && ((width & 1) || (height & 1))) return -1;
  for (size_t p = 0; p < n; ++p) {
    float* o = rgba + 4 * p;
    switch (format) {
      case 3:
        o[0] = (float)(b[3 * p] * 257); o[1] = (float)(b[3 * p + 1] * 257);
        o[2] = (float)(b[3 * p + 2] * 257); o[3] = 65535.0f;
        break;
      case 4:
        o[0] = (float)(b[4 * p] * 257); o[1] = (float)(b[4 * p + 1] * 257);
        o[2] = (float)(b[4 * p + 2] * 257); o[3] = (float)(b[4 * p + 3] * 257);
        break;
      case 16:
        memcpy(o, (const float*)in + 4 * p, 16);
        break;
      case 6:
        o[0] = (float)q[3 * p]; o[1] = (float)q[3 * p + 1]; o[2] = (float)q[3 * p + 2];
        o[3] = (float)65535.0;
        break;
      case 8:
        o[0] = (float)q[4 * p]; o[1] = (float)q[4 * p + 1]; o[2] = (float)q[4 * p + 2];
        o[3] = (float)q[4 * p + 3];
        break;
      case 444:
      case 420: {
        uint16_t rgb[3];
        unsigned u, v;
        if (format == 444) {
          u = b[n + p];
          v = b[2 * n + p];
        } else {
          const int w2 = (int)(width >> 1), h2 = (int)(height >> 1);
          const int x = (int)(p % width), y = (int)(p / width);
          u = chroma_bilinear(b + n, w2, h2, x, y);
          v = chroma_bilinear(b + n + (size_t)w2 * h2, w2, h2, x, y);
        }
        sws_yuv_to_rgb16(b[p], u, v, rgb);
        o[0] = (float)rgb[0]; o[1] = (float)rgb[1]; o[2] = (float)rgb[2];
        o[3] = (float)65535.0;
        break;
      }
      default:
        return -1;
    }
  }
  return 0;
}

/* The convert pass the fused output replaces: FloatsToRaw's four uint16 per
 * pixel (format 8) or FloatsToYuv444's planar BT.601 bytes (format 444), as
 * src/rd_riemersma_cpu.cpp:719-753 and :776-801 restate them: (int)float >> 8
 * per channel, then ((66r + 129g + 25b + 128) >> 8) + 16 and the two chroma
 * rows, clamped to a byte.  Returns -1 for an unknown format. */
int orc_narrow_frame(int format, const float* rgba, size_t width, size_t height, void* out) {
  const size_t n = width * height;
  for (size_t p = 0; p < n; ++p) {
    const float* s = rgba + 4 * p;
    if (format == 8) {
      uint16_t* u = (uint16_t*)out + 4 * p;
      u[0] = (uint16_t)s[0]; u[1] = (uint16_t)s[1]; u[2] = (uint16_t)s[2]; u[3] = (uint16_t)s[3];
    } else if (format == 444) {
      unsigned char* o = (unsigned char*)out;
      const int r8 = (int)s[0] >> 8, g8 = (int)s[1] >> 8, b8 = (int)s[2] >> 8;
      const int yv = ((66 * r8 + 129 * g8 + 25 * b8 + 128) >> 8) + 16;
      const int uv = ((-38 * r8 - 74 * g8 + 112 * b8 + 128) >> 8) + 128;
      const int vv = ((112 * r8 - 94 * g8 - 18 * b8 + 128) >> 8) + 128;
      o[p] = (unsigned char)(yv < 0 ? 0 : (yv > 255 ? 255 : yv));
      o[n + p] = (unsigned char)(uv < 0 ? 0 : (uv > 255 ? 255 : uv));
      o[2 * n + p] = (unsigned char)(vv < 0 ? 0 : (vv > 255 ? 255 : vv));
    } else {
      return -1;
    }
  }
  return 0;
}
