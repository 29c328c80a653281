/*
 * oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's CPU algorithm for the Riemersma hot
 * path: the ImageMagick-semantics colour octree (palette + tree), the Hilbert
 * visit orders, the sequential memoised walk and the block walk.  It is the
 * checker that the CUDA engines are compared against.  Only tests/, the smoke
 * entry point and bench.py's CPU-baseline leg may load it; no product code
 * links or calls it.
 *
 * Parity of this restatement is pinned two ways: against the reference's own
 * CPU sources compiled unmodified into oracle/_ref (see oracle/Makefile), and
 * against the golden vectors in tests/golden/ that were generated from that
 * build.
 *
 * Every function cites the reference file:line it restates.
 */
#ifndef RDB_ORACLE_H_
#define RDB_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* include/rd_types.h:156-158 (PaletteEntry): four doubles, Q16 range. */
typedef struct orc_entry {
  double r, g, b, a;
} orc_entry;

/* include/rd_octree.h:43-52 (QNode). */
typedef struct orc_node {
  int32_t child[16];
  int32_t parent;
  double total_color[4];
  double quantize_error;
  uint64_t number_unique;
  uint32_t color_number;
  uint32_t id;
  uint32_t level;
} orc_node;

typedef struct orc_tree {
  orc_node* nodes;
  size_t node_count;
  size_t node_cap;
  orc_entry* colormap; /* kMaxColormapSize entries */
  int color_count;
  int maximum_colors;
  int depth;
  size_t node_live_count;
  double pruning_threshold;
  double next_threshold;
  int associate_alpha;
  int32_t root;
} orc_tree;

/* rd_types.h helpers */
float orc_clamp_pixel(double v);
unsigned char orc_scale_quantum_to_char(float q);
int orc_cache_offset(int associate_alpha, double r, double g, double b, double a);
void orc_build_error_weights(double w[16]);

/* rd_riemersma.h:88-94 */
int orc_curve_level(size_t width, size_t height);
/* rd_riemersma_cpu.cpp:167-189 */
void orc_hilbert_point(int64_t n, int level, int* x, int* y);
/* Sequential visit order (RiemersmaWalkCpu's order clipped to the image):
 * pixel indices, W*H of them.  Returns the count. */
size_t orc_seq_order(size_t width, size_t height, int32_t* out);
/* rd_riemersma_cpu.cpp:269-356 (BuildCurveIndex): block-mode order and owner. */
size_t orc_block_order(size_t width, size_t height, int32_t* out, int32_t* owner);

/* rd_octree.cpp:219-409 (ColorTree::Build). pixels: W*H*4 floats RGBA, Q16. */
int orc_tree_build(orc_tree* t, const float* pixels, size_t width, size_t height,
                   int max_colors, int associate_alpha, int grayscale);
void orc_tree_free(orc_tree* t);
/* rd_octree.cpp:178-217 + rd_riemersma_cpu.cpp:82-92: descent + ClosestColor. */
int orc_tree_lookup(const orc_tree* t, double r, double g, double b, double a);

/* rd_riemersma_cpu.cpp:359-417 (RiemersmaWalkCpu), curve == nullptr form.
 * pixels (W*H*4 floats) are dithered in place; idx_out (W*H bytes, may be NULL)
 * receives each visited pixel's palette index (the low 8 bits). */
void orc_walk_seq(const orc_tree* t, const orc_entry* palette, int count,
                  int associate_alpha, double diffusion, int use_cache,
                  size_t width, size_t height, float* pixels, uint8_t* idx_out);

/* rd_riemersma_cpu.cpp:477-805 (RiemersmaBlocksCpu), non-fused RgbaF path,
 * frames = 1.  Returns 0 on success, -1 for the two refusals (count > 256 or
 * block < 16).  idx_out (may be NULL) receives the index written to each pixel
 * by the owner scatter; pixels the curve never reaches are left untouched in
 * both buffers. */
int orc_walk_blocks(const orc_tree* t, const orc_entry* palette, int count,
                    int associate_alpha, double diffusion, int block,
                    size_t width, size_t height, float* pixels, uint8_t* idx_out);

/* The chosen index at every block-list position, in list order (the buffer
 * the reference's block engines dump as `.idx.bin`).  chosen_out holds
 * W*H+1 bytes; returns the list length or -1 for the refusals. */
int orc_block_chosen(const orc_tree* t, const orc_entry* palette, int count, int assoc,
                     double diffusion, int block, size_t width, size_t height,
                     const float* pixels, uint8_t* chosen_out);

/* Video frame formats (codes as the library's RDB_* formats: 3 RGB8, 4 RGBA8,
 * 16 RgbaF, 6 rgb48, 8 rgba64, 444 planar 4:4:4, 420 planar 4:2:0).
 * orc_widen_frame: src/rd_riemersma_cpu.cpp:496-516 (gather_pixel),
 * include/rd_types.h:75-97, and src/rd_blocks_cuda.cu:660-706 for 4:2:0.
 * orc_narrow_frame (formats 8 and 444): src/rd_riemersma_cpu.cpp:719-753.
 * Both return -1 on an unknown format. */
int orc_widen_frame(int format, const void* in, size_t width, size_t height, float* rgba);
int orc_narrow_frame(int format, const float* rgba, size_t width, size_t height, void* out);

/* src/rd_approx_cuda.cu:73-88 (BuildInverseFilter). g has taps+1 entries. */
void orc_inverse_filter(int taps, double diffusion, double* g);

#ifdef __cplusplus
}
#endif

#endif
