/*
 * rdb.h -- C ABI of the B200 Riemersma engines (librdb_b200.so).
 *
 * Plain pointers, sizes and POD structs only; no C++ or CUDA types cross this
 * boundary (streams travel as void*).  Every entry point returns 0 on success
 * or an RDB_E_* code; rdb_last_error() then gives a human-readable message
 * for the calling thread.  The reference's engine API (include/rd_riemersma.h
 * of rdither) reports errors as a std::string that is empty on success; the
 * C++ drop-in layer (stipple_b200/dropin/rd_b200_dropin.cpp) maps these codes
 * back to that form.
 *
 * Each declaration names the reference interface it stands in for.
 */
#ifndef RDB_H_
#define RDB_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RDB_OK 0
#define RDB_E_INVALID 1     /* bad argument */
#define RDB_E_CUDA 2        /* CUDA runtime error, or no usable device */
#define RDB_E_NOMEM 3       /* device allocation failed or budget exceeded */
#define RDB_E_UNSUPPORTED 4 /* refused by the engine's stated limits */
#define RDB_E_DEVICE 5      /* a kernel reported an error status */
#define RDB_E_TIMEOUT 6     /* a bounded wait expired */

/* Pixel layouts. */
#define RDB_RGB8 3     /* 3 bytes per pixel */
#define RDB_RGBA8 4    /* 4 bytes per pixel */
#define RDB_RGBAF32 16 /* 4 floats per pixel, ImageMagick Q16 range (RgbaF) */

/* Engines. */
#define RDB_ENGINE_SEQ 0    /* sequential-exact walk (RiemersmaWalkCpu / RiemersmaWalkCuda) */
#define RDB_ENGINE_BLOCKS 1 /* block-parallel walk (RiemersmaBlocksCpu / RiemersmaBlocksCuda) */
#define RDB_ENGINE_JACOBI 2 /* order-free approximation (RiemersmaApproxCuda) */

/* Message for the calling thread's last failing call ("" if none). */
const char* rdb_last_error(void);

/* ---- device ---------------------------------------------------------------
 * Replaces CudaAvailable() (include/rd_riemersma.h:284). */
int rdb_device_count(int* count);
/* Device name as "<name> (sm_XY)", the form RiemersmaWalkCuda reports. */
int rdb_device_name(int device, char* buf, size_t len);
/* Replaces CudaAllocPinned / CudaFreePinned (include/rd_riemersma.h:480-481). */
void* rdb_alloc_pinned(size_t bytes);
void rdb_free_pinned(void* p);
/* Whole frames of width x height that one host-buffer call of `engine` can
 * hold on `device` within min(free memory, vram_budget) (budget 0 = free
 * memory): staging plus the engine's scratch per frame, after the fixed
 * per-call tables; at most 4096.  Replaces CudaMaxFrames
 * (include/rd_riemersma.h:288), which sizes the reference's own buffers. */
int rdb_max_frames(int device, int engine, size_t width, size_t height, size_t vram_budget);

/* ---- palette building -----------------------------------------------------
 * Replaces rd::ColorTree::Build (include/rd_octree.h:62-63): ImageMagick's
 * octree classification, reduction to at most `max_colors` and colormap, on
 * the host.  `row_stride` is in bytes (0 = packed). */
typedef struct rdb_octree rdb_octree;
typedef struct rdb_context rdb_context;
int rdb_octree_build(const void* pixels, int layout, size_t width, size_t height,
                     size_t row_stride, int max_colors, int associate_alpha, int grayscale,
                     rdb_octree** out);
/* The same build of an image in DEVICE memory (ctx's device), its rows after
 * the build's first loop classified on the device: each run of equal pixels
 * adds to one node per level, contributions are computed in parallel and each
 * node's are added in the reference's row-major order by one thread, so every
 * node's error, count and totals -- the tree and the colormap -- are those of
 * rdb_octree_build.  The root's accumulated error, which decides nothing once
 * it exceeds every other node's, is summed in another order (checked; when it
 * does not exceed them the rows are classified on the host instead).  The
 * node array lists the live nodes in another order than rdb_octree_build's
 * (and without the pruned ones).  Synchronous on `stream`.  *device_rows (may
 * be NULL) receives how many rows the device classified. */
int rdb_octree_build_device(rdb_context* ctx, const void* pixels, int layout, size_t width,
                            size_t height, size_t row_stride, int max_colors, int associate_alpha,
                            int grayscale, void* stream, rdb_octree** out, int* device_rows);
int rdb_octree_color_count(const rdb_octree* t);
int rdb_octree_node_count(const rdb_octree* t);
int rdb_octree_depth(const rdb_octree* t);
/* count x 4 doubles (r, g, b, a) */
void rdb_octree_colormap(const rdb_octree* t, double* out);
/* node_count x 16 child ids, parent, colour number, unique-pixel count */
void rdb_octree_nodes(const rdb_octree* t, int32_t* child, int32_t* parent,
                      uint32_t* color_number, uint64_t* number_unique);
void rdb_octree_free(rdb_octree* t);
/* Palette files: rdither's --palette-export / --palette-from text form
 * (.txt or .text paths).  The writer is ImWritePalette's text branch
 * (src/rd_im.cpp:994-1030): a header, then per colour "index r g b a hex"
 * tab-separated, Q16 with six decimals.  The reader is ImReadPalette's
 * (:1175-1350): rows "index r g b [a] [hex]" (alpha read only when the hex
 * column follows), indices contiguous from 0 (a gap is refused), r, g, b
 * rounded through float, colours sorted by (r, g, b, a), and the tree built
 * from that one-row strip with as many colours as rows (no alpha association;
 * greyscale when every row is grey) -- refused if it merges any.  The tree's
 * colormap is then the palette; `associate_alpha` receives 1 when some row's
 * alpha is not opaque (the reference's palette flag).  `expect_colors` > 0
 * refuses a file with another count.  Other extensions return
 * RDB_E_UNSUPPORTED (the image form is rdb_palette_*_png). */
int rdb_palette_write_text(const double* colors /* count x 4 */, int count, const char* path);
int rdb_palette_read_text(const char* path, int expect_colors, rdb_octree** out,
                          int* associate_alpha);
/* The image form of the same files, as PNG.  The writer is ImWritePalette's
 * image branch (src/rd_im.cpp:1047-1118): a 1 x count strip of 8-bit colours,
 * each channel narrowed by ImageMagick's ScaleQuantumToChar, as an indexed PNG
 * (count <= 256).  The reader is ImReadPalette's image branch (:1362-1388)
 * with ImAdoptPaletteFromColormap (:731-888): an indexed PNG gives its PLTE
 * entries in order (alpha from tRNS), any other PNG its distinct RGB values in
 * scan order; 8-bit samples scale by 257 to Q16; `expect_colors` > 0 must
 * equal the colours the image holds; duplicates are dropped; the tree is
 * built from a swatch (8 x 8 per colour, ceil(sqrt(n)) per row) with as many
 * colours as entries, no alpha association, greyscale when every entry is
 * grey.  The tree's colormap is the palette. */
int rdb_palette_write_png(const double* colors /* count x 4 */, int count, const char* path);
int rdb_palette_read_png(const char* path, int expect_colors, rdb_octree** out);
/* 1 when every pixel has r == g == b (the reference's greyscale rule,
 * src/rd_cli.cpp:2452-2456). */
int rdb_is_grayscale(const void* pixels, int layout, size_t width, size_t height,
                     size_t row_stride);

/* ---- context -------------------------------------------------------------
 * Device state kept across calls: resident palettes, visit-order tables per
 * geometry, memo slabs and scratch.  The reference keeps comparable state in
 * its blocks engine's DeviceState slots (src/rd_blocks_cuda.cu:855-1002).
 * A context is used by one host thread at a time. */
/* memory_budget: bytes of device memory the context may hold (0 = 90 % of free). */
int rdb_context_create(int device, size_t memory_budget, rdb_context** out);
void rdb_context_destroy(rdb_context* ctx);
/* Device bytes currently held by the context. */
size_t rdb_context_bytes(const rdb_context* ctx);
/* Passes the last segmented sequential walk on this context took (0 before
 * any; 1 when every segment's speculation held on the first pass).  No
 * reference counterpart: the reference walks one chain. */
int rdb_context_last_passes(const rdb_context* ctx);
/* Sweeps the last block-sweep approximation (rdb_options.jacobi_form 0) ran on
 * this context, and whether its last sweep changed no block's end queue (so
 * its result is exactly the cache-free walk).  No reference counterpart. */
int rdb_context_last_sweeps(const rdb_context* ctx, int* converged);

/* Device-side counters of the segmented sequential walk, kept while profiling
 * is on (rdb_context_profile(ctx, 1) clears them).  Walk-kernel times are CUDA
 * events recorded on the launching stream around each walk launch.  No
 * reference counterpart. */
typedef struct rdb_kernel_stats {
  int64_t walk_launches;   /* segment-walk kernel launches */
  double walk_ms;          /* their summed device time */
  int64_t walk_positions;  /* positions those launches walked, warm-ups included */
  int64_t passes;          /* segmented-walk passes */
  int64_t launches;        /* kernels the context launched for the sequential engine */
  int64_t seg_len;         /* segment length of the last segmented walk */
  int64_t chains;          /* segments (concurrent chains) of the last segmented walk */
  int block_threads;       /* launch shape of the last block walk: threads per CTA ... */
  int block_min_ctas;      /* ... and the CTAs per SM it was compiled for (the tuner's pick) */
  double octree_ms[4];     /* device palette builds (rdb_octree_build_device and the server's):
                              host first loop, device classification with its transfers,
                              host absorb, host reduction and colormap; summed, wall clock */
} rdb_kernel_stats;
int rdb_context_profile(rdb_context* ctx, int enable);
/* The block engine's index dump, the reference's `<prefix>.idx.bin`
 * (src/rd_opencl.cpp:2137-2147, written when RD_OCL_DUMP names a prefix):
 * while `prefix` is set, every block-engine call of the context (rdb_dither
 * with RDB_ENGINE_BLOCKS, rdb_dither_frames*) writes `<prefix>.idx.bin`, the
 * palette index chosen at every position of every image's block-mode list
 * (src/rd_riemersma_cpu.cpp:269-356), one byte each, in list order, images in
 * call order, replacing the file of the previous call.  The call then waits
 * for the device.  NULL or "" turns it off. */
int rdb_context_dump_indices(rdb_context* ctx, const char* prefix);
int rdb_context_stats(const rdb_context* ctx, rdb_kernel_stats* out);

/* Dependent latency in SM cycles of each operation on the sequential walk's
 * per-step chain, measured on `device` by one thread timing chains of
 * dependent operations with clock64().  A diagnostic for the chain-latency
 * roofline; no reference counterpart. */
typedef struct rdb_latency_table {
  double dadd;            /* __dadd_rn */
  double dmul;            /* __dmul_rn */
  double f64_to_f32;      /* half of a double -> float -> double round trip */
  double f32_to_f64;
  double f32_to_int;      /* float -> int (truncating) */
  double shared_load;     /* shared-memory pointer chase */
  double global_load_l1;  /* global pointer chase hitting L1 */
  double global_load_l2;  /* global pointer chase hitting L2 (L1 bypassed) */
  double int_op;          /* integer add / xor */
} rdb_latency_table;
int rdb_probe_latency(int device, rdb_latency_table* out);

/* A palette and its colour tree, in the reference's own terms
 * (rd::Palette, include/rd_riemersma.h:63-67; rd::QNode, include/rd_octree.h:43-52). */
typedef struct rdb_palette_desc {
  int count;                      /* palette entries, 1..256 */
  int associate_alpha;
  const double* colors;           /* count x 4 (palette.entries) */
  const double* search_colors;    /* count x 4 (tree colormap); NULL = colors */
  int node_count;
  int root;
  const int32_t* child;           /* node_count x 16, -1 = none */
  const int32_t* parent;          /* node_count, may be NULL */
  const uint32_t* color_number;   /* node_count */
  const uint64_t* number_unique;  /* node_count */
} rdb_palette_desc;

int rdb_palette_create(rdb_context* ctx, const rdb_palette_desc* desc, int* palette_id);
/* The device plan blob for a palette, built on the host (no device needed):
 * header, palette tables, live child table, per-node search runs and the
 * post-order slot map (layout in stipple_b200/csrc/rdb_plan.h).  Writes at
 * most `cap` bytes and the full size to *size. */
int rdb_plan_build(const rdb_palette_desc* desc, void* out, size_t cap, size_t* size);
int rdb_palette_from_octree(rdb_context* ctx, const rdb_octree* t, int* palette_id);
/* Every stream other than the context's own on which the palette was used
 * must be synchronised first (the context's stream is drained here); the
 * palette's device blocks return to the context's pool. */
int rdb_palette_destroy(rdb_context* ctx, int palette_id);
/* The palette's uniform-key table (stipple_b200/csrc/rdb_uniform.h) copied to
 * host memory: one byte per 6-bit-per-channel memo key, holding the colour
 * number every target with that key receives, or 255 when the search result
 * can vary inside the key (or is colour 255).  2^18 bytes; 2^24 for a palette
 * that associates alpha (254 is then never a uniform colour either).  No
 * reference counterpart: it is how the sequential engines skip the memo for
 * such keys. */
int rdb_palette_uniform(rdb_context* ctx, int palette_id, uint8_t* out, size_t cap);

/* ---- dithering -----------------------------------------------------------
 * One image.  Device pointers. */
typedef struct rdb_job {
  const void* pixels;   /* device, row-major, `layout` */
  size_t row_stride;    /* bytes between rows (0 = packed) */
  int width;
  int height;
  int layout;
  int palette_id;
  uint8_t* indices;     /* device, width*height bytes: palette index per pixel */
  float* rgba_out;      /* optional device RgbaF result (width*height*4 floats); may equal
                           `pixels` for RDB_RGBAF32 (in place, as the reference works) */
} rdb_job;

typedef struct rdb_options {
  double diffusion;     /* dither:diffusion-amount, default 1.0 (DitherParams::diffusion) */
  int use_cache;        /* sequential engine: ImageMagick's memo table, default 1 */
  int block;            /* blocks engine: positions per block, >= 16, default 512 */
  int jacobi_iters;     /* default 20 (ApproxOptions::iterations) */
  int jacobi_taps;      /* default 96 (ApproxOptions::taps), 1..4096 */
  int jacobi_fp64;      /* default 0 (ApproxOptions::fp64) */
  int cache_bits;       /* sequential engine: log2 shared-memory memo cache entries, 0 = auto */
  int seq_mode;         /* sequential engine: 0 = auto, 1 = one warp walks each image whole,
                           2 = speculative segmented walk on warps (exact; rdb_ssw.h),
                           3 = the same on thread walkers (exact; rdb_tsw.h; its forms:
                           walk_form).  Auto: images under 8192 pixels mode 1, others 3.
                           Mode 2 and the host-checked loop of mode 3 (loop_mode 1) wait
                           for the stream between passes. */
  int seg_len;          /* segmented walk: positions per segment, 0 = auto */
  int warm_len;         /* segmented walk: warm-up positions before each segment, 0 = auto */
  int max_passes;       /* segmented walk: give up after this many passes (0 = no limit); the
                           walk then reports RDB_E_DEVICE -- never an inexact result */
  int loop_mode;        /* segmented thread walk: 0 = automatic (the device-side loop below
                           unless the context is profiling), 1 = the host checks each pass,
                           2 = the device-side loop: one CUDA graph whose while-conditional
                           node repeats the passes until a control kernel sees convergence,
                           so the call returns without waiting for the device (errors then
                           surface at rdb_synchronize) */
  int jacobi_form;      /* approximation engine (RDB_ENGINE_JACOBI): 0 = block sweeps (default):
                           the block-mode list cut into blocks of 256 positions, every block
                           walked in parallel, cache-free, each starting from its
                           predecessor's end queue of the previous sweep (zeros in the first),
                           up to jacobi_iters sweeps and stopping at the first sweep in which
                           no block's end queue changed -- from then on the result is exactly
                           the cache-free walk along the block-mode list (the reference's walk
                           with its memo table off); 1 = the point iteration with the
                           truncated inverse filter (jacobi_taps, jacobi_fp64), as the
                           reference's approx engine */
  int seg_window;       /* segmented thread walk: segments walked per pass beyond the verified
                           front (-1 = every unverified segment each pass).  One image: that
                           many (0 = as many as the device holds resident at once, less one
                           CTA's 128, so the pass stays one wave).  Several:
                           that many in total (0 = twice the resident segments), shared among
                           the images after every pass in proportion to the segments each has
                           left, at least 256 each. */
  int walk_form;        /* segmented thread walk: 1 = paired warps: per 32 segments a chain warp
                           runs each step's dependent chain and a sum warp keeps the running
                           sums of the pending pixels, handing each over through shared memory
                           (a shorter step, fewer segments resident); 2 = one thread per
                           segment doing both (more segments resident); 0 = automatic: paired
                           for one image without alpha, whose walk is latency-bound, one
                           thread per segment for several (throughput-bound) and for alpha
                           palettes (whose paired form fits one CTA per SM).  Same results. */
} rdb_options;

void rdb_options_default(rdb_options* o);

/* Dithers `n_jobs` images with one engine on `stream` (cudaStream_t, NULL =
 * the context's stream).  The sequential engine runs every job as its own
 * exact walk inside one persistent launch (a warp per image, longest first);
 * with n_jobs == 1 it is the plain one-image-per-launch form.  The blocks
 * engine requires one palette and one layout across the jobs.  Asynchronous:
 * the call returns after enqueueing; rdb_synchronize() waits and reports any
 * kernel status.
 *
 * Replaces RiemersmaWalkCuda (include/rd_riemersma.h:214-217),
 * RiemersmaBlocksCuda (:450-464) and RiemersmaApproxCuda (:303-307) at the
 * device-buffer level. */
int rdb_dither(rdb_context* ctx, int engine, const rdb_job* jobs, int n_jobs,
               const rdb_options* opts, void* stream);
int rdb_synchronize(rdb_context* ctx, void* stream);

/* Host-buffer form: copies `pixels` (host) to the device, dithers, and copies
 * the index map (and RgbaF result when rgba_out != NULL) back.  Pinned
 * buffers make the copies asynchronous DMA.  Synchronous. */
typedef struct rdb_host_job {
  const void* pixels;
  size_t row_stride;
  int width;
  int height;
  int layout;
  int palette_id;
  uint8_t* indices;     /* host, width*height */
  float* rgba_out;      /* optional host RgbaF result */
} rdb_host_job;

int rdb_dither_host(rdb_context* ctx, int engine, const rdb_host_job* jobs, int n_jobs,
                    const rdb_options* opts);

/* ---- video frames through the blocks engine ------------------------------
 * A batch of equal-size frames in the decoder's own format, dithered by the
 * blocks engine and written in the encoder's own format: the input is widened
 * to Q16 floats per visit and the output narrowed per pixel inside the
 * engine's gather and scatter, so no RgbaF frame exists on either side.
 * Replaces RiemersmaBlocksCuda's upload_u16 / in_mode / emit_u16 /
 * emit_yuv444 forms (include/rd_riemersma.h:325-464) and RiemersmaBlocksCpu's
 * gather_raw / raw_out arguments (:224-268), byte for byte with the latter:
 *   in   RGB16 / RGBA16   each uint16 widened as a float; alpha 65535 if absent
 *        YUV444P8         swscale's 8-bit YCbCr -> 16-bit RGB (rd_types.h:75-97)
 *        YUV420P8         chroma upsampled 2x bilinearly first
 *                         (src/rd_blocks_cuda.cu:660-706); even sizes only
 *        RGB8 / RGBA8 / RGBAF32 as for rdb_dither
 *   out  RGBA16           uint16 of the colour's Q16 float; alpha from the
 *                         palette when it associates alpha, else the source's
 *        YUV444P8         BT.601 limited range of the colour's top 8 bits
 *        RGBAF32          the rdb_dither result (may equal `in` for RGBAF32 in)
 * The cell the block list never visits takes its source value in the output
 * format (src/rd_riemersma_cpu.cpp:755-801).  Frames are packed: planar
 * formats hold Y, Cb, Cr planes of width*height bytes (4:4:4) or width*height
 * and two of width*height/4 (4:2:0) per frame. */
#define RDB_RGB16 6      /* rgb48le, 3 uint16 per pixel (frames only) */
#define RDB_RGBA16 8     /* rgba64le, 4 uint16 per pixel (frames only) */
#define RDB_YUV444P8 444 /* planar 8-bit YCbCr 4:4:4 (frames only) */
#define RDB_YUV420P8 420 /* planar 8-bit YCbCr 4:2:0, input only (frames only) */

typedef struct rdb_frames {
  const void* in;          /* `frames` frames, in_frame_bytes apart */
  size_t in_frame_bytes;   /* 0 = packed (rdb_frame_bytes) */
  int in_format;
  int width;
  int height;
  int frames;
  int palette_id;          /* at most 256 colours (one index byte per pixel) */
  int out_format;          /* RDB_RGBA16, RDB_YUV444P8 or RDB_RGBAF32 */
  void* out;               /* `frames` frames, out_frame_bytes apart */
  size_t out_frame_bytes;  /* 0 = packed */
  uint8_t* indices;        /* optional index map, width*height per frame */
} rdb_frames;

/* Bytes of one packed frame of `format`, or 0 for an unknown format. */
size_t rdb_frame_bytes(int format, int width, int height);

/* Device buffers; asynchronous on `stream` like rdb_dither. */
int rdb_dither_frames(rdb_context* ctx, const rdb_frames* f, const rdb_options* opts,
                      void* stream);
/* Host buffers: uploads `in`, dithers, downloads `out` (and `indices`).
 * Synchronous. */
int rdb_dither_frames_host(rdb_context* ctx, const rdb_frames* f, const rdb_options* opts);

/* ---- serving ----------------------------------------------------------------
 * A request loop over one device: requests of mixed sizes, palettes and
 * engines are submitted from any thread; host threads build each request's
 * palette (the library's octree, rdb_octree_build); requests are admitted
 * while the device-memory bound of everything in flight, plus the buffers
 * the workers' contexts keep between batches, stays within `memory_budget`
 * (a context keeps at most an equal share of it; when a request cannot be
 * admitted, idle contexts release theirs); idle device workers (each its own
 * context and stream, held during a batch to what it had plus the batch's
 * bound)
 * take every admitted request of one engine and one option set as one batch,
 * so requests that arrive while others are on the device join the next
 * batch and batches on different workers overlap.  Results are bit-identical
 * to the same request alone.  No reference counterpart: rdither dithers one
 * job per call. */
typedef struct rdb_server rdb_server;

typedef struct rdb_server_options {
  int device;
  size_t memory_budget;   /* admission cap in bytes (0 = 90 % of free memory) */
  int workers;            /* device workers (0 = 4) */
  int max_batch;          /* requests per batch (0 = 512) */
  int host_threads;       /* palette builders on the host (0 = the CPUs this process may run
                             on: its affinity mask, capped by a cgroup CPU quota) */
  int device_palettes;    /* 0 (default): host threads build each request's palette
                             (rdb_octree_build) before admission, many at once; 1: each device
                             worker builds its batch's palettes on the device from the uploaded
                             pixels (rdb_octree_build_device), one after another -- faster per
                             build for RGB at 256 colours, slower with alpha, and serialised on
                             the workers, so a mixed stream is served far slower */
} rdb_server_options;

typedef struct rdb_request {
  const void* pixels;     /* host, row-major, `layout`; must stay valid until completion */
  size_t row_stride;      /* bytes (0 = packed) */
  int width;
  int height;
  int layout;
  int colors;             /* palette size requested from the octree */
  int associate_alpha;    /* palette associates alpha (RGBA input only) */
  int engine;             /* RDB_ENGINE_* */
  rdb_options options;
  uint8_t* indices;       /* host, width*height */
  float* rgba_out;        /* optional host RgbaF result */
} rdb_request;

typedef struct rdb_request_result {
  int status;             /* RDB_OK or the failing call's code */
  double queue_ms;        /* submit -> palette built */
  double admit_ms;        /* palette built -> on the device */
  double device_ms;       /* batch call (uploads, walk, downloads) */
  double total_ms;        /* submit -> result in host memory */
  int batch_size;         /* requests in its batch */
} rdb_request_result;

/* Stages of a request's latency, in order (rdb_server_stats.stage_*). */
enum {
  RDB_STAGE_BUILD_WAIT = 0, /* submit -> a palette builder takes it */
  RDB_STAGE_BUILD = 1,      /* octree build on the host */
  RDB_STAGE_ADMIT = 2,      /* built -> a device worker starts its batch (memory admission,
                               free worker) */
  RDB_STAGE_DEVICE = 3,     /* the batch call: palette upload, H2D, walk, D2H */
  RDB_STAGE_TOTAL = 4,      /* submit -> result in host memory */
  RDB_STAGES = 5
};

typedef struct rdb_server_stats {
  int64_t completed;
  int64_t failed;
  int64_t pixels;
  int64_t batches;
  double p50_ms;          /* total latency percentiles over completed requests */
  double p99_ms;
  double max_ms;
  double mpx_per_s;       /* pixels / (last completion - first submission) */
  size_t peak_admitted_bytes; /* most bytes counted against the budget at once
                                 (admitted requests plus idle contexts' buffers) */
  double stage_p50_ms[RDB_STAGES]; /* per-stage percentiles (RDB_STAGE_*) */
  double stage_p99_ms[RDB_STAGES];
  int host_threads;       /* palette builders running */
  int workers;            /* device workers running */
} rdb_server_stats;

int rdb_server_create(const rdb_server_options* opts, rdb_server** out);
/* Device bytes the server counts for `req` while it is admitted (its staging,
 * visit order, palette tables, the scratch of the engine path it takes and,
 * with device_palettes, its palette build's scratch): a request whose bytes
 * exceed the server's budget is refused at submission.  Reads the pixels
 * only to classify greyscale for a device palette build. */
size_t rdb_request_bytes(const rdb_request* req, int device_palettes);

/* Non-blocking; the request (and its buffers) must outlive its completion. */
int rdb_server_submit(rdb_server* s, const rdb_request* req, uint64_t* ticket);
/* Waits up to timeout_ms (< 0 = forever) for one request; RDB_E_TIMEOUT when
 * it is not done yet.  The ticket is released once waited for successfully. */
int rdb_server_wait(rdb_server* s, uint64_t ticket, int timeout_ms, rdb_request_result* out);
int rdb_server_stats_get(rdb_server* s, rdb_server_stats* out);
/* Forgets the statistics gathered so far (latencies, counts, throughput span,
 * peak admission), e.g. after a warm-up stream; requests in flight count
 * toward the new window when they complete. */
int rdb_server_stats_reset(rdb_server* s);
/* Finishes everything submitted, then stops the threads. */
void rdb_server_destroy(rdb_server* s);

/* Sequential-exact walk of one image without allocating any device memory.
 * This entry point has no counterpart in the reference.
 *
 * It is for callers that cannot call cudaMalloc: code running where a host
 * framework owns every device allocation (a plugin inside an application with
 * its own pooling allocator, which must not have memory taken behind its back),
 * code on a latency-critical path where cudaMalloc's implicit device
 * synchronisation is not acceptable, and code that must not fail halfway for
 * lack of memory.  The caller passes the palette plan (host memory, made by
 * rdb_plan_build), the pixels and the index map (device memory); everything
 * else -- memo table, visit order, curve scratch, palette copy, launch
 * descriptor -- lives in one fixed 5 MiB array in device memory that the
 * library declares statically, so every GPU that loads the library holds it
 * until the process exits.
 *
 * Limits: at most 4096 pixels per side and 1048576 pixels, palettes without
 * associated alpha (an alpha memo has 2^24 keys), plan blob <= 64 KiB; larger
 * inputs are refused with RDB_E_UNSUPPORTED and a message.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) and keeps
 * it for the life of the process, so make that first call before any stream
 * capture on the device, and do not use this entry point on a device after
 * cudaDeviceReset (the address it kept is then stale).  The work is enqueued on
 * `stream` (NULL = legacy default stream); device-side status is not reported.
 * `plan` is copied on `stream`: keep it valid and unchanged until the stream
 * reaches the call (from pinned memory that copy is asynchronous).  All calls share the one array and it keeps the last call's
 * contents (the memo table is told apart by a generation counter, the work
 * counter is cleared each call), so calls that overlap on the GPU -- on
 * different streams, or from different threads -- race and corrupt each
 * other's results: serialise them. */
int rdb_dither_seq_noalloc(const void* plan, size_t plan_bytes, const void* pixels,
                           size_t row_stride, int width, int height, int layout,
                           uint8_t* indices, double diffusion, int use_cache, void* stream);

/* Error weights 16^(-i/15) by ImageMagick's recurrence (rd_types.h:169-176)
 * and the Jacobi inverse filter (src/rd_approx_cuda.cu:73-88, exposed by the
 * reference as ApproxInverseFilter). */
void rdb_error_weights(double out[16]);
int rdb_inverse_filter(int taps, double diffusion, double* out /* taps+1 */);

/* The block-mode gap: pixel index of the one cell the block list never
 * visits, or -1 when it lies outside the image (src/rd_riemersma_cpu.cpp:439-455). */
int64_t rdb_block_gap(int width, int height);

#ifdef __cplusplus
}
#endif

#endif /* RDB_H_ */
