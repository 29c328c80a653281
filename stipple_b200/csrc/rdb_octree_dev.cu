// rdb_octree_dev.cu -- the second classification loop of the octree build on
// the device (rdb_octree_build_device in include/rdb.h).
//
// ColorTree::Build (src/rd_octree.cpp:219-409) classifies the image row by
// row.  After its first loop (a few rows at full depth, run on the host by
// Octree::Begin) every remaining row is classified to a fixed depth L, and
// each run of equal pixels within a row visits exactly one node per level
// 1..L, adding weight * sqrt(dist) to that node's error and, at level L, its
// pixel count and colour totals to that leaf.  What a run adds depends only on
// the run (its colour and length), so every contribution is computed in
// parallel; the sums are floating-point and order-dependent, so each node's
// contributions are then added in the reference's order -- row-major run order
// -- by one warp per node, starting from the node's value after the first
// loop:
//   1. runs: a pixel starts a run when it differs from its left neighbour (or
//      starts its row); a scan numbers the runs in row-major order;
//   2. per run and level: the node's path key (NodeKey) and the contribution;
//      per run: its leaf key;
//   3. a stable radix sort by key groups each node's contributions in run
//      order (stable sorts keep the input order within a key);
//   4. one warp per node adds them in that order (its lanes load 32 at a
//      time); one warp per leaf adds the run totals in order.
// Integer counts are exact in any order.  The root's error, which the
// reference accumulates across every visit, is summed in another order: its
// exact bits decide nothing once it exceeds every other node's error (see
// Octree::Absorb, which checks that and otherwise hands the rows back to the
// host loop).
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include "rdb_numeric.h"
#include "rdb_octree_dev.h"

namespace rdb {
namespace {

__device__ __forceinline__ float4 pixel_at(const OctreeRowsLaunch& L, int64_t i) {
  const int64_t y = L.y0 + i / L.width;
  const int64_t x = i % L.width;
  const unsigned char* row = L.pixels + y * L.row_stride;
  if (L.layout == 16) return reinterpret_cast<const float4*>(row)[x];
  const unsigned char* q = row + static_cast<int64_t>(L.layout) * x;
  return make_float4(static_cast<float>(q[0]) * 257.0f, static_cast<float>(q[1]) * 257.0f,
                     static_cast<float>(q[2]) * 257.0f,
                     L.layout == 4 ? static_cast<float>(q[3]) * 257.0f : 65535.0f);
}

__device__ __forceinline__ bool same(float4 a, float4 b) {
  return a.x == b.x && a.y == b.y && a.z == b.z && a.w == b.w;
}

// rd_types.h:179-192 (AssociateAlphaPixel) on a float sample.
__device__ __forceinline__ void associate(bool assoc, float4 s, double (&o)[4]) {
  o[3] = static_cast<double>(s.w);
  if (!assoc || s.w == 65535.0f) {
    o[0] = s.x;
    o[1] = s.y;
    o[2] = s.z;
    return;
  }
  const double alpha = __dmul_rn(kQuantumScale, static_cast<double>(s.w));
  o[0] = __dmul_rn(alpha, static_cast<double>(s.x));
  o[1] = __dmul_rn(alpha, static_cast<double>(s.y));
  o[2] = __dmul_rn(alpha, static_cast<double>(s.z));
}

__global__ void RunStarts(OctreeRowsLaunch L, int* flag) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= L.pixels_n) return;
  flag[i] = (i % L.width == 0 || !same(pixel_at(L, i), pixel_at(L, i - 1))) ? 1 : 0;
}

// run id -> its first pixel (flag scanned exclusively: id of a starting pixel)
__global__ void RunFirst(OctreeRowsLaunch L, const int* flag, const int* id, int* first) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= L.pixels_n) return;
  if (flag[i]) first[id[i]] = static_cast<int>(i);
}

// Per run: the node key and error contribution at every level (element
// r * levels + level - 1), and the leaf key.  Follows Classify's arithmetic
// (src/rd_octree.cpp:305-362) operation for operation.
__global__ void RunContrib(OctreeRowsLaunch L, const int* first, int runs, uint64_t* keys,
                           double* vals, uint64_t* leaf_keys, int* leaf_runs) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= runs) return;
  const int64_t p = first[r];
  const int64_t next = r + 1 < runs ? first[r + 1] : L.pixels_n;
  // A run ends at its row's end too: the next run starts the next row there.
  const double weight = static_cast<double>(next - p);
  double px[4];
  associate(L.assoc != 0, pixel_at(L, p), px);
  unsigned byte[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) byte[c] = scale_char(clamp_pixel(px[c]));
  double half = (kQuantumRange + 1.0) / 2.0;
  const double midpoint = kQuantumRange / 2.0;
  double mid[4] = {midpoint, midpoint, midpoint, midpoint};
  int bit = kMaxTreeDepth - 1;
  const int bits = L.assoc ? 4 : 3;
  uint32_t path = 0;
  for (int level = 1; level <= L.levels; ++level, --bit) {
    half = __dmul_rn(half, 0.5);
    unsigned id = ((byte[0] >> bit) & 1u) | (((byte[1] >> bit) & 1u) << 1) | (((byte[2] >> bit) & 1u) << 2);
    if (L.assoc) id |= ((byte[3] >> bit) & 1u) << 3;
    mid[0] = __dadd_rn(mid[0], (id & 1u) ? half : -half);
    mid[1] = __dadd_rn(mid[1], (id & 2u) ? half : -half);
    mid[2] = __dadd_rn(mid[2], (id & 4u) ? half : -half);
    mid[3] = __dadd_rn(mid[3], (id & 8u) ? half : -half);
    path = (path << bits) | id;
    const double e0 = __dmul_rn(kQuantumScale, __dadd_rn(px[0], -mid[0]));
    const double e1 = __dmul_rn(kQuantumScale, __dadd_rn(px[1], -mid[1]));
    const double e2 = __dmul_rn(kQuantumScale, __dadd_rn(px[2], -mid[2]));
    const double e3 = L.assoc ? __dmul_rn(kQuantumScale, __dadd_rn(px[3], -mid[3])) : 0.0;
    double dist = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(e0, e0), __dmul_rn(e1, e1)), __dmul_rn(e2, e2)),
                            __dmul_rn(e3, e3));
    if (isnan(dist)) dist = 0.0;
    const int64_t at = static_cast<int64_t>(r) * L.levels + level - 1;
    keys[at] = (static_cast<uint64_t>(level) << 32) | path;
    vals[at] = __dmul_rn(weight, __dsqrt_rn(dist));
  }
  leaf_keys[r] = (static_cast<uint64_t>(L.levels) << 32) | path;
  leaf_runs[r] = r;
}

__device__ __forceinline__ int find_key(const uint64_t* keys, int n, uint64_t k) {
  int lo = 0, hi = n - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    if (keys[mid] < k) lo = mid + 1; else if (keys[mid] > k) hi = mid - 1; else return mid;
  }
  return -1;
}

// One warp per node: its error from the first loop's value, then every
// contribution in run order; and the sum of its running values (what the root
// gains from it).  The 32 lanes load 32 contributions at a time into shared
// memory (the next 32 in flight meanwhile) and lane 0 adds them one by one in
// order, so the sums are the sequential ones bit for bit while the loads run
// in parallel -- a node can hold millions of contributions.
__global__ void NodeSums(const OctreeRowsLaunch L, const uint64_t* ukeys, const int* offset,
                         const int* count, const int* nseg, const double* vals, double* qerr,
                         double* gain) {
  __shared__ double buf[8][32];
  const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  if (s >= *nseg) return;
  const int at = find_key(L.init_keys, L.init_n, ukeys[s]);
  double acc = at >= 0 ? L.init_qerr[at] : 0.0;
  double g = 0.0;
  const double* v = vals + offset[s];
  const int n = count[s];
  double next = lane < n ? v[lane] : 0.0;
  for (int base = 0; base < n; base += 32) {
    buf[w][lane] = next;
    __syncwarp();
    next = base + 32 + lane < n ? v[base + 32 + lane] : 0.0;
    if (lane == 0) {
      const int m = min(32, n - base);
      for (int j = 0; j < m; ++j) {
        acc = __dadd_rn(acc, buf[w][j]);
        g = __dadd_rn(g, acc);
      }
    }
    __syncwarp();
  }
  if (lane == 0) {
    qerr[s] = acc;
    gain[s] = g;
  }
}

// One warp per leaf: count and totals, runs in order (rd_octree.cpp:355-359).
// Each lane forms one run's four weighted terms into shared memory; lanes 0..3
// then add channel 0..3 in run order, 32 runs at a time.
__global__ void LeafSums(const OctreeRowsLaunch L, const uint64_t* ukeys, const int* offset,
                         const int* count, const int* nseg, const int* runs_sorted,
                         const int* first, int runs, uint64_t* number, double* totals) {
  __shared__ double buf[8][32][4];
  const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  if (s >= *nseg) return;
  const int at = find_key(L.init_keys, L.init_n, ukeys[s]);
  unsigned long long num = at >= 0 ? L.init_count[at] : 0;
  double t = 0.0;  // lane c < 4: channel c's total
  if (at >= 0 && lane < 4) t = L.init_total[4 * at + lane];
  const int n = count[s];
  const int* rs = runs_sorted + offset[s];
  int r_next = lane < n ? rs[lane] : 0;
  for (int base = 0; base < n; base += 32) {
    const int r = r_next;
    r_next = base + 32 + lane < n ? rs[base + 32 + lane] : 0;
    unsigned long long run_len = 0;
    double term[4] = {0.0, 0.0, 0.0, 0.0};
    if (base + lane < n) {
      const int64_t p = first[r];
      const int64_t next = r + 1 < runs ? first[r + 1] : L.pixels_n;
      double px[4];
      associate(L.assoc != 0, pixel_at(L, p), px);
      const double wgt = __dmul_rn(static_cast<double>(next - p), kQuantumScale);
      run_len = static_cast<unsigned long long>(next - p);
      term[0] = __dmul_rn(wgt, static_cast<double>(clamp_pixel(px[0])));
      term[1] = __dmul_rn(wgt, static_cast<double>(clamp_pixel(px[1])));
      term[2] = __dmul_rn(wgt, static_cast<double>(clamp_pixel(px[2])));
      term[3] = __dmul_rn(wgt, static_cast<double>(clamp_pixel(L.assoc ? px[3] : kOpaqueAlpha)));
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) buf[w][lane][c] = term[c];
    // A run lies within one row, so 32 of them sum below 2^32.
    num += __reduce_add_sync(0xffffffffu, static_cast<unsigned>(run_len));
    __syncwarp();
    if (lane < 4) {
      const int m = min(32, n - base);
      for (int j = 0; j < m; ++j) t = __dadd_rn(t, buf[w][j][lane]);
    }
    __syncwarp();
  }
  if (lane == 0) number[s] = num;
  if (lane < 4) totals[4 * s + lane] = t;
}

unsigned Blocks(int64_t n, int t) { return static_cast<unsigned>((n + t - 1) / t); }

// CUB's temporary storage for the largest call of a launch of P pixels.
std::size_t OctreeRowsTemp(int64_t P, int levels) {
  const int E = static_cast<int>(P * levels);
  std::size_t most = 0, need = 0;
  cub::DoubleBuffer<uint64_t> k(nullptr, nullptr);
  cub::DoubleBuffer<double> v(nullptr, nullptr);
  cub::DoubleBuffer<int> r(nullptr, nullptr);
  cub::DeviceRadixSort::SortPairs(nullptr, need, k, v, E, 0, 36);
  most = std::max(most, need);
  cub::DeviceRadixSort::SortPairs(nullptr, need, k, r, static_cast<int>(P), 0, 36);
  most = std::max(most, need);
  cub::DeviceScan::ExclusiveSum(nullptr, need, static_cast<int*>(nullptr), static_cast<int*>(nullptr), E);
  most = std::max(most, need);
  cub::DeviceRunLengthEncode::Encode(nullptr, need, static_cast<uint64_t*>(nullptr),
                                     static_cast<uint64_t*>(nullptr), static_cast<int*>(nullptr),
                                     static_cast<int*>(nullptr), E);
  most = std::max(most, need);
  return most;
}

// Bounds on the distinct keys of a launch: nodes of levels 1..levels (and
// leaves at the last level) of a tree of the given fan-out, at most one per
// element.
int64_t NodeBound(int64_t elements, int levels, int fan) {
  int64_t total = 0, at = 1;
  for (int l = 1; l <= levels && total < elements; ++l) {
    at = at > elements ? at : at * fan;
    total += at;
  }
  return total < elements ? total : elements;
}
int64_t LeafBound(int64_t runs, int levels, int fan) {
  int64_t at = 1;
  for (int l = 1; l <= levels && at < runs; ++l) at *= fan;
  return at < runs ? at : runs;
}

}  // namespace

std::size_t OctreeRowsScratch(int64_t pixels, int levels, bool assoc) {
  const int fan = assoc ? 16 : 8;
  const std::size_t P = static_cast<std::size_t>(pixels);
  const std::size_t E = P * static_cast<std::size_t>(levels);
  const std::size_t U = static_cast<std::size_t>(NodeBound(static_cast<int64_t>(E), levels, fan));
  const std::size_t UL = static_cast<std::size_t>(LeafBound(pixels, levels, fan));
  // flag, id, first (int, P); keys x2, vals x2 (E); leaf keys x2, leaf runs x2
  // (P); unique keys, counts, offsets, errors, gains (U); leaf keys, counts,
  // offsets, numbers, totals (UL); CUB temp; alignment slack.
  return 3 * P * 4 + 4 * E * 8 + 2 * P * 8 + 2 * P * 4 + U * (8 + 4 + 4 + 8 + 8) +
         UL * (8 + 4 + 4 + 8 + 32) + OctreeRowsTemp(pixels, levels) + 64 * 256;
}

cudaError_t ClassifyRowsDevice(const OctreeRowsLaunch& L, void* scratch, std::size_t scratch_bytes,
                               cudaStream_t s, OctreeRows* out) {
  const int64_t P = L.pixels_n;
  if (P <= 0) return cudaSuccess;
  const int64_t E0 = P * L.levels;
  unsigned char* base = static_cast<unsigned char*>(scratch);
  std::size_t used = 0;
  auto take = [&](std::size_t bytes) -> void* {
    used = (used + 255) & ~static_cast<std::size_t>(255);
    void* p = base + used;
    used += bytes;
    return p;
  };
  int* flag = static_cast<int*>(take(P * 4));
  int* id = static_cast<int*>(take(P * 4));
  int* first = static_cast<int*>(take(P * 4));
  uint64_t* keys = static_cast<uint64_t*>(take(E0 * 8));
  uint64_t* keys2 = static_cast<uint64_t*>(take(E0 * 8));
  double* vals = static_cast<double*>(take(E0 * 8));
  double* vals2 = static_cast<double*>(take(E0 * 8));
  uint64_t* lkeys = static_cast<uint64_t*>(take(P * 8));
  uint64_t* lkeys2 = static_cast<uint64_t*>(take(P * 8));
  int* lruns = static_cast<int*>(take(P * 4));
  int* lruns2 = static_cast<int*>(take(P * 4));
  const int fan = L.assoc ? 16 : 8;
  const int64_t U = NodeBound(E0, L.levels, fan);
  const int64_t UL = LeafBound(P, L.levels, fan);
  uint64_t* ukeys = static_cast<uint64_t*>(take(U * 8));
  int* ucount = static_cast<int*>(take(U * 4));
  int* uoff = static_cast<int*>(take(U * 4));
  double* qerr = static_cast<double*>(take(U * 8));
  double* gain = static_cast<double*>(take(U * 8));
  uint64_t* lukeys = static_cast<uint64_t*>(take(UL * 8));
  int* lcount = static_cast<int*>(take(UL * 4));
  int* loff = static_cast<int*>(take(UL * 4));
  uint64_t* lnum = static_cast<uint64_t*>(take(UL * 8));
  double* ltot = static_cast<double*>(take(UL * 32));
  int* nseg = static_cast<int*>(take(2 * sizeof(int)));
  void* temp = take(0);
  if (used > scratch_bytes) return cudaErrorMemoryAllocation;
  const std::size_t temp_bytes = scratch_bytes - used;
  // Every CUB call below needs at most OctreeRowsTemp(P, levels) bytes.
  if (temp_bytes < OctreeRowsTemp(P, L.levels)) return cudaErrorMemoryAllocation;

  cudaError_t e;
  RunStarts<<<Blocks(P, 256), 256, 0, s>>>(L, flag);
  std::size_t need = temp_bytes;
  if ((e = cub::DeviceScan::ExclusiveSum(temp, need, flag, id, static_cast<int>(P), s)) != cudaSuccess) return e;
  RunFirst<<<Blocks(P, 256), 256, 0, s>>>(L, flag, id, first);
  // The run count: the last pixel's id plus its flag.
  int tail[2] = {0, 0};
  if ((e = cudaMemcpyAsync(&tail[0], id + P - 1, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(&tail[1], flag + P - 1, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess) {
    return e;
  }
  const int runs = tail[0] + tail[1];
  const int64_t E = static_cast<int64_t>(runs) * L.levels;
  RunContrib<<<Blocks(runs, 128), 128, 0, s>>>(L, first, runs, keys, vals, lkeys, lruns);
  const int end_bit = 36;
  cub::DoubleBuffer<uint64_t> dk(keys, keys2);
  cub::DoubleBuffer<double> dv(vals, vals2);
  need = temp_bytes;
  if ((e = cub::DeviceRadixSort::SortPairs(temp, need, dk, dv, static_cast<int>(E), 0, end_bit, s)) !=
      cudaSuccess) {
    return e;
  }
  cub::DoubleBuffer<uint64_t> lk(lkeys, lkeys2);
  cub::DoubleBuffer<int> lr(lruns, lruns2);
  need = temp_bytes;
  if ((e = cub::DeviceRadixSort::SortPairs(temp, need, lk, lr, runs, 0, end_bit, s)) != cudaSuccess) {
    return e;
  }
  need = temp_bytes;
  if ((e = cub::DeviceRunLengthEncode::Encode(temp, need, dk.Current(), ukeys, ucount, nseg,
                                              static_cast<int>(E), s)) != cudaSuccess) {
    return e;
  }
  need = temp_bytes;
  if ((e = cub::DeviceRunLengthEncode::Encode(temp, need, lk.Current(), lukeys, lcount, nseg + 1, runs, s)) !=
      cudaSuccess) {
    return e;
  }
  int n[2] = {0, 0};
  if ((e = cudaMemcpyAsync(n, nseg, sizeof(n), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess) {
    return e;
  }
  need = temp_bytes;
  if ((e = cub::DeviceScan::ExclusiveSum(temp, need, ucount, uoff, n[0], s)) != cudaSuccess) return e;
  need = temp_bytes;
  if ((e = cub::DeviceScan::ExclusiveSum(temp, need, lcount, loff, n[1], s)) != cudaSuccess) return e;
  // One warp per node / leaf, eight per block.
  NodeSums<<<Blocks(n[0], 8), 256, 0, s>>>(L, ukeys, uoff, ucount, nseg, dv.Current(), qerr, gain);
  LeafSums<<<Blocks(n[1], 8), 256, 0, s>>>(L, lukeys, loff, lcount, nseg + 1, lr.Current(), first, runs,
                                           lnum, ltot);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  out->keys.resize(static_cast<std::size_t>(n[0]));
  out->qerr.resize(static_cast<std::size_t>(n[0]));
  std::vector<double> g(static_cast<std::size_t>(n[0]));
  out->leaf_keys.resize(static_cast<std::size_t>(n[1]));
  out->leaf_count.resize(static_cast<std::size_t>(n[1]));
  out->leaf_total.resize(4 * static_cast<std::size_t>(n[1]));
  if ((e = cudaMemcpyAsync(out->keys.data(), ukeys, n[0] * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(out->qerr.data(), qerr, n[0] * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(g.data(), gain, n[0] * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(out->leaf_keys.data(), lukeys, n[1] * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(out->leaf_count.data(), lnum, n[1] * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(out->leaf_total.data(), ltot, n[1] * 32, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess) {
    return e;
  }
  double root = 0.0;
  for (double v : g) root += v;
  out->root_gain = root;
  return cudaSuccess;
}

}  // namespace rdb
