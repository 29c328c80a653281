// rdb_probe.cu -- dependent-latency table of the operations on the sequential
// walk's per-step chain (rdb_probe_latency in include/rdb.h).
//
// One thread runs chains of kOps operations in which every operation consumes
// the previous result, timed with clock64(): the cycles between issue of one
// and issue of the next are the operation's latency.  Conversions are timed
// as a round trip closed by a DADD with a runtime zero (so the compiler cannot
// fold the round trip away) and the DADD's own latency is subtracted; loads
// are pointer chases over tables that live in shared memory, in L1 (a 4 KB
// table read twice before timing) and in L2 only (an 8 MB table read with
// .cg loads, which bypass L1, after a warming pass).
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/rdb.h"
#include "rdb_runtime.h"

namespace rdb {
namespace {

constexpr int kOps = 512;
constexpr int kSmemWords = 1024;
constexpr int kL1Words = 1024;                       // 4 KB
constexpr int kL2Words = 2 * 1024 * 1024;            // 8 MB
constexpr int kL2Stride = 32;                        // words: one 128-byte line per hop

__device__ __forceinline__ uint32_t ld_cg(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.global.cg.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

__device__ __forceinline__ uint32_t ld_ca(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.global.ca.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

__global__ void ProbeKernel(double seed, double zero, const uint32_t* l1, const uint32_t* l2,
                            double* out_cycles, double* sink) {
  __shared__ uint32_t sm[kSmemWords];
  if (threadIdx.x != 0) return;
  for (int i = 0; i < kSmemWords; ++i) sm[i] = static_cast<uint32_t>((i * 97 + 1) % kSmemWords);
  double x = seed;
  long long t0, t1;

  // DADD
  t0 = clock64();
#pragma unroll 64
  for (int i = 0; i < kOps; ++i) x = __dadd_rn(x, zero);
  t1 = clock64();
  const double dadd = static_cast<double>(t1 - t0) / kOps;
  // DMUL (by a runtime one)
  const double one = __dadd_rn(zero, 1.0);
  t0 = clock64();
#pragma unroll 64
  for (int i = 0; i < kOps; ++i) x = __dmul_rn(x, one);
  t1 = clock64();
  const double dmul = static_cast<double>(t1 - t0) / kOps;
  // double -> float -> double round trip, closed by a DADD
  t0 = clock64();
#pragma unroll 64
  for (int i = 0; i < kOps; ++i) x = __dadd_rn(static_cast<double>(__double2float_rn(x)), zero);
  t1 = clock64();
  const double cvt_pair = static_cast<double>(t1 - t0) / kOps - dadd;
  // float -> int -> double, closed by a DADD (the byte rule's float -> int)
  t0 = clock64();
#pragma unroll 64
  for (int i = 0; i < kOps; ++i) {
    const int v = __float2int_rz(__double2float_rn(x));
    x = __dadd_rn(static_cast<double>(v), zero);
  }
  t1 = clock64();
  const double f2i = static_cast<double>(t1 - t0) / kOps - dadd - cvt_pair;
  // integer ALU: alternating add and xor with runtime operands
  uint32_t v = static_cast<uint32_t>(x);
  const uint32_t k = static_cast<uint32_t>(one) + 2u;
  t0 = clock64();
#pragma unroll 64
  for (int i = 0; i < kOps / 2; ++i) v = (v + k) ^ (k << 1);
  t1 = clock64();
  const double int_op = static_cast<double>(t1 - t0) / kOps;
  // shared-memory pointer chase
  uint32_t p = (static_cast<uint32_t>(x) + (v & 1u)) & (kSmemWords - 1);
  t0 = clock64();
#pragma unroll 16
  for (int i = 0; i < kOps; ++i) p = sm[p];
  t1 = clock64();
  const double lds = static_cast<double>(t1 - t0) / kOps;
  // L1-resident global chase (warmed by two untimed passes)
  uint32_t q = p & (kL1Words - 1);
  for (int i = 0; i < 2 * kL1Words; ++i) q = ld_ca(l1 + q);
  t0 = clock64();
#pragma unroll 16
  for (int i = 0; i < kOps; ++i) q = ld_ca(l1 + q);
  t1 = clock64();
  const double ldg_l1 = static_cast<double>(t1 - t0) / kOps;
  // L2-resident global chase (.cg: not cached in L1)
  uint32_t r = (q & 7u) * kL2Stride;
  for (int i = 0; i < kL2Words / kL2Stride; ++i) r = ld_cg(l2 + r);
  t0 = clock64();
#pragma unroll 16
  for (int i = 0; i < kOps; ++i) r = ld_cg(l2 + r);
  t1 = clock64();
  const double ldg_l2 = static_cast<double>(t1 - t0) / kOps;

  out_cycles[0] = dadd;
  out_cycles[1] = dmul;
  out_cycles[2] = cvt_pair / 2.0;
  out_cycles[3] = cvt_pair / 2.0;
  out_cycles[4] = f2i;
  out_cycles[5] = lds;
  out_cycles[6] = ldg_l1;
  out_cycles[7] = ldg_l2;
  out_cycles[8] = int_op;
  *sink = x + static_cast<double>(p + q + r);
}

}  // namespace
}  // namespace rdb

extern "C" int rdb_probe_latency(int device, rdb_latency_table* out) {
  using namespace rdb;
  if (!out) return Fail(RDB_E_INVALID, "rdb_probe_latency: null output");
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return CudaFail(e, "rdb_probe_latency: cudaSetDevice");
  uint32_t* l1 = nullptr;
  uint32_t* l2 = nullptr;
  double* res = nullptr;
  const auto cleanup = [&] {
    cudaFree(l1);
    cudaFree(l2);
    cudaFree(res);
  };
  if ((e = cudaMalloc(&l1, kL1Words * sizeof(uint32_t))) != cudaSuccess ||
      (e = cudaMalloc(&l2, kL2Words * sizeof(uint32_t))) != cudaSuccess ||
      (e = cudaMalloc(&res, 16 * sizeof(double))) != cudaSuccess) {
    cleanup();
    return CudaFail(e, "rdb_probe_latency: allocation");
  }
  // Chase tables: l1[i] = next index, a long cycle over the 4 KB table; l2
  // visits one word per 128-byte line, lines in a scrambled cycle.
  uint32_t* h1 = new uint32_t[kL1Words];
  for (int i = 0; i < kL1Words; ++i) h1[i] = static_cast<uint32_t>((i * 389 + 7) % kL1Words);
  const int lines = kL2Words / kL2Stride;
  uint32_t* h2 = new uint32_t[kL2Words]();
  for (int i = 0; i < lines; ++i) {
    const int next = static_cast<int>((static_cast<int64_t>(i) * 40503 + 12345) % lines);
    h2[i * kL2Stride] = static_cast<uint32_t>(next * kL2Stride);
  }
  e = cudaMemcpy(l1, h1, kL1Words * sizeof(uint32_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(l2, h2, kL2Words * sizeof(uint32_t), cudaMemcpyHostToDevice);
  delete[] h1;
  delete[] h2;
  if (e != cudaSuccess) {
    cleanup();
    return CudaFail(e, "rdb_probe_latency: upload");
  }
  ProbeKernel<<<1, 32>>>(1.5, 0.0, l1, l2, res, res + 12);
  double cyc[9] = {0};
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(cyc, res, sizeof(cyc), cudaMemcpyDeviceToHost);
  cleanup();
  if (e != cudaSuccess) return CudaFail(e, "rdb_probe_latency: kernel");
  out->dadd = cyc[0];
  out->dmul = cyc[1];
  out->f64_to_f32 = cyc[2];
  out->f32_to_f64 = cyc[3];
  out->f32_to_int = cyc[4];
  out->shared_load = cyc[5];
  out->global_load_l1 = cyc[6];
  out->global_load_l2 = cyc[7];
  out->int_op = cyc[8];
  return RDB_OK;
}
