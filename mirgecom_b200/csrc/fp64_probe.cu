// FP64 throughput probes: the compute roofline of the float64 path.
//
// The float64 right-hand side runs its contractions on the float64 tensor
// cores (mma.m8n8k4.f64, "DMMA") and its pointwise math on the FP64 FMA
// pipe, so its compute roofline is set by those two rates.  No published
// or driver-measured figure exists for them on this part, so they are
// measured here: each kernel runs independent chains of the one
// instruction (enough per warp to cover its latency) over a grid that
// fills every SM, and the host times it with CUDA events.
//   kind 0: DFMA  -- 8 independent fma.rn.f64 chains per thread, 2 flops each
//   kind 1: DMMA  -- 8 independent m8n8k4 accumulators per warp, 512 flops each
#include <cuda_runtime.h>

#include "../../include/mgc_b200.h"

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) k_probe_dfma(int iters, double seed, double* sink) {
  double x[kChains];
  const double a = 1.0 - 1e-12 * (threadIdx.x + 1), b = 1e-9 * seed;
#pragma unroll
  for (int i = 0; i < kChains; ++i) x[i] = seed + i;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < kChains; ++i) x[i] = fma(x[i], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < kChains; ++i) s += x[i];
  sink[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) k_probe_dmma(int iters, double seed, double* sink) {
  double d[kChains][2];
  const double a = 1e-3 * (threadIdx.x & 31), b = seed * 1e-3;
#pragma unroll
  for (int i = 0; i < kChains; ++i) d[i][0] = d[i][1] = 0.0;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < kChains; ++i)
      asm volatile(
          "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
          : "+d"(d[i][0]), "+d"(d[i][1])
          : "d"(a), "d"(b));
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < kChains; ++i) s += d[i][0] + d[i][1];
  sink[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" {

double mgc_fp64_probe_flops(int kind, int nblocks, int threads, int iters) {
  if (nblocks <= 0 || threads <= 0 || iters <= 0) return 0.0;
  if (kind == 0) return 2.0 * kChains * (double)iters * threads * nblocks;
  if (kind == 1) return 512.0 * kChains * (double)iters * (threads / 32) * nblocks;
  return 0.0;
}

int mgc_fp64_probe(int kind, int nblocks, int threads, int iters, double* sink,
                   void* stream) {
  if (nblocks <= 0 || threads <= 0 || threads > 256 || threads % 32 || iters <= 0 || !sink)
    return MGC_E_INVALID;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (kind == 0)
    k_probe_dfma<<<nblocks, threads, 0, s>>>(iters, 1.5, sink);
  else if (kind == 1)
    k_probe_dmma<<<nblocks, threads, 0, s>>>(iters, 1.5, sink);
  else
    return MGC_E_INVALID;
  return cudaGetLastError() == cudaSuccess ? MGC_OK : MGC_E_CUDA;
}

}  // extern "C"
