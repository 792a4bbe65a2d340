// FP64 throughput probes: the measured denominators of the FP64 kernels'
// rooflines (the FP64 fill and pattern on the CUDA cores, the FP64 LU's
// trailing update on the FP64 tensor cores).  Register-only loops with
// independent accumulator chains per thread; nothing is read from memory, and
// one store per thread keeps the compiler from removing the work.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace necb {
namespace peak {

constexpr int kThreads = 256;
constexpr int kChains = 8;

// kChains independent FMA chains per thread: 2 * kChains flops per iteration
__global__ void __launch_bounds__(kThreads) dfma_peak_kernel(double* sink, int iters) {
  double a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; k++) a[k] = 1e-3 * (threadIdx.x + k);
  const double b = 0.999999999, c = 1e-12;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < kChains; k++) a[k] = fma(a[k], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kChains; k++) s += a[k];
  sink[(int64_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// four independent m8n8k4 FP64 MMA chains per warp: 4 * 512 flops per
// iteration and warp
__global__ void __launch_bounds__(kThreads) dmma_peak_kernel(double* sink, int iters) {
  double acc[4][2];
#pragma unroll
  for (int k = 0; k < 4; k++) acc[k][0] = acc[k][1] = 0.0;
  const double a = 1e-3 * (threadIdx.x & 31), b = 0.5;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 4; k++)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                   : "+d"(acc[k][0]), "+d"(acc[k][1])
                   : "d"(a), "d"(b));
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 4; k++) s += acc[k][0] + acc[k][1];
  sink[(int64_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace peak
}  // namespace necb
