// FP64 trailing update of the plain FP64 LU on the FP64 tensor cores:
// C -= A B for complex128 A (m x k), B (k x n), C (m x n), row-major, with
// mma.sync m8n8k4 f64 (Blackwell's FP64 tensor-core instruction; tcgen05 has
// no FP64 kind).  Each complex product is four real ones:
//   Cr -= Ar Br - Ai Bi,   Ci -= Ar Bi + Ai Br
// CTA tile 64 x 64 complex, 4 warps of 32 x 32 (4 x 4 fragments of 8 x 8,
// real and imaginary accumulators: 64 doubles per thread), k in steps of 16
// staged in shared memory with real and imaginary parts in separate padded
// planes (conflict-free fragment loads), double-buffered.
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

namespace necb {

constexpr int kDmmaBM = 64, kDmmaBN = 64, kDmmaBK = 16, kDmmaThreads = 128, kDmmaPad = 4;

__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

struct DmmaSmem {
  double Ar[2][kDmmaBK][kDmmaBM + kDmmaPad], Ai[2][kDmmaBK][kDmmaBM + kDmmaPad];
  double Br[2][kDmmaBK][kDmmaBN + kDmmaPad], Bi[2][kDmmaBK][kDmmaBN + kDmmaPad];
};

__global__ void __launch_bounds__(kDmmaThreads) gemm_dmma_kernel(const double2* __restrict__ A, int64_t lda,
                                                                 const double2* __restrict__ B, int64_t ldb,
                                                                 double2* C, int64_t ldc, int64_t m, int64_t n,
                                                                 int k) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  DmmaSmem& S = *reinterpret_cast<DmmaSmem*>(smem_raw);
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int64_t m0 = (int64_t)blockIdx.y * kDmmaBM, n0 = (int64_t)blockIdx.x * kDmmaBN;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;  // warp's 32 x 32 block in the CTA tile
  const int g = lane >> 2, q = lane & 3;                   // fragment coordinates
  double cr[4][4][2], ci[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      cr[i][j][0] = cr[i][j][1] = 0.0;
      ci[i][j][0] = ci[i][j][1] = 0.0;
    }
  // global -> registers for one k tile: A 64 x 16 and B 16 x 64 complex,
  // 8 of each per thread
  double2 ra[8], rb[8];
  auto load = [&](int k0) {
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int e = t + u * kDmmaThreads;         // 0..1023
      const int r = e >> 4, c = e & 15;           // A: row r, k column c
      const int64_t gr = m0 + r, gc = k0 + c;
      ra[u] = (gr < m && gc < k) ? A[gr * lda + gc] : make_double2(0.0, 0.0);
      const int kr = e >> 6, nc = e & 63;         // B: k row kr, column nc
      const int64_t gk = k0 + kr, gn = n0 + nc;
      rb[u] = (gk < k && gn < n) ? B[gk * ldb + gn] : make_double2(0.0, 0.0);
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int e = t + u * kDmmaThreads;
      const int r = e >> 4, c = e & 15;
      S.Ar[buf][c][r] = ra[u].x;
      S.Ai[buf][c][r] = ra[u].y;
      const int kr = e >> 6, nc = e & 63;
      S.Br[buf][kr][nc] = rb[u].x;
      S.Bi[buf][kr][nc] = rb[u].y;
    }
  };
  load(0);
  store(0);
  __syncthreads();
  const int ktiles = (k + kDmmaBK - 1) / kDmmaBK;
  for (int kt = 0; kt < ktiles; kt++) {
    const int buf = kt & 1;
    if (kt + 1 < ktiles) load((kt + 1) * kDmmaBK);  // in flight during the MMAs
#pragma unroll
    for (int kk = 0; kk < kDmmaBK; kk += 4) {
      double ar[4], ai[4], br[4], bi[4];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        ar[i] = S.Ar[buf][kk + q][wm + 8 * i + g];
        ai[i] = S.Ai[buf][kk + q][wm + 8 * i + g];
      }
#pragma unroll
      for (int j = 0; j < 4; j++) {
        br[j] = S.Br[buf][kk + q][wn + 8 * j + g];
        bi[j] = S.Bi[buf][kk + q][wn + 8 * j + g];
      }
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const double nai = -ai[i];
#pragma unroll
        for (int j = 0; j < 4; j++) {
          dmma_8x8x4(cr[i][j][0], cr[i][j][1], ar[i], br[j]);
          dmma_8x8x4(cr[i][j][0], cr[i][j][1], nai, bi[j]);
          dmma_8x8x4(ci[i][j][0], ci[i][j][1], ar[i], bi[j]);
          dmma_8x8x4(ci[i][j][0], ci[i][j][1], ai[i], br[j]);
        }
      }
    }
    if (kt + 1 < ktiles) store(buf ^ 1);
    __syncthreads();
  }
  // C fragment: row g, columns 2q, 2q+1 of each 8 x 8 tile
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int64_t row = m0 + wm + 8 * i + g;
    if (row >= m) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int64_t col = n0 + wn + 8 * j + 2 * q + h;
        if (col >= n) continue;
        double2* p = C + row * ldc + col;
        double2 v = *p;
        v.x -= cr[i][j][h];
        v.y -= ci[i][j][h];
        *p = v;
      }
    }
  }
}

}  // namespace necb
