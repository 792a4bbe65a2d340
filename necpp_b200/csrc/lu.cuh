// Dense complex LU with partial pivoting (replaces Eigen::PartialPivLU in
// lu_decompose, src/matrix_algebra.cpp:217-266).
//
// Storage is row-major (M[r*ld + c]) so that a row interchange is a swap of
// two contiguous segments.  Right-looking blocked algorithm, block nb:
//   1. panel_kernel   rows [k0,n) x cols [k0,k0+kb): cooperative kernel, the
//                     panel's rows spread over P CTAs in shared memory; per
//                     column one bounded grid barrier (candidate pivots and
//                     their rows are published in double-buffered slots);
//   2. laswp_kernel   the kb interchanges on the columns outside the panel;
//   3. trsm_kernel    U12 = L11^-1 A12 (unit lower, in shared memory);
//   4. trailing update A22 -= L21 U12 (gemm_kernel here for FP64; the mixed
//                     path uses the tensor-core kernel of gemm_tc.cuh).
// Pivots are global row indices (0-based); piv[k] = row swapped with k.
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

namespace necb {

template <typename R>
struct cvec;
template <>
struct cvec<double> {
  using T = double2;
};
template <>
struct cvec<float> {
  using T = float2;
};

template <typename T>
__device__ __forceinline__ T cmul(T a, T b) {
  T r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename T>
__device__ __forceinline__ T cdiv(T a, T b) {  // Smith's algorithm
  T r;
  if (fabs(b.x) < fabs(b.y)) {
    auto ratio = b.x / b.y;
    auto den = (b.x * ratio) + b.y;
    r.x = ((a.x * ratio) + a.y) / den;
    r.y = ((a.y * ratio) - a.x) / den;
  } else {
    auto ratio = b.y / b.x;
    auto den = (b.y * ratio) + b.x;
    r.x = ((a.y * ratio) + a.x) / den;
    r.y = (a.y - (a.x * ratio)) / den;
  }
  return r;
}

enum : int {
  kLuStatSingular = 1 << 8,
  kLuStatBarrierTimeout = 1 << 9,
  kLuStatNonFinite = 1 << 10,
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <typename R>
struct PanelArgs {
  typename cvec<R>::T* M;
  int64_t ld, n, k0;
  int kb, rpc;
  int* piv;
  R* cand_val;                       // [2*P]
  int* cand_row;                     // [2*P]
  typename cvec<R>::T* cand_rows;    // [2*P*NB]
  typename cvec<R>::T* rowc;         // [2*NB]
  unsigned* counter;                 // zeroed before launch
  int* status;
};

constexpr int kPanelThreads = 256;
constexpr long long kBarrierSpinLimit = 1LL << 26;

template <typename R, int NB>
__global__ void __launch_bounds__(kPanelThreads) panel_kernel(PanelArgs<R> A) {
  using T = typename cvec<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S = reinterpret_cast<T*>(smem_raw);  // [rpc][NB]
  T* prow = S + (size_t)A.rpc * NB;        // [NB]
  T* crow = prow + NB;                     // [NB]
  __shared__ R red_val[kPanelThreads / 32];
  __shared__ int red_row[kPanelThreads / 32];
  __shared__ int s_p, s_owner, s_abort;

  const int b = blockIdx.x, P = gridDim.x, tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int64_t k0 = A.k0;
  const int kb = A.kb;
  const int64_t rbeg = k0 + (int64_t)b * A.rpc;
  const int64_t rend = min(A.n, rbeg + (int64_t)A.rpc);
  const int nr = rend > rbeg ? (int)(rend - rbeg) : 0;
  if (tid == 0) s_abort = 0;

  for (int idx = tid; idx < nr * kb; idx += kPanelThreads) {
    int r = idx / kb, c = idx - r * kb;
    S[r * NB + c] = A.M[(rbeg + r) * A.ld + k0 + c];
  }
  __syncthreads();

  for (int c = 0; c < kb; c++) {
    const int64_t gc = k0 + c;
    const int slot = c & 1;
    // local pivot candidate: largest |a|^2, ties to the lowest row
    R best = (R)-1;
    int brow = 0x7fffffff;
    for (int r = tid; r < nr; r += kPanelThreads) {
      int64_t g = rbeg + r;
      if (g >= gc) {
        T v = S[r * NB + c];
        R m = v.x * v.x + v.y * v.y;
        if (m > best || (m == best && g < brow)) {
          best = m;
          brow = (int)g;
        }
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      R ov = __shfl_down_sync(0xffffffffu, best, off);
      int orow = __shfl_down_sync(0xffffffffu, brow, off);
      if (ov > best || (ov == best && orow < brow)) {
        best = ov;
        brow = orow;
      }
    }
    if (lane == 0) {
      red_val[warp] = best;
      red_row[warp] = brow;
    }
    __syncthreads();
    if (tid == 0) {
      for (int w = 1; w < kPanelThreads / 32; w++)
        if (red_val[w] > best || (red_val[w] == best && red_row[w] < brow)) {
          best = red_val[w];
          brow = red_row[w];
        }
      red_val[0] = best;
      red_row[0] = brow;
      A.cand_val[slot * P + b] = best;
      A.cand_row[slot * P + b] = brow;
    }
    __syncthreads();
    best = red_val[0];
    brow = red_row[0];
    if (best >= (R)0) {
      const T* src = S + (size_t)(brow - rbeg) * NB;
      for (int q = tid; q < kb; q += kPanelThreads) A.cand_rows[((size_t)slot * P + b) * NB + q] = src[q];
    }
    if (gc >= rbeg && gc < rend) {
      const T* src = S + (size_t)(gc - rbeg) * NB;
      for (int q = tid; q < kb; q += kPanelThreads) A.rowc[slot * NB + q] = src[q];
    }
    __syncthreads();
    // grid barrier (bounded)
    if (tid == 0) {
      __threadfence();
      atomicAdd(A.counter, 1u);
      const unsigned target = (unsigned)(c + 1) * (unsigned)P;
      long long spins = 0;
      while (ld_acquire_u32(A.counter) < target) {
        if (++spins > kBarrierSpinLimit) {
          atomicOr(A.status, kLuStatBarrierTimeout);
          s_abort = 1;
          break;
        }
        __nanosleep(32);
      }
      __threadfence();
    }
    __syncthreads();
    if (s_abort) break;
    // global pivot: every CTA reduces the same candidates identically
    if (warp == 0) {
      R gb = (R)-1;
      int gr = 0x7fffffff, go = 0;
      for (int q = lane; q < P; q += 32) {
        R v = __ldcg(A.cand_val + slot * P + q);
        int rr = __ldcg(A.cand_row + slot * P + q);
        if (v > gb || (v == gb && rr < gr)) {
          gb = v;
          gr = rr;
          go = q;
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        R ov = __shfl_down_sync(0xffffffffu, gb, off);
        int orow = __shfl_down_sync(0xffffffffu, gr, off);
        int oo = __shfl_down_sync(0xffffffffu, go, off);
        if (ov > gb || (ov == gb && orow < gr)) {
          gb = ov;
          gr = orow;
          go = oo;
        }
      }
      if (lane == 0) {
        if (!(gb > (R)0)) {  // zero (or NaN) pivot column
          if (b == 0) atomicOr(A.status, gb == (R)0 ? kLuStatSingular : kLuStatNonFinite);
          gr = (int)gc;
          go = -1;
        }
        s_p = gr;
        s_owner = go;
      }
    }
    __syncthreads();
    const int64_t p = s_p;
    const int ob = s_owner;
    for (int q = tid; q < kb; q += kPanelThreads) {
      if (ob >= 0) {
        prow[q] = __ldcg(A.cand_rows + ((size_t)slot * P + ob) * NB + q);
      } else {
        T z;
        z.x = (R)1;
        z.y = (R)0;
        prow[q] = (gc >= rbeg && gc < rend) ? S[(gc - rbeg) * NB + q] : z;
      }
      crow[q] = __ldcg(A.rowc + slot * NB + q);
    }
    __syncthreads();
    if (ob >= 0 && p != gc) {
      if (p >= rbeg && p < rend)
        for (int q = tid; q < kb; q += kPanelThreads) S[(p - rbeg) * NB + q] = crow[q];
      if (gc >= rbeg && gc < rend)
        for (int q = tid; q < kb; q += kPanelThreads) S[(gc - rbeg) * NB + q] = prow[q];
    }
    if (b == 0 && tid == 0) A.piv[gc] = (int)p;
    __syncthreads();
    T pv = prow[c];
    if (ob < 0) {
      pv.x = (R)1;
      pv.y = (R)0;
    }
    for (int r = tid; r < nr; r += kPanelThreads) {
      if (rbeg + r > gc) S[r * NB + c] = cdiv(S[r * NB + c], pv);
    }
    __syncthreads();
    const int w = kb - c - 1;
    if (w > 0) {
      for (int idx = tid; idx < nr * w; idx += kPanelThreads) {
        int r = idx / w;
        int q = c + 1 + (idx - r * w);
        if (rbeg + r > gc) {
          T l = S[r * NB + c];
          T u = prow[q];
          T a = S[r * NB + q];
          a.x -= l.x * u.x - l.y * u.y;
          a.y -= l.x * u.y + l.y * u.x;
          S[r * NB + q] = a;
        }
      }
    }
    __syncthreads();
  }
  for (int idx = tid; idx < nr * kb; idx += kPanelThreads) {
    int r = idx / kb, c = idx - r * kb;
    A.M[(rbeg + r) * A.ld + k0 + c] = S[r * NB + c];
  }
}

// ---------------------------------------------------------------------------
// Block-local pivoting (mixed-precision path).  The pivot of column k is the
// largest entry among the rows of k's own 64-row diagonal block instead of
// the whole column, so a panel needs no grid-wide reduction: one CTA factors
// the diagonal block, a row-parallel kernel forms L21 = A21 U11^-1.  The
// mixed path refines every solution against the FP64 matrix and falls back
// to full partial pivoting if the refinement does not converge.

// LU with partial pivoting inside the kb x kb diagonal block at (k0, k0).
// 64 threads; thread t owns row t.  piv[k0 + c] receives the global row.
template <typename T, int NB>
__global__ void __launch_bounds__(NB) diag_lu_kernel(T* M, int64_t ld, int64_t k0, int kb, int* piv, int* status) {
  using R = decltype(T{}.x);
  __shared__ T D[NB][NB + 1];
  __shared__ R rv[NB / 32];
  __shared__ int ri[NB / 32];
  __shared__ int s_p;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (int r = 0; r < kb; r++)
    if (t < kb) D[r][t] = M[(k0 + r) * ld + k0 + t];
  __syncthreads();
  for (int c = 0; c < kb; c++) {
    R best = (R)-1;
    int brow = 0x7fffffff;
    if (t >= c && t < kb) {
      T v = D[t][c];
      best = v.x * v.x + v.y * v.y;
      brow = t;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      R ov = __shfl_down_sync(0xffffffffu, best, off);
      int orow = __shfl_down_sync(0xffffffffu, brow, off);
      if (ov > best || (ov == best && orow < brow)) {
        best = ov;
        brow = orow;
      }
    }
    if (lane == 0) {
      rv[warp] = best;
      ri[warp] = brow;
    }
    __syncthreads();
    if (t == 0) {
      for (int w = 1; w < NB / 32; w++)
        if (rv[w] > best || (rv[w] == best && ri[w] < brow)) {
          best = rv[w];
          brow = ri[w];
        }
      if (!(best > (R)0)) {
        atomicOr(status, best == (R)0 ? kLuStatSingular : kLuStatNonFinite);
        brow = c;
      }
      s_p = brow;
      piv[k0 + c] = (int)(k0 + brow);
    }
    __syncthreads();
    const int p = s_p;
    if (p != c && t < kb) {
      T a = D[c][t];
      D[c][t] = D[p][t];
      D[p][t] = a;
    }
    __syncthreads();
    if (t > c && t < kb) {
      T l = cdiv(D[t][c], D[c][c]);
      D[t][c] = l;
      for (int q = c + 1; q < kb; q++) {
        T u = D[c][q];
        T a = D[t][q];
        a.x -= l.x * u.x - l.y * u.y;
        a.y -= l.x * u.y + l.y * u.x;
        D[t][q] = a;
      }
    }
    __syncthreads();
  }
  for (int r = 0; r < kb; r++)
    if (t < kb) M[(k0 + r) * ld + k0 + t] = D[r][t];
}

// L21 = A21 U11^-1 for rows [k0+kb, n) of the panel columns: one thread per
// row, U11 in shared memory, the row staged through shared memory.
template <typename T, int NB>
__global__ void __launch_bounds__(128) trsm_right_kernel(T* M, int64_t ld, int64_t n, int64_t k0, int kb) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* U = reinterpret_cast<T*>(smem_raw);  // [NB][NB+1]
  T* X = U + NB * (NB + 1);                // [128][NB+1]
  const int t = threadIdx.x;
  const int64_t r0 = k0 + kb + (int64_t)blockIdx.x * 128;
  for (int idx = t; idx < kb * kb; idx += 128) {
    const int r = idx / kb, c = idx - r * kb;
    U[r * (NB + 1) + c] = M[(k0 + r) * ld + k0 + c];
  }
  // coalesced staging of 128 rows x kb
  for (int idx = t; idx < 128 * kb; idx += 128) {
    const int r = idx / kb, c = idx - r * kb;
    T v;
    v.x = 0;
    v.y = 0;
    if (r0 + r < n) v = M[(r0 + r) * ld + k0 + c];
    X[r * (NB + 1) + c] = v;
  }
  __syncthreads();
  T* x = X + t * (NB + 1);
  for (int q = 0; q < kb; q++) {
    T v = cdiv(x[q], U[q * (NB + 1) + q]);
    x[q] = v;
    for (int p = q + 1; p < kb; p++) {
      T u = U[q * (NB + 1) + p];
      T a = x[p];
      a.x -= v.x * u.x - v.y * u.y;
      a.y -= v.x * u.y + v.y * u.x;
      x[p] = a;
    }
  }
  __syncthreads();
  for (int idx = t; idx < 128 * kb; idx += 128) {
    const int r = idx / kb, c = idx - r * kb;
    if (r0 + r < n) M[(r0 + r) * ld + k0 + c] = X[r * (NB + 1) + c];
  }
}

// Row interchanges of one panel on the columns outside it.
template <typename T>
__global__ void laswp_kernel(T* M, int64_t ld, int64_t n, int64_t k0, int kb, const int* piv) {
  int64_t col = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= n || (col >= k0 && col < k0 + kb)) return;
  for (int c = 0; c < kb; c++) {
    int64_t p = piv[k0 + c];
    int64_t g = k0 + c;
    if (p != g) {
      T a = M[g * ld + col];
      T b = M[p * ld + col];
      M[g * ld + col] = b;
      M[p * ld + col] = a;
    }
  }
}

// U12 = L11^-1 A12 for one panel; one CTA per 32 columns of A12.
template <typename T, int NB>
__global__ void __launch_bounds__(256) trsm_kernel(T* M, int64_t ld, int64_t n, int64_t k0, int kb) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* L = reinterpret_cast<T*>(smem_raw);  // [NB][NB]
  T* X = L + NB * NB;                      // [NB][32]
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int64_t c0 = k0 + kb + (int64_t)blockIdx.x * 32;
  const int64_t col = c0 + tx;
  for (int idx = threadIdx.x; idx < kb * kb; idx += 256) {
    int r = idx / kb, q = idx - r * kb;
    L[r * NB + q] = M[(k0 + r) * ld + k0 + q];
  }
  for (int r = ty; r < kb; r += 8) {
    T v;
    v.x = 0;
    v.y = 0;
    if (col < n) v = M[(k0 + r) * ld + col];
    X[r * 32 + tx] = v;
  }
  __syncthreads();
  for (int r = 0; r < kb - 1; r++) {
    T xr = X[r * 32 + tx];
    for (int q = r + 1 + ty; q < kb; q += 8) {
      T l = L[q * NB + r];
      T a = X[q * 32 + tx];
      a.x -= l.x * xr.x - l.y * xr.y;
      a.y -= l.x * xr.y + l.y * xr.x;
      X[q * 32 + tx] = a;
    }
    __syncthreads();
  }
  if (col < n)
    for (int r = ty; r < kb; r += 8) M[(k0 + r) * ld + col] = X[r * 32 + tx];
}

// C -= A * B, complex, CUDA-core tiles of 64x64, 256 threads, 4x4 per thread.
// A: m x k (row-major, lda), B: k x n2 (row-major, ldb), C: m x n2.
template <typename R>
__global__ void __launch_bounds__(256) gemm_sub_kernel(const typename cvec<R>::T* A, int64_t lda,
                                                       const typename cvec<R>::T* B, int64_t ldb,
                                                       typename cvec<R>::T* C, int64_t ldc, int64_t m,
                                                       int64_t n2, int k) {
  using T = typename cvec<R>::T;
  constexpr int BM = 64, BN = 64, BK = 16;
  __shared__ T sA[BK][BM + 1];
  __shared__ T sB[BK][BN + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int64_t m0 = (int64_t)blockIdx.y * BM, n0 = (int64_t)blockIdx.x * BN;
  R accr[4][4], acci[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      accr[i][j] = 0;
      acci[i][j] = 0;
    }
  for (int kk = 0; kk < k; kk += BK) {
    for (int idx = threadIdx.x; idx < BM * BK; idx += 256) {
      int r = idx / BK, q = idx - r * BK;
      T v;
      v.x = 0;
      v.y = 0;
      if (m0 + r < m && kk + q < k) v = A[(m0 + r) * lda + kk + q];
      sA[q][r] = v;
    }
    for (int idx = threadIdx.x; idx < BK * BN; idx += 256) {
      int q = idx / BN, cc = idx - q * BN;
      T v;
      v.x = 0;
      v.y = 0;
      if (kk + q < k && n0 + cc < n2) v = B[(int64_t)(kk + q) * ldb + n0 + cc];
      sB[q][cc] = v;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < BK; q++) {
      T a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = sA[q][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = sB[q][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
          accr[i][j] += a[i].x * b[j].x - a[i].y * b[j].y;
          acci[i][j] += a[i].x * b[j].y + a[i].y * b[j].x;
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    int64_t r = m0 + ty + 16 * i;
    if (r >= m) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      int64_t cc = n0 + tx + 16 * j;
      if (cc >= n2) continue;
      T v = C[r * ldc + cc];
      v.x -= accr[i][j];
      v.y -= acci[i][j];
      C[r * ldc + cc] = v;
    }
  }
}

}  // namespace necb
