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
#include <type_traits>

#include <cuda_runtime.h>

#include "gemm_tc.cuh"

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
// the diagonal block, then
//   L21 = A21 U11^-1   trsm_panel_kernel<RIGHT>, one row of A21 per thread
//   U12 = L11^-1 A12   trsm_panel_kernel<LEFT>,  one column of A12 per thread
// The mixed path refines every solution against the FP64 matrix and falls
// back to full partial pivoting if the refinement does not converge.

constexpr int kBlk = 64;  // diagonal block edge

template <typename T>
__device__ __forceinline__ T czero() {
  T z;
  z.x = 0;
  z.y = 0;
  return z;
}

template <typename T>
__device__ __forceinline__ T crecip(T b) {  // 1 / b, Smith's algorithm
  T r;
  if (fabs(b.x) < fabs(b.y)) {
    const auto ratio = b.x / b.y;
    const auto den = (b.x * ratio) + b.y;
    r.x = ratio / den;
    r.y = -1 / den;
  } else {
    const auto ratio = b.y / b.x;
    const auto den = (b.y * ratio) + b.x;
    r.x = 1 / den;
    r.y = -ratio / den;
  }
  return r;
}

// 1 / x for a pivot's |p|^2 in [1e-30, 1e30]: the hardware's approximate
// reciprocal refined by one Newton-Raphson step (r <- r (2 - x r)), a few
// ulp at most; the refinement of the solution absorbs it
__device__ __forceinline__ float pivot_rcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r * fmaf(-x, r, 2.f);
}
__device__ __forceinline__ double pivot_rcp(double x) { return 1.0 / x; }

// LU with partial pivoting inside the kb x kb diagonal block at (k0, k0)
// (kb <= 64), in place.  piv[k0 + c] receives the global row exchanged with
// row k0 + c (exchanges applied in order, as LAPACK's ipiv), src[k0 + r]
// the block row that ends up in row r (the same permutation as a gather),
// dinv[c] 1 / U[c][c].
//
// Rows are not moved while factoring: the pivot of column c is chosen among
// the rows not yet used as pivots (largest |v|^2, lowest row on ties), rows
// already used are left alone by later updates, and the block is written
// out in pivot order at the end, which gives the same L and U as exchanging
// rows at every step.  The block is factored in panels of 8 columns.  Warp
// 0 holds a 64 x 8 panel in registers (lane l: rows l and l+32) and factors
// it with shuffles only, while the other warps apply the previous panel's
// update to the columns beyond the current panel (lookahead).  Then all
// warps form the panel's 8 U rows on the trailing columns (forward
// substitution, one column per thread) and apply the K = 8 update to the
// next panel's columns.  Three barriers per panel.
constexpr int kDiagThreads = 256;
constexpr int kDiagPanel = 8;

template <typename T>
__global__ void __launch_bounds__(kDiagThreads) diag_lu_kernel(T* M, int64_t ld, int64_t k0, int kb, int* piv,
                                                               int* src, T* dinv, int* status) {
  using R = decltype(T{}.x);
  constexpr int NB = kBlk, PER = NB * NB / kDiagThreads, W = kDiagPanel;
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ T D[NB][NB + 1];
  __shared__ int s_seq[NB];                // physical row of pivot c
  __shared__ int s_row_at[NB], s_pos[NB];  // interchange bookkeeping
  __shared__ unsigned char s_used[2][NB];  // after panel j (buffer j & 1): row outside the block or a pivot
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  {
    T v[PER];  // all loads in flight before the first shared-memory store
#pragma unroll
    for (int i = 0; i < PER; i++) {
      const int e = t + i * kDiagThreads, r = e / NB, c = e % NB;
      v[i] = (r < kb && c < kb) ? M[(k0 + r) * ld + k0 + c] : czero<T>();
    }
#pragma unroll
    for (int i = 0; i < PER; i++) {
      const int e = t + i * kDiagThreads;
      D[e / NB][e % NB] = v[i];
    }
  }
  if (t < NB) {
    s_row_at[t] = t;
    s_pos[t] = t;
  }
  __syncthreads();
  // the LAPACK interchange of pivot c, recorded in order of c by one thread
  auto record = [&](int c) {
    const int p = s_seq[c];
    const int i = s_pos[p], rc = s_row_at[c];
    piv[k0 + c] = (int)(k0 + i);
    s_row_at[c] = p;
    s_row_at[i] = rc;
    s_pos[p] = c;
    s_pos[rc] = i;
  };
  // columns [qa, qb) of the rows not in `used` -= (panel at pj0, width pw)
  // times its U rows: one column and every G-th row per thread, four rows
  // at a time
  auto update = [&](int tid, int nthr, int pj0, int pw, const unsigned char* used, int qa, int qb) {
    const int nq = qb - qa;
    if (nq <= 0) return;
    const int G = max(1, nthr / nq);
    if (tid >= G * nq) return;
    const int q = qa + tid % nq, g = tid / nq;
    T u[W];
#pragma unroll
    for (int k = 0; k < W; k++) u[k] = k < pw ? D[s_seq[pj0 + k]][q] : czero<T>();
    for (int r0 = g; r0 < kb; r0 += 4 * G) {
      T acc[4];
      bool act[4];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int r = r0 + i * G;
        act[i] = r < kb && !used[r];
        acc[i] = act[i] ? D[r][q] : czero<T>();
      }
#pragma unroll
      for (int k = 0; k < W; k++) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
          if (act[i]) {
            const T l = D[r0 + i * G][pj0 + k];
            acc[i].x -= l.x * u[k].x - l.y * u[k].y;
            acc[i].y -= l.x * u[k].y + l.y * u[k].x;
          }
        }
      }
#pragma unroll
      for (int i = 0; i < 4; i++)
        if (act[i]) D[r0 + i * G][q] = acc[i];
    }
  };
  // warp 0's view of the used rows: bit h for row lane + 32 h
  unsigned used = (lane >= kb ? 1u : 0u) | (lane + 32 >= kb ? 2u : 0u);
  for (int j0 = 0, j = 0; j0 < kb; j0 += W, j++) {
    const int w = min(W, kb - j0);
    if (warp == 0) {
      T P[W][2];
#pragma unroll
      for (int k = 0; k < W; k++) {
        P[k][0] = D[lane][j0 + k];
        P[k][1] = D[lane + 32][j0 + k];
      }
#pragma unroll
      for (int k = 0; k < W; k++) {
        if (k >= w) break;
        const T v0 = P[k][0], v1 = P[k][1];
        const R m0 = v0.x * v0.x + v0.y * v0.y, m1 = v1.x * v1.x + v1.y * v1.y;
        const bool ok0 = !(used & 1u) && m0 >= (R)0, ok1 = !(used & 2u) && m1 >= (R)0;  // NaN never wins
        // |v|^2 >= 0 orders like its bit pattern
        // |v|^2 >= 0 orders like its bit pattern; the row rides in the low
        // six bits (63 - row: ties, to 2^-17 relative, go to the lowest row)
        const unsigned key0 = ok0 ? (__float_as_uint((float)m0) & ~63u) | (unsigned)(63 - lane) : 0u;
        const unsigned key1 = ok1 ? (__float_as_uint((float)m1) & ~63u) | (unsigned)(31 - lane) : 0u;
        const unsigned kmax = __reduce_max_sync(FULL, key0 > key1 ? key0 : key1);
        int p;
        if (kmax > 63u) {
          p = 63 - (int)(kmax & 63u);
        } else {  // all zero, or no finite candidate: go on with the first free row
          const unsigned any = __ballot_sync(FULL, ok0 || ok1);
          if (lane == 0) atomicOr(status, any ? kLuStatSingular : kLuStatNonFinite);
          const unsigned f0 = __ballot_sync(FULL, !(used & 1u)), f1 = __ballot_sync(FULL, !(used & 2u));
          p = f0 ? __ffs(f0) - 1 : 32 + __ffs(f1) - 1;
        }
        const int pl = p & 31;
        const bool ph = p >= 32;
        // the pivot and the pivot row's later panel entries, from lane pl
        const T ps = ph ? v1 : v0;
        T pv, u[W];
        pv.x = __shfl_sync(FULL, ps.x, pl);
        pv.y = __shfl_sync(FULL, ps.y, pl);
#pragma unroll
        for (int k2 = k + 1; k2 < W; k2++) {
          const T us = ph ? P[k2][1] : P[k2][0];
          u[k2].x = __shfl_sync(FULL, us.x, pl);
          u[k2].y = __shfl_sync(FULL, us.y, pl);
        }
        if (lane == pl) used |= ph ? 2u : 1u;
        // 1/pv = conj(pv) / |pv|^2, with Smith's division outside the safe range
        const R d2 = pv.x * pv.x + pv.y * pv.y;
        T pinv;
        if (d2 > (R)1e-30 && d2 < (R)1e30) {
          const R rr = pivot_rcp(d2);
          pinv.x = pv.x * rr;
          pinv.y = -pv.y * rr;
        } else {
          pinv = crecip(pv);
        }
        if (!(used & 1u)) P[k][0] = cmul(v0, pinv);
        if (!(used & 2u)) P[k][1] = cmul(v1, pinv);
#pragma unroll
        for (int k2 = k + 1; k2 < W; k2++) {
          if (!(used & 1u)) {
            P[k2][0].x -= P[k][0].x * u[k2].x - P[k][0].y * u[k2].y;
            P[k2][0].y -= P[k][0].x * u[k2].y + P[k][0].y * u[k2].x;
          }
          if (!(used & 2u)) {
            P[k2][1].x -= P[k][1].x * u[k2].x - P[k][1].y * u[k2].y;
            P[k2][1].y -= P[k][1].x * u[k2].y + P[k][1].y * u[k2].x;
          }
        }
        if (lane == 0) {
          s_seq[j0 + k] = p;
          dinv[j0 + k] = pinv;
        }
      }
#pragma unroll
      for (int k = 0; k < W; k++) {
        if (k < w) {
          D[lane][j0 + k] = P[k][0];
          D[lane + 32][j0 + k] = P[k][1];
        }
      }
      s_used[j & 1][lane] = (unsigned char)(used & 1u);
      s_used[j & 1][lane + 32] = (unsigned char)((used >> 1) & 1u);
    } else if (j > 0) {
      // lookahead: the previous panel's update of the columns beyond this
      // panel, and its interchanges
      update(t - 32, kDiagThreads - 32, j0 - W, W, s_used[(j - 1) & 1], j0 + W, kb);
      if (t == kDiagThreads - 32)
        for (int c = j0 - W; c < j0; c++) record(c);
    }
    __syncthreads();
    const int q0 = j0 + w, nq = kb - q0;  // trailing columns
    if (nq <= 0) continue;
    // U rows of the panel's pivots on the trailing columns
    if (t < nq) {
      // every load before the first store (the stores may alias the loads'
      // rows for all the compiler knows)
      const int q = q0 + t;
      int pr[W];
      T u[W];
#pragma unroll
      for (int i = 0; i < W; i++) pr[i] = i < w ? s_seq[j0 + i] : 0;
#pragma unroll
      for (int i = 0; i < W; i++) u[i] = D[pr[i]][q];
#pragma unroll
      for (int i = 1; i < W; i++)
#pragma unroll
        for (int k = 0; k < i; k++) {
          const T lk = D[pr[i]][j0 + k];
          u[i].x -= lk.x * u[k].x - lk.y * u[k].y;
          u[i].y -= lk.x * u[k].y + lk.y * u[k].x;
        }
#pragma unroll
      for (int i = 0; i < W; i++)
        if (i < w) D[pr[i]][q] = u[i];
    }
    __syncthreads();
    // this panel's update of the next panel's columns: column q0 + (t & 7),
    // rows t >> 3 and (t >> 3) + 32
    {
      const int q = q0 + (t & 7), r = t >> 3;
      if (q < kb && q < q0 + W) {
        const unsigned char* used_j = s_used[j & 1];
        int pr[W];
        T u[W];
#pragma unroll
        for (int k = 0; k < W; k++) pr[k] = k < w ? s_seq[j0 + k] : 0;
#pragma unroll
        for (int k = 0; k < W; k++) u[k] = k < w ? D[pr[k]][q] : czero<T>();
        const bool act_a = r < kb && !used_j[r], act_b = r + 32 < kb && !used_j[r + 32];
        T a = D[r][q], b = D[r + 32][q];
#pragma unroll
        for (int k = 0; k < W; k++) {
          const T la = D[r][j0 + k], lb = D[r + 32][j0 + k];
          a.x -= la.x * u[k].x - la.y * u[k].y;
          a.y -= la.x * u[k].y + la.y * u[k].x;
          b.x -= lb.x * u[k].x - lb.y * u[k].y;
          b.y -= lb.x * u[k].y + lb.y * u[k].x;
        }
        if (act_a) D[r][q] = a;
        if (act_b) D[r + 32][q] = b;
      }
    }
    __syncthreads();
  }
  if (t == 0)
    for (int c = (kb - 1) / W * W; c < kb; c++) record(c);  // the last panel's interchanges
  if (t < kb) src[k0 + t] = s_seq[t];
  for (int c = kb + t; c < NB; c += kDiagThreads) dinv[c] = czero<T>();
  // row c of the factors is physical row s_seq[c]
#pragma unroll
  for (int i = 0; i < PER; i++) {
    const int e = t + i * kDiagThreads, r = e / NB, c = e % NB;
    if (r < kb && c < kb) M[(k0 + r) * ld + k0 + c] = D[s_seq[r]][c];
  }
}

// Panel triangular solves with one 64-vector per thread, staged through
// shared memory with coalesced rows:
//   RIGHT: rows [s0, n) of the panel columns at k0:  x <- x U11^-1 (L21)
//   LEFT:  columns [s0, n) of the panel rows at k0:   x <- L11^-1 x (U12)
// Both are the row-vector solve x <- x T^-1 with T upper triangular (U11,
// or L11 transposed with a unit diagonal), done in 8 x 8 register blocks so
// the loop body stays small (a fully unrolled 64 x 64 solve outgrows the
// instruction cache).
constexpr int kTrsmW = 128;  // vectors per CTA (= threads)
template <typename T>
constexpr size_t trsm_panel_smem() {
  return (size_t)(kBlk * (kBlk + 1) + kTrsmW * (kBlk + 1) + kBlk) * sizeof(T);
}

// The tensor-core update's packed operands (gemm_tc.cuh, format F), written
// by the panel solves that produce them instead of by separate packing
// passes; kdim = F::kKMul * 64 (one 64-wide panel), the layouts of
// pack_a_kernel and pack_b_kernel.
template <class F>
__device__ __forceinline__ void emit_a(typename F::T* Ap, int64_t row, int k, float2 a) {
  tc::put_a<F>(Ap + row * (F::kKMul * kBlk), kBlk, k, a);
}
// eight consecutive k (k0 a multiple of 8) of column j of B: 16-byte stores
// (kbp: the operand's K per part, a multiple of 64)
template <class F>
__device__ __forceinline__ void emit_b8(typename F::T* Bp, int64_t j, int k0, const float2 (&b)[8], int kbp = kBlk) {
  typename F::T* re = Bp + (2 * j) * (F::kKMul * (int64_t)kbp) + k0;
  typename F::T* im = re + F::kKMul * kbp;
  if constexpr (F::kFormat == 2) {
    __align__(16) float v[4][8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const float br = tc::to_tf32(b[i].x), bi = tc::to_tf32(b[i].y);
      v[0][i] = br, v[1][i] = -bi, v[2][i] = bi, v[3][i] = br;
    }
#pragma unroll
    for (int s = 0; s < 2; s++) {
      *reinterpret_cast<uint4*>(re + s * kbp) = *reinterpret_cast<const uint4*>(&v[s][0]);
      *reinterpret_cast<uint4*>(re + s * kbp + 4) = *reinterpret_cast<const uint4*>(&v[s][4]);
      *reinterpret_cast<uint4*>(im + s * kbp) = *reinterpret_cast<const uint4*>(&v[2 + s][0]);
      *reinterpret_cast<uint4*>(im + s * kbp + 4) = *reinterpret_cast<const uint4*>(&v[2 + s][4]);
    }
  } else {
    __align__(16) __nv_bfloat16 v[12][8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      __nv_bfloat16 rh, rl, ih, il;
      tc::split_bf16(b[i].x, rh, rl);
      tc::split_bf16(b[i].y, ih, il);
      const __nv_bfloat16 nih = __hneg(ih), nil = __hneg(il);
      v[0][i] = rh, v[1][i] = nih, v[2][i] = rl, v[3][i] = nil, v[4][i] = rh, v[5][i] = nih;
      v[6][i] = ih, v[7][i] = rh, v[8][i] = il, v[9][i] = rl, v[10][i] = ih, v[11][i] = rh;
    }
#pragma unroll
    for (int s = 0; s < 6; s++) {
      *reinterpret_cast<uint4*>(re + s * kbp) = *reinterpret_cast<const uint4*>(v[s]);
      *reinterpret_cast<uint4*>(im + s * kbp) = *reinterpret_cast<const uint4*>(v[6 + s]);
    }
  }
}

template <typename T, bool LEFT, class F = tc::SplitBf16>
__global__ void __launch_bounds__(kTrsmW) trsm_panel_kernel(T* M, int64_t ld, int64_t n, int64_t k0, int64_t sbeg,
                                                            const T* dinv, typename F::T* Ap = nullptr,
                                                            int64_t abase = 0) {
  constexpr int NB = kBlk, W = kTrsmW, B = 8;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T(*Tri)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(smem_raw);
  T(*X)[NB + 1] = Tri + NB;
  T* di = reinterpret_cast<T*>(X + W);
  const int t = threadIdx.x;
  const int64_t s0 = sbeg + (int64_t)blockIdx.x * W;
  const int cnt = (int)min((int64_t)W, n - s0);
  // triangle: 32 elements per thread, loads batched by 8
  for (int b = 0; b < NB * NB / W; b += 8) {
    T v[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int e = t + (b + i) * W;
      v[i] = M[(k0 + e / NB) * ld + k0 + e % NB];
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int e = t + (b + i) * W, r = e / NB, c = e % NB;
      if (LEFT)
        Tri[c][r] = r > c ? v[i] : czero<T>();  // L11^T, strictly upper part
      else
        Tri[r][c] = v[i];
    }
  }
  if (!LEFT && t < NB) di[t] = dinv[t];
  // the vectors: 64 elements per thread, loads batched by 16
  for (int b = 0; b < NB; b += 16) {
    T v[16];
#pragma unroll
    for (int i = 0; i < 16; i++) {
      const int e = t + (b + i) * W;
      if (LEFT) {
        const int r = e / W, cc = e % W;
        v[i] = cc < cnt ? M[(k0 + r) * ld + s0 + cc] : czero<T>();
      } else {
        const int rr = e / NB, c = e % NB;
        v[i] = rr < cnt ? M[(s0 + rr) * ld + k0 + c] : czero<T>();
      }
    }
#pragma unroll
    for (int i = 0; i < 16; i++) {
      const int e = t + (b + i) * W;
      if (LEFT)
        X[e % W][e / W] = v[i];
      else
        X[e / NB][e % NB] = v[i];
    }
  }
  __syncthreads();
  T* x = X[t];
#pragma unroll 1
  for (int Q = 0; Q < NB; Q += B) {
    T xq[B];
#pragma unroll
    for (int i = 0; i < B; i++) xq[i] = x[Q + i];
#pragma unroll
    for (int i = 0; i < B; i++) {
      if (!LEFT) xq[i] = cmul(xq[i], di[Q + i]);
#pragma unroll
      for (int j = i + 1; j < B; j++) {
        const T u = Tri[Q + i][Q + j];
        xq[j].x -= xq[i].x * u.x - xq[i].y * u.y;
        xq[j].y -= xq[i].x * u.y + xq[i].y * u.x;
      }
    }
#pragma unroll
    for (int i = 0; i < B; i++) x[Q + i] = xq[i];
#pragma unroll 1
    for (int P = Q + B; P < NB; P += B) {
      T xp[B];
#pragma unroll
      for (int j = 0; j < B; j++) xp[j] = x[P + j];
#pragma unroll
      for (int i = 0; i < B; i++)
#pragma unroll
        for (int j = 0; j < B; j++) {
          const T u = Tri[Q + i][P + j];
          xp[j].x -= xq[i].x * u.x - xq[i].y * u.y;
          xp[j].y -= xq[i].x * u.y + xq[i].y * u.x;
        }
#pragma unroll
      for (int j = 0; j < B; j++) x[P + j] = xp[j];
    }
  }
  __syncthreads();
  for (int b = 0; b < NB; b += 16) {
#pragma unroll
    for (int i = 0; i < 16; i++) {
      const int e = t + (b + i) * W;
      if (LEFT) {
        const int r = e / W, cc = e % W;
        if (cc < cnt) M[(k0 + r) * ld + s0 + cc] = X[cc][r];
      } else {
        const int rr = e / NB, c = e % NB;
        if (rr < cnt) {
          M[(s0 + rr) * ld + k0 + c] = X[rr][c];
          // L21 rows are the A operand of the update that follows
          if constexpr (!LEFT && std::is_same<T, float2>::value)
            if (Ap) emit_a<F>(Ap, s0 + rr - abase, c, X[rr][c]);
        }
      }
    }
  }
}

// The same panel solves with the 64 unknowns of a vector spread over eight
// warps: warp g holds block g (8 unknowns) of 32 vectors, one per lane.  In
// stage Q warp Q finishes its block (the 8 x 8 triangle, in registers) and
// posts it to shared memory; after one barrier every warp g > Q subtracts
// its contribution (64 complex multiply-adds per lane).  Eight stages
// replace the 64-step chain of one thread per vector.  The triangle is kept
// column-block-major with an odd stride per block so that the eight warps
// of a stage read distinct banks.  kb = 64 (callers solve full blocks).
constexpr int kTrsm8Vec = 32;  // vectors per CTA per lane slot
constexpr int kTrsm8TriStride = kBlk * 9 + 1;
template <typename T, int VPL = 1>
constexpr size_t trsm8_smem() {
  return (size_t)(8 * kTrsm8TriStride + 8 * VPL * kTrsm8Vec * 9 + kBlk) * sizeof(T);
}

// VPL vectors per lane: 32 * VPL vectors per CTA share one triangle load.
template <typename T, bool LEFT, int VPL = 1, class F = tc::SplitBf16>
__global__ void __launch_bounds__(256) trsm8_panel_kernel(T* M, int64_t ld, int64_t n, int64_t k0, int64_t sbeg,
                                                          const T* dinv, typename F::T* Bp = nullptr,
                                                          int64_t bbase = 0) {
  constexpr int NB = kBlk, V = kTrsm8Vec * VPL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Tri = reinterpret_cast<T*>(smem_raw);             // element (i, j) at (j>>3)*stride + i*9 + (j&7)
  T* Xs = Tri + 8 * kTrsm8TriStride;                   // finished blocks: (Q * V + vector) * 9 + i
  T* di = Xs + 8 * V * 9;
  const int t = threadIdx.x, lane = t & 31, g = t >> 5;
  // triangle (RIGHT: U11 upper; LEFT: L11 transposed, strictly upper)
  for (int e = t; e < NB * NB; e += 256) {
    const int r = e / NB, c = e % NB;
    const T v = M[(k0 + r) * ld + k0 + c];
    if (LEFT)
      Tri[(r >> 3) * kTrsm8TriStride + c * 9 + (r & 7)] = r > c ? v : czero<T>();
    else
      Tri[(c >> 3) * kTrsm8TriStride + r * 9 + (c & 7)] = v;
  }
  if (!LEFT && t < NB) di[t] = dinv[t];
  // this thread's block of its vectors (vector slot s = lane + 32 * w)
  T acc[VPL][8];
  int64_t vec[VPL];
  bool valid[VPL];
#pragma unroll
  for (int w = 0; w < VPL; w++) {
    vec[w] = sbeg + (int64_t)blockIdx.x * V + lane + 32 * w;
    valid[w] = vec[w] < n;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int c = g * 8 + j;
      acc[w][j] = valid[w] ? (LEFT ? M[(k0 + c) * ld + vec[w]] : M[vec[w] * ld + k0 + c]) : czero<T>();
    }
  }
  __syncthreads();
#pragma unroll 1
  for (int Q = 0; Q < 8; Q++) {
    if (g == Q) {
      // the diagonal 8 x 8 triangle of block Q
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const T dq = LEFT ? czero<T>() : di[Q * 8 + i];
#pragma unroll
        for (int w = 0; w < VPL; w++)
          if (!LEFT) acc[w][i] = cmul(acc[w][i], dq);
#pragma unroll
        for (int j = i + 1; j < 8; j++) {
          const T u = Tri[Q * kTrsm8TriStride + (Q * 8 + i) * 9 + j];
#pragma unroll
          for (int w = 0; w < VPL; w++) {
            acc[w][j].x -= acc[w][i].x * u.x - acc[w][i].y * u.y;
            acc[w][j].y -= acc[w][i].x * u.y + acc[w][i].y * u.x;
          }
        }
      }
#pragma unroll
      for (int w = 0; w < VPL; w++)
#pragma unroll
        for (int i = 0; i < 8; i++) Xs[(Q * V + lane + 32 * w) * 9 + i] = acc[w][i];
    }
    __syncthreads();
    if (g > Q) {
      const T* tb = Tri + g * kTrsm8TriStride + (Q * 8) * 9;
#pragma unroll
      for (int i = 0; i < 8; i++) {
        T x[VPL];
#pragma unroll
        for (int w = 0; w < VPL; w++) x[w] = Xs[(Q * V + lane + 32 * w) * 9 + i];
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const T u = tb[i * 9 + j];
#pragma unroll
          for (int w = 0; w < VPL; w++) {
            acc[w][j].x -= x[w].x * u.x - x[w].y * u.y;
            acc[w][j].y -= x[w].x * u.y + x[w].y * u.x;
          }
        }
      }
    }
  }
#pragma unroll
  for (int w = 0; w < VPL; w++) {
    if (!valid[w]) continue;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int c = g * 8 + j;
      if (LEFT)
        M[(k0 + c) * ld + vec[w]] = acc[w][j];
      else
        M[vec[w] * ld + k0 + c] = acc[w][j];
    }
    // U12 columns are the B operand of the update that follows
    if constexpr (LEFT && std::is_same<T, float2>::value)
      if (Bp) emit_b8<F>(Bp, vec[w] - bbase, g * 8, acc[w]);
  }
}

// Row-block solves X <- X U11^-1 (L21 rows) and Y <- L11^-1 Y (U12
// columns) against a 64 x 64 LU staged in shared memory, left-looking by
// 8-column blocks with every thread on the current block.  The eight 8 x 8
// diagonal blocks are inverted first (W_b = U_bb^-1 with the reciprocal
// diagonal, V_b = L_bb^-1, one column per lane), so that a block is
//   pair (row, j):  a_j = A_j - sum_{k < 8b} X_k U_kj        (dot product)
//                   x_j = sum_{i <= j} a_i W_b[i][j]           (8-lane shuffles)
// and one barrier separates two blocks.  The operands of the dot products
// are stored with k contiguous (U transposed, U12 columns transposed) and
// read two k at a time with 16-byte loads; rows of kS = 66 elements keep
// those loads aligned and free of bank conflicts across eight rows.
constexpr int kS = kBlk + 2;

__device__ __forceinline__ void named_barrier(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}
__device__ __forceinline__ float2 ld2(const float2* p) { return *p; }
__device__ __forceinline__ void csub(float2& a, float2 x, float2 y) {  // a -= x y
  a.x -= x.x * y.x - x.y * y.y;
  a.y -= x.x * y.y + x.y * y.x;
}
__device__ __forceinline__ void cadd(float2& a, float2 x, float2 y) {  // a += x y
  a.x += x.x * y.x - x.y * y.y;
  a.y += x.x * y.y + x.y * y.x;
}
// a -= sum_{k < n2 * 2} p[k] q[k], both 16-byte aligned, two accumulators
__device__ __forceinline__ float2 dot_sub(float2 a, const float2* p, const float2* q, int n2) {
  float2 b = make_float2(0.f, 0.f);
#pragma unroll 4
  for (int k = 0; k < n2; k++) {
    const float4 u = reinterpret_cast<const float4*>(p)[k], v = reinterpret_cast<const float4*>(q)[k];
    csub(a, make_float2(u.x, u.y), make_float2(v.x, v.y));
    csub(b, make_float2(u.z, u.w), make_float2(v.z, v.w));
  }
  return make_float2(a.x + b.x, a.y + b.y);
}
// W_b = U_bb^-1 (U_ii^-1 = di[i]), column j = lane of warp b (lanes 0-7):
// w_i = (delta_ij - sum_{i < m <= j} U_im w_m) di_i, for i = j down to 0.
// Ut[j][k] = U[k][j]; W[(b * 8 + i) * 8 + j].
__device__ __forceinline__ void invert_u_block(const float2* Ut, const float2* di, float2* W, int b, int j) {
  float2 w[8];
#pragma unroll
  for (int i = 7; i >= 0; i--) {
    float2 v = make_float2(i == j ? 1.f : 0.f, 0.f);
#pragma unroll
    for (int m = i + 1; m < 8; m++)
      if (m <= j) csub(v, Ut[(8 * b + m) * kS + 8 * b + i], w[m]);
    w[i] = i <= j ? cmul(v, di[8 * b + i]) : make_float2(0.f, 0.f);
  }
#pragma unroll
  for (int i = 0; i < 8; i++) W[(b * 8 + i) * 8 + j] = w[i];
}
// V_b = L_bb^-1 (unit lower), column m = lane - 8 of warp b (lanes 8-15):
// v_m = 1, v_i = -sum_{m <= q < i} L_iq v_q.  Dl[i][k] = L[i][k];
// V[(b * 8 + i) * 8 + m].
__device__ __forceinline__ void invert_l_block(const float2* Dl, float2* V, int b, int m) {
  float2 v[8];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    float2 a = make_float2(i == m ? 1.f : 0.f, 0.f);
#pragma unroll
    for (int q = 0; q < i; q++)
      if (q >= m) csub(a, Dl[(8 * b + i) * kS + 8 * b + q], v[q]);
    v[i] = i >= m ? a : make_float2(0.f, 0.f);
  }
#pragma unroll
  for (int i = 0; i < 8; i++) V[(b * 8 + i) * 8 + m] = v[i];
}
// block b of an L21 row: pair (row r, column j = lane & 7); X rows of kS
__device__ __forceinline__ void l21_step(float2* X, const float2* Ut, const float2* W, int b, int r, int lane) {
  const int j = lane & 7;
  const float2 a = dot_sub(X[r * kS + 8 * b + j], X + r * kS, Ut + (8 * b + j) * kS, 4 * b);
  float2 x = make_float2(0.f, 0.f);
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const float2 ai = make_float2(__shfl_sync(0xffffffffu, a.x, (lane & ~7) + i),
                                  __shfl_sync(0xffffffffu, a.y, (lane & ~7) + i));
    cadd(x, ai, W[(b * 8 + i) * 8 + j]);
  }
  X[r * kS + 8 * b + j] = x;
}
// staging of the panel's LU: element (r, c) into Ut[c][r] (r <= c) or
// Dl[r][c] (r > c, when Dl is given); 16-byte loads of two columns
__device__ __forceinline__ void stage_lu(const float2* M, int64_t ld, int64_t k0, float2* Ut, float2* Dl,
                                         const float4* v, int t, int nthreads, int nv) {
  for (int i = 0; i < nv; i++) {
    const int e = t + i * nthreads;
    if (e >= kBlk * kBlk / 2) break;
    const int r = e / 32, c = (e % 32) * 2;
    const float2 a0 = make_float2(v[i].x, v[i].y), a1 = make_float2(v[i].z, v[i].w);
    if (r <= c) Ut[c * kS + r] = a0; else if (Dl) Dl[r * kS + c] = a0;
    if (r <= c + 1) Ut[(c + 1) * kS + r] = a1; else if (Dl) Dl[r * kS + c + 1] = a1;
  }
}

// The rest of an outer block's rows and columns for a 64-wide inner panel,
// in one launch.  For the panel at k0, whose LU is in M[k0.., k0..] with
// its rows in pivot order and whose row order is src_rows[k0 + r] (the
// block row that ends up in row r), r0 = k0 + 64 and the outer block's end
// c_hi:
//   L21 rows [r0, c_hi):   X = A[rows, k0..k0+64) U11^-1
//   U12 columns J:          Y = L11^-1 A[k0.., J], the panel's rows taken in
//                           pivot order (the gather of laswp_block_kernel)
//   A[rows, J] -= X Y
// CTA (x, h) takes the 16 columns J = [r0 + 16x, ...) and the 32 rows
// [r0 + 32h, ...), both below c_hi.  Warps 0-7 solve the L21 rows (pair =
// row, column of the block), warps 8-11 the U12 columns (pair = column, row
// of the block; the 8 rows of a column in consecutive lanes), and the
// update is accumulated block by block as X and Y blocks are finished, two
// entries per L21 thread.  Each CTA solves the L21 rows of its row group
// and the U12 columns of its column group; the results are stored by the
// last CTA to load among those that read the same inputs (an arrival
// counter per row group and per column group, reset by that CTA), so no CTA
// overwrites an input another CTA has yet to load.  Warp 12 counts the CTA
// in once its loads are done, outside the solve's barriers.  The U12
// columns also go out as the bulk update's packed B operand (column j -
// r0).  The caller guarantees k0 + 64 <= n and c_hi <= n; cnt holds
// kTopRowGroups + gridDim.x zeroed counters, gridDim.y <= kTopRowGroups.
constexpr int kTopCols = 16, kTopRows = 32;
constexpr int kTopSolveThreads = 384;
constexpr int kTopThreads = kTopSolveThreads + 32;
constexpr int kTopRowGroups = 32;  // row groups of 32 (outer blocks up to 1088 columns)
constexpr int kTopCnt = 128;       // counters the caller provides
__host__ __device__ constexpr size_t panel_top_smem() {
  return (size_t)(2 * kBlk * kS + kTopRows * kS + kTopCols * kS + 2 * 8 * 64 + kBlk) * sizeof(float2);
}
template <class F>
__global__ void __launch_bounds__(kTopThreads) panel_top_kernel(float2* M, int64_t ld, int64_t k0, int64_t c_hi,
                                                                 const int* src_rows, const float2* dinv,
                                                                 typename F::T* Bp, unsigned* cnt) {
  constexpr int NB = kBlk, NT = kTopSolveThreads;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* Ut = reinterpret_cast<float2*>(smem_raw);  // U11 transposed
  float2* Dl = Ut + NB * kS;                         // L11
  float2* X = Dl + NB * kS;                          // L21 rows
  float2* Yt = X + kTopRows * kS;                    // U12 columns, transposed
  float2* W = Yt + kTopCols * kS;                    // inverted diagonal blocks of U11
  float2* V = W + 8 * 64;                            // and of L11
  float2* di = V + 8 * 64;
  __shared__ int s_last[2];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int64_t r0 = k0 + NB;
  const int64_t j0 = r0 + (int64_t)blockIdx.x * kTopCols;
  const int64_t row0 = r0 + (int64_t)blockIdx.y * kTopRows;
  const int lr = t >> 3, lc = 2 * (t & 7);  // C pair (t < 256): row lr, columns lc, lc + 1
  const bool crow = t < 256 && row0 + lr < c_hi;
  float2 cc[2] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
  if (t < NT) {
    // all loads in flight before the first shared-memory store
    float4 dv[6], xv[3];
    float2 yv[3];
#pragma unroll
    for (int i = 0; i < 6; i++) {
      const int e = t + i * NT;
      if (e < NB * NB / 2) dv[i] = *reinterpret_cast<const float4*>(M + (k0 + e / 32) * ld + k0 + (e % 32) * 2);
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const int e = t + i * NT;
      if (e < kTopRows * NB / 2)
        xv[i] = row0 + e / 32 < c_hi ? *reinterpret_cast<const float4*>(M + (row0 + e / 32) * ld + k0 + (e % 32) * 2)
                                     : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const int e = t + i * NT;
      if (e < NB * kTopCols) {
        const int s = min(max(src_rows[k0 + e / kTopCols], 0), NB - 1);
        const int64_t c = j0 + e % kTopCols;
        yv[i] = c < c_hi ? M[(k0 + s) * ld + c] : czero<float2>();
      }
    }
    if (t < 256) {
#pragma unroll
      for (int m = 0; m < 2; m++) {
        const int64_t c = j0 + lc + m;
        cc[m] = crow && c < c_hi ? M[(row0 + lr) * ld + c] : czero<float2>();
      }
    }
    if (t < NB) di[t] = dinv[t];
    stage_lu(M, ld, k0, Ut, Dl, dv, t, NT, 6);
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const int e = t + i * NT;
      if (e < kTopRows * NB / 2) {
        X[(e / 32) * kS + (e % 32) * 2] = make_float2(xv[i].x, xv[i].y);
        X[(e / 32) * kS + (e % 32) * 2 + 1] = make_float2(xv[i].z, xv[i].w);
      }
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const int e = t + i * NT;
      if (e < NB * kTopCols) Yt[(e % kTopCols) * kS + e / kTopCols] = yv[i];
    }
  }
  __syncthreads();  // every load of this CTA is behind it
  if (warp == NT / 32) {
    // count the CTA in; learn whether it is the last of its row group and
    // of its column group
    if (lane == 0) {
      __threadfence();
      const unsigned a = atomicAdd(&cnt[blockIdx.y], 1u);
      const unsigned c = atomicAdd(&cnt[kTopRowGroups + blockIdx.x], 1u);
      s_last[0] = a == gridDim.x - 1;
      s_last[1] = c == gridDim.y - 1;
      if (s_last[0]) cnt[blockIdx.y] = 0;
      if (s_last[1]) cnt[kTopRowGroups + blockIdx.x] = 0;
      __threadfence();
    }
  } else {
    if (warp < 8) {
      if (lane < 8)
        invert_u_block(Ut, di, W, warp, lane);
      else if (lane < 16)
        invert_l_block(Dl, V, warp, lane - 8);
    }
    named_barrier(1, NT);
    const int uc = (t - 256) >> 3, ui = t & 7;  // U12 pair (t >= 256): column uc, row ui of the block
#pragma unroll 1
    for (int b = 0; b < 8; b++) {
      if (t < 256) {
        if (b > 0) {  // C -= X_q Y_q for the block finished last
#pragma unroll
          for (int k = 0; k < 8; k += 2) {
            const float4 x = *reinterpret_cast<const float4*>(X + lr * kS + 8 * (b - 1) + k);
#pragma unroll
            for (int m = 0; m < 2; m++) {
              const float4 y = *reinterpret_cast<const float4*>(Yt + (lc + m) * kS + 8 * (b - 1) + k);
              csub(cc[m], make_float2(x.x, x.y), make_float2(y.x, y.y));
              csub(cc[m], make_float2(x.z, x.w), make_float2(y.z, y.w));
            }
          }
        }
        l21_step(X, Ut, W, b, lr, lane);
      } else {
        const float2 a = dot_sub(Yt[uc * kS + 8 * b + ui], Dl + (8 * b + ui) * kS, Yt + uc * kS, 4 * b);
        float2 y = make_float2(0.f, 0.f);
#pragma unroll
        for (int m = 0; m < 8; m++) {
          const float2 am = make_float2(__shfl_sync(0xffffffffu, a.x, (lane & ~7) + m),
                                        __shfl_sync(0xffffffffu, a.y, (lane & ~7) + m));
          cadd(y, V[(b * 8 + ui) * 8 + m], am);
        }
        Yt[uc * kS + 8 * b + ui] = y;
      }
      named_barrier(1, NT);
    }
    if (t < 256) {
#pragma unroll
      for (int k = 0; k < 8; k += 2) {
        const float4 x = *reinterpret_cast<const float4*>(X + lr * kS + 56 + k);
#pragma unroll
        for (int m = 0; m < 2; m++) {
          const float4 y = *reinterpret_cast<const float4*>(Yt + (lc + m) * kS + 56 + k);
          csub(cc[m], make_float2(x.x, x.y), make_float2(y.x, y.y));
          csub(cc[m], make_float2(x.z, x.w), make_float2(y.z, y.w));
        }
      }
    }
  }
  __syncthreads();
  if (s_last[0] && t < NT) {
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const int e = t + i * NT;
      if (e < kTopRows * NB / 2 && row0 + e / 32 < c_hi) {
        const float2 a0 = X[(e / 32) * kS + (e % 32) * 2], a1 = X[(e / 32) * kS + (e % 32) * 2 + 1];
        *reinterpret_cast<float4*>(M + (row0 + e / 32) * ld + k0 + (e % 32) * 2) = make_float4(a0.x, a0.y, a1.x, a1.y);
      }
    }
  }
  if (s_last[1] && t < NB * kTopCols / 8) {  // one column and eight rows per thread
    const int c = t % kTopCols, g = t / kTopCols;
    const int64_t col = j0 + c;
    if (col < c_hi) {
      float2 yb[8];
#pragma unroll
      for (int i = 0; i < 8; i++) {
        yb[i] = Yt[c * kS + 8 * g + i];
        M[(k0 + 8 * g + i) * ld + col] = yb[i];
      }
      if (Bp) emit_b8<F>(Bp, col - r0, g * 8, yb);
    }
  }
  if (crow) {
#pragma unroll
    for (int m = 0; m < 2; m++) {
      const int64_t c = j0 + lc + m;
      if (c < c_hi) M[(row0 + lr) * ld + c] = cc[m];
    }
  }
}

// L21 rows [sbeg, n_end) of the panel at k0 (x <- x U11^-1) in the form of
// panel_top_kernel's L21 half, written back with the update's packed A'
// rows (row - abase) when Ap is given.  Persistent: a CTA stages the
// panel's U11 and its inverted diagonal blocks once and then takes 32-row
// chunks blockIdx.x, blockIdx.x + gridDim.x, ...; the next chunk's rows are
// loaded while the current one is written back.  A small grid keeps the
// solve, which only the trailing update waits for, on a few SMs beside the
// panel chain.
constexpr int kL21Rows = 32;
__host__ __device__ constexpr size_t l21_rows_smem() {
  return (size_t)(kBlk * kS + kL21Rows * kS + 8 * 64 + kBlk) * sizeof(float2);
}
template <class F>
__global__ void __launch_bounds__(256) l21_rows_kernel(float2* M, int64_t ld, int64_t n_end, int64_t k0,
                                                        int64_t sbeg, const float2* dinv, typename F::T* Ap,
                                                        int64_t abase) {
  constexpr int NB = kBlk;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* Ut = reinterpret_cast<float2*>(smem_raw);
  float2* X = Ut + NB * kS;
  float2* W = X + kL21Rows * kS;
  float2* di = W + 8 * 64;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int64_t nchunks = (n_end - sbeg + kL21Rows - 1) / kL21Rows;
  int64_t chunk = blockIdx.x;
  float4 xv[4];
  auto load_rows = [&](int64_t ch) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int e = t + i * 256;
      const int64_t row = sbeg + ch * kL21Rows + e / 32;
      xv[i] = ch < nchunks && row < n_end ? *reinterpret_cast<const float4*>(M + row * ld + k0 + (e % 32) * 2)
                                          : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };
  {
    float4 dv[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int e = t + i * 256;
      dv[i] = *reinterpret_cast<const float4*>(M + (k0 + e / 32) * ld + k0 + (e % 32) * 2);
    }
    load_rows(chunk);
    if (t < NB) di[t] = dinv[t];
    stage_lu(M, ld, k0, Ut, nullptr, dv, t, 256, 8);
  }
  __syncthreads();
  if (lane < 8) invert_u_block(Ut, di, W, warp, lane);
  for (; chunk < nchunks; chunk += gridDim.x) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int e = t + i * 256;
      X[(e / 32) * kS + (e % 32) * 2] = make_float2(xv[i].x, xv[i].y);
      X[(e / 32) * kS + (e % 32) * 2 + 1] = make_float2(xv[i].z, xv[i].w);
    }
    __syncthreads();
#pragma unroll 1
    for (int b = 0; b < 8; b++) {
      l21_step(X, Ut, W, b, t >> 3, lane);
      __syncthreads();
    }
    load_rows(chunk + gridDim.x);
    // write back: element (r, k) with consecutive k across a warp (coalesced
    // rows of M and of the packed A')
    const int64_t row0 = sbeg + chunk * kL21Rows;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int e = t + i * 256, r = e / NB, k = e % NB;
      const int64_t row = row0 + r;
      if (row < n_end) {
        const float2 v = X[r * kS + k];
        M[row * ld + k0 + k] = v;
        if (Ap) emit_a<F>(Ap, row - abase, k, v);
      }
    }
    __syncthreads();
  }
}

// Row interchanges of a block-pivoted panel: the kb <= 64 exchanges stay
// inside rows [k0, k0+kb), so each column is one gather of those rows
// (src[k0 + r]: the block row that ends up in row r).  A CTA covers 32
// columns of [c_lo, c_hi) with 8 row groups; all reads finish (barrier)
// before any write.  Columns [k0, skip_hi) (the diagonal block, and the
// columns panel_top_kernel gathers itself) are skipped.
template <typename T>
__global__ void __launch_bounds__(256) laswp_block_kernel(T* M, int64_t ld, int64_t c_lo, int64_t c_hi, int64_t k0,
                                                          int kb, const int* src_rows, int64_t skip_hi) {
  constexpr int NB = kBlk, RG = 8, PER = NB / RG;
  __shared__ int src[NB];
  const int t = threadIdx.x, tx = t & 31, g = t >> 5;
  if (t < NB) src[t] = t < kb ? min(max(src_rows[k0 + t], 0), NB - 1) : t;
  __syncthreads();
  const int64_t col = c_lo + (int64_t)blockIdx.x * 32 + tx;
  const bool act = col < c_hi && !(col >= k0 && col < skip_hi);
  T v[PER];
#pragma unroll
  for (int i = 0; i < PER; i++) {
    const int r = g + RG * i;
    if (act && r < kb && src[r] != r) v[i] = M[(k0 + src[r]) * ld + col];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < PER; i++) {
    const int r = g + RG * i;
    if (act && r < kb && src[r] != r) M[(k0 + r) * ld + col] = v[i];
  }
}

// U12 of an outer row block in one launch: rows [K0, K0 + nb*64), columns
// [c_lo, c_hi) of M, in place.  With `swap`, each 64-row block first takes
// the row order its diagonal LU chose (the gather of laswp_block_kernel,
// src_rows[r0 + r] = the block row that ends up in row r).  Then
// X = L^-1 A with the unit-lower diagonal block L = M[K0.., K0..] of the
// outer block, left-looking by 64-row blocks:
//     X_b = L_bb^-1 (A_b - sum_{j<b} L_bj X_j).
// One CTA per 16 columns, 8 warps; lane = column + 16 x half, and warp g
// holds rows 8g..8g+7 of the current block in registers, four per half.
// Finished rows stay in shared memory for the later blocks; each L tile is
// staged once per CTA.  The in-block solve runs in eight stages, one barrier
// each: warp Q finishes its 8 x 8 triangle (the upper half taking the lower
// half's four rows by shuffle) and posts its rows, warps g > Q fold them
// in.  Sixteen columns per CTA keep three CTAs on an SM and halve the
// sequential work of each.  This
// replaces, per outer block, the deferred interchanges of the far columns
// and a tensor-core update plus a panel solve for each 64-row block.
constexpr int kU12MaxBlocks = 8;  // outer blocks up to 512 columns
constexpr int kU12Cols = 16;      // columns per CTA
__host__ __device__ constexpr size_t u12_rows_smem(int nb) {
  return (size_t)(nb * kBlk * (kU12Cols + 1) + kBlk * (kBlk + 1)) * sizeof(float2);
}
template <class F>
__global__ void __launch_bounds__(256, 3) u12_rows_kernel(float2* M, int64_t ld, int64_t K0, int nb, int64_t c_lo,
                                                       int64_t c_hi, const int* src_rows, int swap,
                                                       typename F::T* Bp) {
  constexpr int NB = kBlk, CW = kU12Cols;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2(*Xs)[CW + 1] = reinterpret_cast<float2(*)[CW + 1]>(smem_raw);     // nb*64 finished rows x 16 columns
  float2(*Lt)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(Xs + nb * NB);  // one staged 64 x 64 tile of L
  __shared__ int src[NB];
  const int t = threadIdx.x, lane = t & 31, g = t >> 5;
  const int cl = lane & (CW - 1), h = lane >> 4;  // column in the tile, half of the warp's eight rows
  const int rb = 8 * g + 4 * h;                   // first of this thread's four rows
  const int64_t col = c_lo + (int64_t)blockIdx.x * CW + cl;
  const bool act = col < c_hi;
  // The L tiles in the order they are used, (b, j) for j = 0..b (j == b:
  // the diagonal tile), tile (b, j) = M[K0 + 64 b .., K0 + 64 j ..].  Each
  // one is loaded into registers while the one before is in use, then
  // posted to shared memory (stage).
  float2 pf[NB * NB / 256];
  auto fetch = [&](int tb, int tj) {
    const float2* src_t = M + (K0 + (int64_t)tb * NB) * ld + K0 + (int64_t)tj * NB;
#pragma unroll
    for (int i = 0; i < NB * NB / 256; i++) {
      const int e = t + i * 256;
      pf[i] = src_t[(int64_t)(e >> 6) * ld + (e & 63)];
    }
  };
  auto stage = [&](int tb, int tj) {  // post the fetched tile, fetch the next one
    __syncthreads();
#pragma unroll
    for (int i = 0; i < NB * NB / 256; i++) {
      const int e = t + i * 256;
      Lt[e >> 6][e & 63] = pf[i];
    }
    __syncthreads();
    const int nb_ = tj < tb ? tb : tb + 1, nj = tj < tb ? tj + 1 : 0;
    if (nb_ < nb) fetch(nb_, nj);
  };
  fetch(0, 0);
  for (int b = 0; b < nb; b++) {
    const int64_t r0 = K0 + (int64_t)b * NB;
    if (swap) {
      __syncthreads();
      if (t < NB) src[t] = min(max(src_rows[r0 + t], 0), NB - 1);
      __syncthreads();
    }
    float2 x[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int r = rb + i;
      x[i] = act ? M[(r0 + (swap ? src[r] : r)) * ld + col] : make_float2(0.f, 0.f);
    }
    for (int j = 0; j < b; j++) {
      stage(b, j);
#pragma unroll 4
      for (int k = 0; k < NB; k++) {
        const float2 xv = Xs[j * NB + k][cl];
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const float2 l = Lt[rb + i][k];
          x[i].x -= l.x * xv.x - l.y * xv.y;
          x[i].y -= l.x * xv.y + l.y * xv.x;
        }
      }
    }
    stage(b, b);  // the unit-lower diagonal block (its strict lower part is read)
#pragma unroll 1
    for (int Q = 0; Q < 8; Q++) {
      if (g == Q) {
        // the 8 x 8 triangle of rows 8Q..8Q+7: the lower half first solves
        // its 4 x 4 triangle, the upper half takes those four values from
        // the lane 16 below (same column) and then solves its own
        if (h == 0) {
#pragma unroll
          for (int i = 1; i < 4; i++)
#pragma unroll
            for (int k = 0; k < i; k++) {
              const float2 l = Lt[rb + i][rb + k];
              x[i].x -= l.x * x[k].x - l.y * x[k].y;
              x[i].y -= l.x * x[k].y + l.y * x[k].x;
            }
        }
        float2 y[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
          y[k].x = __shfl_sync(FULL, x[k].x, cl);
          y[k].y = __shfl_sync(FULL, x[k].y, cl);
        }
        if (h == 1) {
#pragma unroll
          for (int i = 0; i < 4; i++)
#pragma unroll
            for (int k = 0; k < 4; k++) {
              const float2 l = Lt[rb + i][8 * Q + k];
              x[i].x -= l.x * y[k].x - l.y * y[k].y;
              x[i].y -= l.x * y[k].y + l.y * y[k].x;
            }
#pragma unroll
          for (int i = 1; i < 4; i++)
#pragma unroll
            for (int k = 0; k < i; k++) {
              const float2 l = Lt[rb + i][rb + k];
              x[i].x -= l.x * x[k].x - l.y * x[k].y;
              x[i].y -= l.x * x[k].y + l.y * x[k].x;
            }
        }
#pragma unroll
        for (int i = 0; i < 4; i++) Xs[b * NB + rb + i][cl] = x[i];
      }
      __syncthreads();
      if (g > Q) {
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const float2 xv = Xs[b * NB + 8 * Q + k][cl];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const float2 l = Lt[rb + i][8 * Q + k];
            x[i].x -= l.x * xv.x - l.y * xv.y;
            x[i].y -= l.x * xv.y + l.y * xv.x;
          }
        }
      }
    }
    if (act) {
#pragma unroll
      for (int i = 0; i < 4; i++) M[(r0 + rb + i) * ld + col] = x[i];
    }
  }
  // the rows are the B operand of the trailing update (K = nb * 64): its
  // packed BF16 form, eight k per store, columns relative to c_lo (every
  // row of Xs was posted before the last stage's barrier)
  if (Bp && act) {
    for (int k8 = 2 * g + h; k8 < nb * 8; k8 += 16) {
      float2 bv[8];
#pragma unroll
      for (int i = 0; i < 8; i++) bv[i] = Xs[k8 * 8 + i][cl];
      emit_b8<F>(Bp, col - c_lo, k8 * 8, bv, nb * NB);
    }
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
