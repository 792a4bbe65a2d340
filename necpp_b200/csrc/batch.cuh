// Batched sweeps: many small structures (an optimiser's population, or a
// frequency sweep of several designs) solved together.  Each problem's
// fill, LU, refined solve, current coefficients and far field are the
// single-problem path's, but the work of all problems shares each launch:
//
//   batch_fill_kernel     one CTA per (problem, 64-row tile, 32-column tile)
//                         work item, through the single-problem fill tile
//   batch_lu_solve_kernel persistent: a CTA takes the next problem (largest
//                         first) from a counter and does its complex64 LU
//                         with partial pivoting (32-wide panels in shared
//                         memory, register-tiled trailing updates) and the
//                         solve refined in FP64 against the FP64 matrix
//   batch_coeff_kernel    basis amplitudes -> a, b, c and currents
//   batch_pattern_kernel  far field, one warp per (problem, direction)
#pragma once
#include <cstdint>

#include "fill.cuh"
#include "lu.cuh"
#include "pattern.cuh"

namespace necb {

constexpr int kBatchThreads = 256;
constexpr int kBatchNB = 32;      // LU panel width
constexpr int kBatchMaxN = 640;   // unknowns per problem on the batched path
constexpr long long kBatchRefineMax = 20;

struct BatchProblem {
  int n;
  int64_t z;  // element offset of the problem's n x n matrices (Z32, Z64)
  int64_t v;  // element offset of its vectors (rhs, x, perm)
};

// smem layout of batch_lu_solve_kernel (bytes)
constexpr size_t kBatchPanelBytes = (size_t)kBatchMaxN * (kBatchNB + 1) * sizeof(float2);
constexpr size_t kBatchUtBytes = (size_t)kBatchNB * (64 + 1) * sizeof(float2);
constexpr size_t kBatchSmem = kBatchPanelBytes + kBatchUtBytes + 2 * kBatchMaxN * sizeof(double2) + 256;

template <int GROUND, bool EXK>
__global__ void __launch_bounds__(kFillTI) batch_fill_kernel(const FillArgs* __restrict__ As,
                                                             const int4* __restrict__ items) {
  const int4 it = items[blockIdx.x];  // x problem, y row tile, z column tile
  fill_tile<GROUND, EXK, false>(As[it.x], ContractArgs{}, it.z, (int64_t)it.y * kFillTI);
}

// CTA-wide argmax of key (>= 0 candidates; -1 none), lowest row on ties.
__device__ __forceinline__ void cta_argmax(float key, int row, float* s_key, int* s_row, int* out_row,
                                           float* out_key) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const float ok = __shfl_xor_sync(0xffffffffu, key, off);
    const int orow = __shfl_xor_sync(0xffffffffu, row, off);
    if (ok > key || (ok == key && orow < row)) {
      key = ok;
      row = orow;
    }
  }
  if (lane == 0) {
    s_key[warp] = key;
    s_row[warp] = row;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float k = s_key[0];
    int r = s_row[0];
    for (int w = 1; w < kBatchThreads / 32; w++)
      if (s_key[w] > k || (s_key[w] == k && s_row[w] < r)) {
        k = s_key[w];
        r = s_row[w];
      }
    *out_row = r;
    *out_key = k;
  }
  __syncthreads();
}

// y <- (LU)^-1 P... : the two triangular solves of the factored A (n x n,
// row-major) on the complex64 vector y in shared memory, in place.
__device__ void batch_trsv(const float2* A, int n, float2* y) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  constexpr int B = 32;
  // forward, unit lower
  for (int j0 = 0; j0 < n; j0 += B) {
    const int jb = min(B, n - j0);
    if (warp == 0) {
      float2 v = lane < jb ? y[j0 + lane] : make_float2(0.f, 0.f);
      for (int c = 0; c < jb - 1; c++) {
        const float2 yc = make_float2(__shfl_sync(0xffffffffu, v.x, c), __shfl_sync(0xffffffffu, v.y, c));
        if (lane > c && lane < jb) {
          const float2 l = A[(int64_t)(j0 + lane) * n + j0 + c];
          v.x -= l.x * yc.x - l.y * yc.y;
          v.y -= l.x * yc.y + l.y * yc.x;
        }
      }
      if (lane < jb) y[j0 + lane] = v;
    }
    __syncthreads();
    for (int i = j0 + jb + t; i < n; i += kBatchThreads) {
      const float2* row = A + (int64_t)i * n + j0;
      float sr = 0.f, si = 0.f;
      for (int c = 0; c < jb; c++) {
        const float2 l = row[c], yc = y[j0 + c];
        sr += l.x * yc.x - l.y * yc.y;
        si += l.x * yc.y + l.y * yc.x;
      }
      y[i].x -= sr;
      y[i].y -= si;
    }
    __syncthreads();
  }
  // backward, upper
  for (int j0 = ((n - 1) / B) * B; j0 >= 0; j0 -= B) {
    const int jb = min(B, n - j0);
    if (warp == 0) {
      float2 v = lane < jb ? y[j0 + lane] : make_float2(0.f, 0.f);
      for (int c = jb - 1; c >= 0; c--) {
        if (lane == c) v = cdiv(v, A[(int64_t)(j0 + c) * n + j0 + c]);
        const float2 xc = make_float2(__shfl_sync(0xffffffffu, v.x, c), __shfl_sync(0xffffffffu, v.y, c));
        if (lane < c) {
          const float2 u = A[(int64_t)(j0 + lane) * n + j0 + c];
          v.x -= u.x * xc.x - u.y * xc.y;
          v.y -= u.x * xc.y + u.y * xc.x;
        }
      }
      if (lane < jb) y[j0 + lane] = v;
    }
    __syncthreads();
    for (int i = t; i < j0; i += kBatchThreads) {
      const float2* row = A + (int64_t)i * n + j0;
      float sr = 0.f, si = 0.f;
      for (int c = 0; c < jb; c++) {
        const float2 u = row[c], xc = y[j0 + c];
        sr += u.x * xc.x - u.y * xc.y;
        si += u.x * xc.y + u.y * xc.x;
      }
      y[i].x -= sr;
      y[i].y -= si;
    }
    __syncthreads();
  }
}

// Per problem (taken largest first from *next): LU of Z32 with partial
// pivoting, then x = Z^-1 b refined in FP64 against Z64 until the relative
// residual reaches tol or stops halving.  status[p]: 0 ok, 1 singular,
// 2 non-finite, 3 not converged (>1e-6); resid[p]: final relative residual.
__global__ void __launch_bounds__(kBatchThreads, 1)
    batch_lu_solve_kernel(int nprob, const int* order, const BatchProblem* probs, float2* Z32, const double2* Z64,
                          int* perm_pool, const double2* b_pool, double2* x_pool, double tol, int* next, int* status,
                          double* resid) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2(*P)[kBatchNB + 1] = reinterpret_cast<float2(*)[kBatchNB + 1]>(smem_raw);
  float2(*Ut)[64 + 1] = reinterpret_cast<float2(*)[64 + 1]>(smem_raw + kBatchPanelBytes);
  double2* xv = reinterpret_cast<double2*>(smem_raw + kBatchPanelBytes + kBatchUtBytes);
  double2* rv = xv + kBatchMaxN;
  float* s_key = reinterpret_cast<float*>(rv + kBatchMaxN);
  int* s_row = reinterpret_cast<int*>(s_key + kBatchThreads / 32);
  __shared__ int s_prob, s_p, s_bad;
  __shared__ float s_k;
  __shared__ double s_red[kBatchThreads / 32][2];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (;;) {
    if (t == 0) {
      const int q = atomicAdd(next, 1);
      s_prob = q < nprob ? order[q] : -1;
      s_bad = 0;
    }
    __syncthreads();
    const int p = s_prob;
    if (p < 0) return;
    const BatchProblem pr = probs[p];
    const int n = pr.n;
    float2* A = Z32 + pr.z;
    int* piv = perm_pool + pr.v;  // pivots during the LU, then the permutation
    // ---------------- LU with partial pivoting ----------------
    for (int k0 = 0; k0 < n; k0 += kBatchNB) {
      const int kb = min(kBatchNB, n - k0), rows = n - k0;
      for (int e = t; e < rows * kBatchNB; e += kBatchThreads) {
        const int r = e / kBatchNB, c = e % kBatchNB;
        P[r][c] = c < kb ? A[(int64_t)(k0 + r) * n + k0 + c] : make_float2(0.f, 0.f);
      }
      __syncthreads();
      for (int c = 0; c < kb; c++) {
        float best = -1.f;
        int brow = c;
        for (int r = c + t; r < rows; r += kBatchThreads) {
          const float2 v = P[r][c];
          const float a = v.x * v.x + v.y * v.y;
          if (a > best) {
            best = a;
            brow = r;
          }
        }
        cta_argmax(best, brow, s_key, s_row, &s_p, &s_k);
        int pc = s_p;
        if (!(s_k > 0.f)) {
          if (t == 0) s_bad = s_k == 0.f ? 1 : 2;
          pc = c;
        }
        if (pc != c && t < kBatchNB) {
          const float2 a = P[c][t];
          P[c][t] = P[pc][t];
          P[pc][t] = a;
        }
        if (t == 0) piv[k0 + c] = k0 + pc;
        __syncthreads();
        const float2 pinv = crecip(P[c][c]);
        for (int r = c + 1 + t; r < rows; r += kBatchThreads) {
          const float2 l = cmul(P[r][c], pinv);
          P[r][c] = l;
          for (int q = c + 1; q < kb; q++) {
            const float2 u = P[c][q];
            P[r][q].x -= l.x * u.x - l.y * u.y;
            P[r][q].y -= l.x * u.y + l.y * u.x;
          }
        }
        __syncthreads();
      }
      for (int e = t; e < rows * kBatchNB; e += kBatchThreads) {
        const int r = e / kBatchNB, c = e % kBatchNB;
        if (c < kb) A[(int64_t)(k0 + r) * n + k0 + c] = P[r][c];
      }
      // the panel's exchanges, in order, on every column outside it (one
      // thread per column: no ordering between threads is needed)
      for (int col = t; col < n; col += kBatchThreads) {
        if (col >= k0 && col < k0 + kb) continue;
        for (int c = 0; c < kb; c++) {
          const int pr2 = piv[k0 + c];
          if (pr2 != k0 + c) {
            const float2 a = A[(int64_t)(k0 + c) * n + col];
            A[(int64_t)(k0 + c) * n + col] = A[(int64_t)pr2 * n + col];
            A[(int64_t)pr2 * n + col] = a;
          }
        }
      }
      __syncthreads();
      const int c0 = k0 + kb, rest = n - c0;
      if (rest > 0) {
        // U12 = L11^-1 A12, one column per thread (L11 in the panel)
        for (int col = c0 + t; col < n; col += kBatchThreads) {
          float2 xcol[kBatchNB];
#pragma unroll
          for (int r = 0; r < kBatchNB; r++) xcol[r] = r < kb ? A[(int64_t)(k0 + r) * n + col] : make_float2(0.f, 0.f);
#pragma unroll
          for (int r = 0; r < kBatchNB; r++) {
#pragma unroll
            for (int q = r + 1; q < kBatchNB; q++) {
              if (q < kb) {
                const float2 l = P[q][r];
                xcol[q].x -= l.x * xcol[r].x - l.y * xcol[r].y;
                xcol[q].y -= l.x * xcol[r].y + l.y * xcol[r].x;
              }
            }
          }
#pragma unroll
          for (int r = 0; r < kBatchNB; r++)
            if (r < kb) A[(int64_t)(k0 + r) * n + col] = xcol[r];
        }
        __syncthreads();
        // A22 -= L21 U12 in 64 x 64 tiles; L21 rows come from the panel
        const int tx = t & 15, ty = t >> 4;
        for (int tj = 0; tj < rest; tj += 64) {
          for (int e = t; e < kBatchNB * 64; e += kBatchThreads) {
            const int q = e / 64, cc = e % 64;
            Ut[q][cc] = (q < kb && tj + cc < rest) ? A[(int64_t)(k0 + q) * n + c0 + tj + cc] : make_float2(0.f, 0.f);
          }
          __syncthreads();
          for (int ti = 0; ti < rest; ti += 64) {
            float accr[4][4], acci[4][4];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
              for (int j = 0; j < 4; j++) {
                accr[i][j] = 0.f;
                acci[i][j] = 0.f;
              }
            for (int q = 0; q < kb; q++) {
              float2 a[4], bq[4];
#pragma unroll
              for (int i = 0; i < 4; i++) {
                const int r = ti + ty + 16 * i;
                a[i] = r < rest ? P[kb + r][q] : make_float2(0.f, 0.f);
              }
#pragma unroll
              for (int j = 0; j < 4; j++) bq[j] = Ut[q][tx + 16 * j];
#pragma unroll
              for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                  accr[i][j] += a[i].x * bq[j].x - a[i].y * bq[j].y;
                  acci[i][j] += a[i].x * bq[j].y + a[i].y * bq[j].x;
                }
            }
#pragma unroll
            for (int i = 0; i < 4; i++) {
              const int r = ti + ty + 16 * i;
              if (r >= rest) continue;
#pragma unroll
              for (int j = 0; j < 4; j++) {
                const int cc = tj + tx + 16 * j;
                if (cc >= rest) continue;
                float2* dst = A + (int64_t)(c0 + r) * n + c0 + cc;
                float2 v = *dst;
                v.x -= accr[i][j];
                v.y -= acci[i][j];
                *dst = v;
              }
            }
          }
          __syncthreads();
        }
      }
      __syncthreads();
    }
    // ---------------- refined solve ----------------
    const double2* b = b_pool + pr.v;
    const double2* Z = Z64 + pr.z;
    float2* y = reinterpret_cast<float2*>(smem_raw);  // the panel area is free now
    int* pm = reinterpret_cast<int*>(y + kBatchMaxN);
    if (t == 0) {  // the pivots -> a permutation (row i of P b is b[pm[i]])
      for (int i = 0; i < n; i++) pm[i] = i;
      for (int k = 0; k < n; k++) {
        const int q = piv[k];
        const int a = pm[k];
        pm[k] = pm[q];
        pm[q] = a;
      }
    }
    for (int i = t; i < n; i += kBatchThreads) {
      xv[i] = make_double2(0.0, 0.0);
      rv[i] = b[i];
    }
    __syncthreads();
    // ||b||^2
    double bn2 = 0.0;
    for (int i = t; i < n; i += kBatchThreads) bn2 += b[i].x * b[i].x + b[i].y * b[i].y;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) bn2 += __shfl_xor_sync(0xffffffffu, bn2, off);
    if (lane == 0) s_red[warp][1] = bn2;
    __syncthreads();
    bn2 = 0.0;
    for (int w = 0; w < kBatchThreads / 32; w++) bn2 += s_red[w][1];
    const double bn = sqrt(bn2);
    double prev = 1e300, rel = 1.0;
    for (int it = 0; it < kBatchRefineMax; it++) {
      for (int i = t; i < n; i += kBatchThreads) {
        const double2 v = rv[pm[i]];
        y[i] = make_float2((float)v.x, (float)v.y);
      }
      __syncthreads();
      batch_trsv(A, n, y);
      for (int i = t; i < n; i += kBatchThreads) {
        xv[i].x += (double)y[i].x;
        xv[i].y += (double)y[i].y;
      }
      __syncthreads();
      // r = b - Z x (FP64), ||r||^2
      double rn2 = 0.0;
      for (int i = warp; i < n; i += kBatchThreads / 32) {
        const double2* row = Z + (int64_t)i * n;
        double sr = 0.0, si = 0.0;
        for (int j = lane; j < n; j += 32) {
          const double2 z = row[j], xx = xv[j];
          sr += z.x * xx.x - z.y * xx.y;
          si += z.x * xx.y + z.y * xx.x;
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          sr += __shfl_xor_sync(0xffffffffu, sr, off);
          si += __shfl_xor_sync(0xffffffffu, si, off);
        }
        if (lane == 0) {
          const double2 r = make_double2(b[i].x - sr, b[i].y - si);
          rv[i] = r;
          rn2 += r.x * r.x + r.y * r.y;
        }
      }
      if (lane == 0) s_red[warp][0] = rn2;
      __syncthreads();
      rn2 = 0.0;
      for (int w = 0; w < kBatchThreads / 32; w++) rn2 += s_red[w][0];
      rel = bn > 0 ? sqrt(rn2) / bn : 0.0;
      __syncthreads();
      if (!(rel == rel) || rel <= tol || rel > 0.5 * prev) break;
      prev = rel;
    }
    double2* x = x_pool + pr.v;
    for (int i = t; i < n; i += kBatchThreads) x[i] = xv[i];
    if (t == 0) {
      int st = s_bad;
      if (st == 0 && !(rel == rel)) st = 2;
      if (st == 0 && rel > 1e-6) st = 3;
      status[p] = st;
      resid[p] = rel;
    }
    __syncthreads();
  }
}

// abc and segment-centre currents of every problem; one thread per segment
// of the concatenated structures (seg_prob: the problem of each segment).
__global__ void batch_coeff_kernel(int64_t nseg_total, const int* seg_prob, const BatchProblem* probs,
                                   const int32_t* cptr, const int32_t* cbasis,
                                   const double* ca, const double* cb, const double* cc, const double2* x_pool,
                                   double* abc, double2* cur) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nseg_total) return;
  const int p = seg_prob[g];
  const double2* sol = x_pool + probs[p].v;
  double air = 0, aii = 0, bir = 0, bii = 0, cir = 0, cii = 0;
  for (int e = cptr[g]; e < cptr[g + 1]; e++) {
    const double2 s = sol[cbasis[e]];
    air += ca[e] * s.x;
    aii += ca[e] * s.y;
    bir += cb[e] * s.x;
    bii += cb[e] * s.y;
    cir += cc[e] * s.x;
    cii += cc[e] * s.y;
  }
  abc[0 * nseg_total + g] = air;
  abc[1 * nseg_total + g] = aii;
  abc[2 * nseg_total + g] = bir;
  abc[3 * nseg_total + g] = bii;
  abc[4 * nseg_total + g] = cir;
  abc[5 * nseg_total + g] = cii;
  cur[g] = make_double2(air + cir, aii + cii);
}

// Far field of every problem at every direction: one warp per (problem,
// direction), the problem's segments staged through shared memory.  The
// per-segment arithmetic is the single-problem kernel's (FP64).
// Power-gain normalisation of every problem (one voltage source):
// gcop = lambda^2 2 pi / (eta P), P = Re(V conj(I)) / 2, I = cur[feed] lambda.
__global__ void batch_gain_norm_kernel(int nprob, const int64_t* seg_off, const int* feed, const double2* volt,
                                       const double* lam, double eta, const double2* cur, double* gcop) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nprob) return;
  const double2 c = cur[seg_off[p] + feed[p]];
  const double L = lam[p];
  const double ir = c.x * L, ii = c.y * L;
  const double2 v = volt[p];
  const double P = 0.5 * (v.x * ir + v.y * ii);  // Re(V conj(I)) / 2
  gcop[p] = L * L * 2.0 * 3.1415926536 / (eta * P);
}

struct BatchPatternArgs {
  int nprob, ndir;
  const double *theta, *phi;
  const int64_t* seg_off;  // nprob + 1
  const double* seg;       // 8 x nseg_total (x y z s b cab sab salp)
  const double* abc;       // 6 x nseg_total
  int64_t nseg_total;
  int ksymp, perfect;
  cplx zrati;
  double eta;
  double2 *eth, *eph;  // nprob x ndir, or null
  const double* gcop;  // per problem, or null
  float* gain;         // nprob x ndir power gain in dB (db10 with the -999.99 floor), or null
};

__global__ void __launch_bounds__(kPatDirs * 32) batch_pattern_kernel(BatchPatternArgs A) {
  __shared__ SegPat seg[kPatChunk];
  const int p = blockIdx.y;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int d = blockIdx.x * kPatDirs + warp;
  const bool active = d < A.ndir;
  const int64_t s0 = A.seg_off[p], ns = A.seg_off[p + 1] - s0;
  const int64_t T = A.nseg_total;
  double thet = 0, phi = 0;
  if (active) {
    thet = A.theta[d];
    phi = A.phi[d];
  }
  double sp, cp, st, ct;
  sincos(phi, &sp, &cp);
  sincos(thet, &st, &ct);
  const double phx = -sp, phy = cp;
  const double roz0 = ct;
  const double thx = roz0 * phy, thy = -roz0 * phx, thz = -st;
  const double rox = -thz * phy, roy = thz * phx;
  cplx ci[2][3];
  for (int k = 0; k < A.ksymp; k++) {
    const double roz = (k == 0) ? roz0 : -roz0;
    cplx sx = mk(0, 0), sy = mk(0, 0), sz = mk(0, 0);
    for (int64_t c0 = 0; c0 < ns; c0 += kPatChunk) {
      __syncthreads();
      for (int t = threadIdx.x; t < kPatChunk; t += blockDim.x) {
        const int64_t i = s0 + c0 + t;
        if (c0 + t < ns) {
          SegPat g;
          g.x = A.seg[i];
          g.y = A.seg[T + i];
          g.z = A.seg[2 * T + i];
          g.s = A.seg[3 * T + i];
          g.cab = A.seg[5 * T + i];
          g.sab = A.seg[6 * T + i];
          g.salp = A.seg[7 * T + i];
          g.air = A.abc[i];
          g.aii = A.abc[T + i];
          g.bir = A.abc[2 * T + i];
          g.bii = A.abc[3 * T + i];
          g.cir = A.abc[4 * T + i];
          g.cii = A.abc[5 * T + i];
          seg_pat_el(g);
          seg[t] = g;
        }
      }
      __syncthreads();
      if (active) {
        const int cnt = (int)min((int64_t)kPatChunk, ns - c0);
        for (int t = lane; t < cnt; t += 32) {
          const SegPat& g = seg[t];
          cplx exa;
          seg_term(g, rox, roy, roz, &exa);
          sx += exa * g.cab;
          sy += exa * g.sab;
          sz += exa * g.salp;
        }
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      sx.re += __shfl_down_sync(0xffffffffu, sx.re, off);
      sx.im += __shfl_down_sync(0xffffffffu, sx.im, off);
      sy.re += __shfl_down_sync(0xffffffffu, sy.re, off);
      sy.im += __shfl_down_sync(0xffffffffu, sy.im, off);
      sz.re += __shfl_down_sync(0xffffffffu, sz.re, off);
      sz.im += __shfl_down_sync(0xffffffffu, sz.im, off);
    }
    ci[k][0] = sx;
    ci[k][1] = sy;
    ci[k][2] = sz;
  }
  if (!active || lane != 0) return;
  cplx cix = ci[0][0], ciy = ci[0][1], ciz = ci[0][2];
  if (A.ksymp == 2) {
    cplx rrv, rrh;
    if (A.perfect) {
      rrv = mk(-1.0, -0.0);
      rrh = mk(-1.0, -0.0);
    } else {
      cplx zrsin = csqrt_(1. - A.zrati * A.zrati * thz * thz);
      rrv = -(roz0 - A.zrati * zrsin) / (roz0 + A.zrati * zrsin);
      rrh = (A.zrati * roz0 - zrsin) / (A.zrati * roz0 + zrsin);
    }
    cplx ix = ci[1][0], iy = ci[1][1], iz = ci[1][2];
    cplx cdp = (ix * phx + iy * phy) * (rrh - rrv);
    cix = cix + ix * rrv + cdp * phx;
    ciy = ciy + iy * rrv + cdp * phy;
    ciz = ciz - iz * rrv;
  }
  const cplx C3 = mk(0.0, -A.eta / (4.0 * 3.1415926536));
  cplx e_t = (cix * thx + ciy * thy + ciz * thz) * C3;
  cplx e_p = (cix * phx + ciy * phy) * C3;
  const int64_t o = (int64_t)p * A.ndir + d;
  if (A.eth) {
    A.eth[o] = make_double2(e_t.re, e_t.im);
    A.eph[o] = make_double2(e_p.re, e_p.im);
  }
  if (A.gain) {
    const double pw = A.gcop[p] * (e_t.re * e_t.re + e_t.im * e_t.im + e_p.re * e_p.re + e_p.im * e_p.im);
    A.gain[o] = pw < 1.0e-20 ? -999.99f : (float)(10.0 * log10(pw));
  }
}

}  // namespace necb
