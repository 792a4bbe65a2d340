// Triangular solves on the row-major LU factors (replaces solve,
// src/matrix_algebra.cpp:271-307), the FP64 residual of the mixed-precision
// refinement, and the basis-to-segment current coefficients (replaces
// c_geometry::get_current_coefficients, src/c_geometry.cpp:3299-3387).
//
// The triangular solves are blocked by TB rows: a one-CTA kernel solves the
// diagonal block (column-oriented, lanes over rows), then a row-parallel
// kernel (one warp per row, coalesced along the row) subtracts the block's
// contribution from every remaining row.
#pragma once
#include <cstdint>

#include "lu.cuh"

namespace necb {

constexpr int kTrsvB = 64;
template <typename T>
constexpr size_t trsv_diag_smem() {
  return sizeof(T) * (kTrsvB * (kTrsvB + 1) + kTrsvB);
}

// Diagonal block of L (unit) or U: x = T_blk^-1 rhs_blk.  64 threads.
template <typename T, bool LOWER>
__global__ void __launch_bounds__(64) trsv_diag_kernel(const T* M, int64_t ld, int64_t n, int64_t b0,
                                                       const T* rhs, T* sol) {
  // dynamic shared memory: D[kTrsvB][kTrsvB + 1] then x[kTrsvB]
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T(*D)[kTrsvB + 1] = reinterpret_cast<T(*)[kTrsvB + 1]>(smem_raw);
  T* x = reinterpret_cast<T*>(smem_raw) + kTrsvB * (kTrsvB + 1);
  const int t = threadIdx.x;
  const int bs = (int)min((int64_t)kTrsvB, n - b0);
  for (int idx = t; idx < bs * bs; idx += 64) {
    int r = idx / bs, q = idx - r * bs;
    D[r][q] = M[(b0 + r) * ld + b0 + q];
  }
  if (t < bs) x[t] = rhs[b0 + t];
  __syncthreads();
  if (LOWER) {
    for (int q = 0; q < bs - 1; q++) {
      T xq = x[q];
      if (t > q && t < bs) {
        T l = D[t][q];
        T a = x[t];
        a.x -= l.x * xq.x - l.y * xq.y;
        a.y -= l.x * xq.y + l.y * xq.x;
        x[t] = a;
      }
      __syncthreads();
    }
  } else {
    for (int q = bs - 1; q >= 0; q--) {
      if (t == q) x[q] = cdiv(x[q], D[q][q]);
      __syncthreads();
      T xq = x[q];
      if (t < q) {
        T u = D[t][q];
        T a = x[t];
        a.x -= u.x * xq.x - u.y * xq.y;
        a.y -= u.x * xq.y + u.y * xq.x;
        x[t] = a;
      }
      __syncthreads();
    }
  }
  if (t < bs) sol[b0 + t] = x[t];
}

// rhs[r] -= sum_{q in block} M[r][q] sol[q] for rows r in [r0, r1).
template <typename T>
__global__ void __launch_bounds__(256) trsv_update_kernel(const T* M, int64_t ld, int64_t n, int64_t b0,
                                                          int64_t r0, int64_t r1, const T* sol, T* rhs) {
  __shared__ T xs[kTrsvB];
  const int bs = (int)min((int64_t)kTrsvB, n - b0);
  if (threadIdx.x < bs) xs[threadIdx.x] = sol[b0 + threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t r = r0 + (int64_t)blockIdx.x * 8 + warp; r < r1; r += (int64_t)gridDim.x * 8) {
    decltype(xs[0].x) sr = 0, si = 0;
    for (int q = lane; q < bs; q += 32) {
      T a = M[r * ld + b0 + q];
      T v = xs[q];
      sr += a.x * v.x - a.y * v.y;
      si += a.x * v.y + a.y * v.x;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      sr += __shfl_down_sync(0xffffffffu, sr, off);
      si += __shfl_down_sync(0xffffffffu, si, off);
    }
    if (lane == 0) {
      T a = rhs[r];
      a.x -= sr;
      a.y -= si;
      rhs[r] = a;
    }
  }
}

// ---------------------------------------------------------------------------
// Persistent triangular sweep: one cooperative launch per triangle.
//
// Row block v (64 rows) is owned by CTA v % grid (blocks visited in order, so
// every wait is on a block owned by a CTA that is already running and never
// waits on a later block: no deadlock with all CTAs co-resident).  For block
// v the CTA accumulates -sum_j M[rows][cols_j] x_j over every earlier block j
// as soon as block j's solution is published (flag == epoch), keeping per-lane
// partial sums (one warp-reduction per row at the end), then one warp solves
// the 64 x 64 diagonal block with register shuffles and publishes x_v.
// LOWER: unit lower L, blocks in ascending order; else upper U (non-unit),
// blocks in descending order.  Reads every element of the triangle once.
constexpr int kSweepThreads = 256;
constexpr long long kSweepSpinLimit = 1LL << 26;

template <typename T, bool LOWER>
__global__ void __launch_bounds__(kSweepThreads) trsv_sweep_kernel(const T* M, int64_t ld, int64_t n,
                                                                   const T* b, T* x, int* flags, int epoch,
                                                                   int* status) {
  using R = decltype(T{}.x);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T(*D)[kTrsvB + 1] = reinterpret_cast<T(*)[kTrsvB + 1]>(smem_raw);  // dynamic: trsv_diag_smem<T>()
  __shared__ T xs[kTrsvB];
  __shared__ T acc[kTrsvB];
  __shared__ int s_abort;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nblk = (int)((n + kTrsvB - 1) / kTrsvB);
  if (tid == 0) s_abort = 0;
  for (int v = blockIdx.x; v < nblk; v += gridDim.x) {
    const int blk = LOWER ? v : nblk - 1 - v;
    const int64_t r0 = (int64_t)blk * kTrsvB;
    const int bs = (int)min((int64_t)kTrsvB, n - r0);
    // each warp owns rows warp, warp+8, ... of the block (8 rows)
    R pr[8], pi[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      pr[q] = 0;
      pi[q] = 0;
    }
    // the diagonal block does not depend on earlier solutions: stage it first
    for (int idx = tid; idx < bs * bs; idx += kSweepThreads) {
      const int r = idx / bs, q = idx - r * bs;
      D[r][q] = M[(r0 + r) * ld + r0 + q];
    }
    for (int u = 0; u < v; u++) {  // earlier blocks in solve order
      const int jb = LOWER ? u : nblk - 1 - u;
      if (tid == 0) {
        long long spins = 0;
        while (*((volatile int*)(flags + jb)) != epoch) {
          if (++spins > kSweepSpinLimit) {
            atomicOr(status, 1 << 9);
            s_abort = 1;
            break;
          }
          __nanosleep(20);
        }
        __threadfence();
      }
      __syncthreads();
      if (s_abort) return;
      const int64_t c0 = (int64_t)jb * kTrsvB;
      const int cs = (int)min((int64_t)kTrsvB, n - c0);
      if (tid < cs) xs[tid] = __ldcg(x + c0 + tid);
      __syncthreads();
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const int rr = warp + 8 * q;
        if (rr < bs) {
          const T* row = M + (r0 + rr) * ld + c0;
          for (int c = lane; c < cs; c += 32) {
            T a = row[c];
            T xv = xs[c];
            pr[q] += a.x * xv.x - a.y * xv.y;
            pi[q] += a.x * xv.y + a.y * xv.x;
          }
        }
      }
      __syncthreads();
    }
    // reduce partial sums, acc = b - sum
#pragma unroll
    for (int q = 0; q < 8; q++) {
      R sr = pr[q], si = pi[q];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        sr += __shfl_down_sync(0xffffffffu, sr, off);
        si += __shfl_down_sync(0xffffffffu, si, off);
      }
      const int rr = warp + 8 * q;
      if (lane == 0 && rr < bs) {
        T bb = b[r0 + rr];
        T o;
        o.x = bb.x - sr;
        o.y = bb.y - si;
        acc[rr] = o;
      }
    }
    __syncthreads();
    if (warp == 0) {
      // lane owns rows lane and lane+32; column sweep with shuffles
      T v0 = lane < bs ? acc[lane] : T{};
      T v1 = lane + 32 < bs ? acc[lane + 32] : T{};
      if (LOWER) {
        for (int q = 0; q < bs - 1; q++) {
          T xq;
          xq.x = __shfl_sync(0xffffffffu, q < 32 ? v0.x : v1.x, q & 31);
          xq.y = __shfl_sync(0xffffffffu, q < 32 ? v0.y : v1.y, q & 31);
          if (lane > q && lane < bs) {
            T l = D[lane][q];
            v0.x -= l.x * xq.x - l.y * xq.y;
            v0.y -= l.x * xq.y + l.y * xq.x;
          }
          if (lane + 32 > q && lane + 32 < bs) {
            T l = D[lane + 32][q];
            v1.x -= l.x * xq.x - l.y * xq.y;
            v1.y -= l.x * xq.y + l.y * xq.x;
          }
        }
      } else {
        for (int q = bs - 1; q >= 0; q--) {
          // finalise x_q = v_q / U_qq on its owner, then broadcast
          if (q < 32) {
            if (lane == q) v0 = cdiv(v0, D[q][q]);
          } else {
            if (lane == q - 32) v1 = cdiv(v1, D[q][q]);
          }
          T xq;
          xq.x = __shfl_sync(0xffffffffu, q < 32 ? v0.x : v1.x, q & 31);
          xq.y = __shfl_sync(0xffffffffu, q < 32 ? v0.y : v1.y, q & 31);
          if (lane < q) {
            T u = D[lane][q];
            v0.x -= u.x * xq.x - u.y * xq.y;
            v0.y -= u.x * xq.y + u.y * xq.x;
          }
          if (lane + 32 < q) {
            T u = D[lane + 32][q];
            v1.x -= u.x * xq.x - u.y * xq.y;
            v1.y -= u.x * xq.y + u.y * xq.x;
          }
        }
      }
      if (lane < bs) x[r0 + lane] = v0;
      if (lane + 32 < bs) x[r0 + lane + 32] = v1;
      __threadfence();
      __syncwarp();
      if (lane == 0) atomicExch(flags + blk, epoch);
    }
    __syncthreads();
  }
}

// y[i] = src[perm[i]] converted to the factor precision.
template <typename TO, typename TI>
__global__ void permute_kernel(const TI* src, const int* perm, TO* dst, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    TI v = src[perm[i]];
    TO o;
    o.x = v.x;
    o.y = v.y;
    dst[i] = o;
  }
}

// x += d (d in the factor precision)
template <typename TD>
__global__ void axpy_kernel(double2* x, const TD* d, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    x[i].x += (double)d[i].x;
    x[i].y += (double)d[i].y;
  }
}

// r = b - Z x (FP64), one warp per row; accumulates ||r||^2 into *rn2.
__global__ void __launch_bounds__(256) residual_kernel(const double2* Z, int64_t ld, int64_t n,
                                                       const double2* x, const double2* b,
                                                       double2* r, double* rn2) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double part = 0.0;
  for (int64_t row = (int64_t)blockIdx.x * 8 + warp; row < n; row += (int64_t)gridDim.x * 8) {
    const double2* zr = Z + row * ld;
    double sr = 0, si = 0;
    for (int64_t q = lane; q < n; q += 32) {
      double2 a = zr[q];
      double2 v = x[q];
      sr += a.x * v.x - a.y * v.y;
      si += a.x * v.y + a.y * v.x;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      sr += __shfl_down_sync(0xffffffffu, sr, off);
      si += __shfl_down_sync(0xffffffffu, si, off);
    }
    if (lane == 0) {
      double2 bb = b[row];
      double2 o = make_double2(bb.x - sr, bb.y - si);
      r[row] = o;
      part += o.x * o.x + o.y * o.y;
    }
  }
  if (lane == 0) atomicAdd(rn2, part);
}

// Current coefficients: for each segment j, sum over the basis functions
// with support on j in ascending basis order (the reference's accumulation
// order), then the segment-centre current (air+cir, aii+cii).
__global__ void coeff_kernel(int64_t n, const int32_t* ptr, const int32_t* basis,
                             const double* a, const double* b, const double* c,
                             const double2* sol, double* abc, double2* cur) {
  int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double air = 0, aii = 0, bir = 0, bii = 0, cir = 0, cii = 0;
  for (int e = ptr[j]; e < ptr[j + 1]; e++) {
    double2 s = sol[basis[e]];
    double ax = a[e], bx = b[e], cx = c[e];
    air += ax * s.x;
    aii += ax * s.y;
    bir += bx * s.x;
    bii += bx * s.y;
    cir += cx * s.x;
    cii += cx * s.y;
  }
  abc[0 * n + j] = air;
  abc[1 * n + j] = aii;
  abc[2 * n + j] = bir;
  abc[3 * n + j] = bii;
  abc[4 * n + j] = cir;
  abc[5 * n + j] = cii;
  cur[j] = make_double2(air + cir, aii + cii);
}

// *out += ||v||^2
__global__ void norm2_kernel(const double2* v, int64_t n, double* out) {
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += v[i].x * v[i].x + v[i].y * v[i].y;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// FP64 -> FP32 copy of a row-major matrix
__global__ void demote_kernel(const double2* src, float2* dst, int64_t count) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (; i < count; i += stride) dst[i] = make_float2((float)src[i].x, (float)src[i].y);
}

// ---------------------------------------------------------------------------
// Triangular sweeps of the mixed-precision refinement, on complex64 factors
// whose 64 x 64 diagonal blocks have been inverted once per factorisation
// (tri_inv_kernel).  Block v of the sweep computes
//     x_v = inv(T_vv) (b_v - sum_{u before v} T_vu x_u)
// One CTA per block (persistent, cooperative).  A single counter holds how
// many blocks of the sweep are complete; blocks complete in sweep order, so
// a CTA reads the counter once and folds in every finished block it has not
// yet seen.  The off-diagonal tile row of each block is loaded before the
// wait, and the diagonal solve is a parallel 64 x 64 product with the
// inverse, so the chain between two blocks is one counter hand-off, one
// read of x_u and two block reductions.

// tinv[2*blk] = L_bb^-1 (unit lower), tinv[2*blk+1] = U_bb^-1, 64 x 64
// row-major each, zero outside the kb x kb triangle.  128 threads: threads
// 0..63 build the columns of L^-1, threads 64..127 those of U^-1.
constexpr size_t tri_inv_smem() { return (size_t)3 * kBlk * (kBlk + 1) * sizeof(float2); }
__global__ void __launch_bounds__(128) tri_inv_kernel(const float2* M, int64_t ld, int64_t n, float2* tinv) {
  constexpr int NB = kBlk;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2(*D)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(smem_raw);
  float2(*X)[NB + 1] = D + NB;
  float2(*Y)[NB + 1] = D + 2 * NB;
  const int t = threadIdx.x;
  const int64_t b0 = (int64_t)blockIdx.x * NB;
  const int kb = (int)min((int64_t)NB, n - b0);
  for (int e = t; e < NB * NB; e += 128) {
    const int r = e / NB, c = e % NB;
    D[r][c] = (r < kb && c < kb) ? M[(b0 + r) * ld + b0 + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  if (t < NB) {
    // column j of L^-1: X[j][j] = 1, X[i][j] = -sum_{k=j}^{i-1} L[i][k] X[k][j]
    const int j = t;
    for (int i = 0; i < NB; i++) {
      float2 v = make_float2(0.f, 0.f);
      if (j < kb && i < kb && i >= j) {
        if (i == j) {
          v.x = 1.f;
        } else {
          float sr = 0.f, si = 0.f;
          for (int k = j; k < i; k++) {
            const float2 a = D[i][k], b = X[k][j];
            sr += a.x * b.x - a.y * b.y;
            si += a.x * b.y + a.y * b.x;
          }
          v = make_float2(-sr, -si);
        }
      }
      X[i][j] = v;
    }
  } else {
    // column j of U^-1: Y[j][j] = 1/U[j][j],
    // Y[i][j] = -(sum_{k=i+1}^{j} U[i][k] Y[k][j]) / U[i][i] for i < j
    const int j = t - NB;
    for (int i = NB - 1; i >= 0; i--) {
      float2 v = make_float2(0.f, 0.f);
      if (j < kb && i <= j) {
        const float2 di = crecip(D[i][i]);
        if (i == j) {
          v = di;
        } else {
          float sr = 0.f, si = 0.f;
          for (int k = i + 1; k <= j; k++) {
            const float2 a = D[i][k], b = Y[k][j];
            sr += a.x * b.x - a.y * b.y;
            si += a.x * b.y + a.y * b.x;
          }
          v = cmul(make_float2(-sr, -si), di);
        }
      }
      Y[i][j] = v;
    }
  }
  __syncthreads();
  float2* out = tinv + (int64_t)blockIdx.x * 2 * NB * NB;
  for (int e = t; e < NB * NB; e += 128) {
    out[e] = X[e / NB][e % NB];
    out[NB * NB + e] = Y[e / NB][e % NB];
  }
}

// The sweeps' "not yet written" marker: every solution element starts as
// this bit pattern (a NaN no arithmetic here produces from finite data), so
// the CTA waiting on the previous block can poll the values themselves.
constexpr unsigned kSweepUnset = 0xFFFFFFFFu;
__device__ __forceinline__ float2 ld_relaxed_f2(const float2* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return make_float2(__uint_as_float((unsigned)v), __uint_as_float((unsigned)(v >> 32)));
}

__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

constexpr int kInvSweepThreads = 256;
constexpr int kInvSweepChunk = 16;                  // solved blocks staged per pass
constexpr unsigned long long kSweepWaitNs = 4000000000ull;  // 4 s

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// The products of each diagonal-block inverse with the tiles before it in
// the sweep order, for the last kSweepDepth steps of each block:
//   W[v][0][d] = inv(L_vv) L_{v,v-1-d}   (zero where v - 1 - d < 0)
//   W[v][1][d] = inv(U_vv) U_{v,v+1+d}   (zero beyond the last block)
// 64 x 64 row-major each, zero outside the matrix.  grid (nblk, 2,
// kSweepDepth), 256 threads; blockIdx.y selects the lower (0) or upper (1)
// product, blockIdx.z the distance d + 1.
constexpr int kSweepDepth = 3;
__global__ void __launch_bounds__(256) next_tile_kernel(const float2* M, int64_t ld, int64_t n, const float2* tinv,
                                                       float2* W) {
  constexpr int NB = kBlk;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2(*Tm)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(smem_raw);  // the tile T_vu
  float2(*Iv)[NB + 1] = Tm + NB;                                         // inv(T_vv)
  const int t = threadIdx.x;
  const int nblk = (int)((n + NB - 1) / NB);
  const int v = blockIdx.x, side = blockIdx.y, d = blockIdx.z;
  const int u = side == 0 ? v - 1 - d : v + 1 + d;
  float2* out = W + (((int64_t)v * 2 + side) * kSweepDepth + d) * NB * NB;
  if (u < 0 || u >= nblk) {
    for (int e = t; e < NB * NB; e += 256) out[e] = make_float2(0.f, 0.f);
    return;
  }
  const float2* inv = tinv + ((int64_t)v * 2 + side) * NB * NB;
  const int64_t r0 = (int64_t)v * NB, c0 = (int64_t)u * NB;
  for (int e = t; e < NB * NB; e += 256) {
    const int r = e / NB, c = e % NB;
    Tm[r][c] = (r0 + r < n && c0 + c < n) ? M[(r0 + r) * ld + c0 + c] : make_float2(0.f, 0.f);
    Iv[r][c] = inv[e];
  }
  __syncthreads();
  // thread t: row t / 4, sixteen columns (t % 4) + 4 j (a warp reads 8 rows
  // of the inverse and 4 runs of the tile per k)
  const int r = t >> 2, cq = t & 3;
  float2 acc[16];
#pragma unroll
  for (int j = 0; j < 16; j++) acc[j] = make_float2(0.f, 0.f);
#pragma unroll 4
  for (int k = 0; k < NB; k++) {
    const float2 a = Iv[r][k];
#pragma unroll
    for (int j = 0; j < 16; j++) {
      const float2 b = Tm[k][cq + 4 * j];
      acc[j].x += a.x * b.x - a.y * b.y;
      acc[j].y += a.x * b.y + a.y * b.x;
    }
  }
#pragma unroll
  for (int j = 0; j < 16; j++) out[r * NB + cq + 4 * j] = acc[j];
}
constexpr size_t next_tile_smem() { return (size_t)2 * kBlk * (kBlk + 1) * sizeof(float2); }

// Hand-off of a solved block to the next CTAs of a thread-block cluster:
// 64-bit stores into their shared memory.
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ unsigned peer_addr(unsigned local, unsigned rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_peer_f2(unsigned addr, float2 v) {  // one 64-bit store
  const unsigned long long u = (unsigned long long)__float_as_uint(v.x) | ((unsigned long long)__float_as_uint(v.y) << 32);
  asm volatile("st.shared::cluster.u64 [%0], %1;" ::"r"(addr), "l"(u) : "memory");
}
// 16-byte load kept in program order with the waits around it (asm
// volatile), so that the compiler does not move it to its first use
__device__ __forceinline__ float4 ld_early_f4(const float4* p) {
  float4 v;
  asm volatile("ld.global.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
  return v;
}
__device__ __forceinline__ float2 ld_volatile_shared_f2(const float2* p) {
  unsigned long long u;
  asm volatile("ld.volatile.shared.u64 %0, [%1];" : "=l"(u) : "r"(smem_addr(p)) : "memory");
  return make_float2(__uint_as_float((unsigned)u), __uint_as_float((unsigned)(u >> 32)));
}

// LOWER: x = L^-1 b (unit lower); !LOWER: x = U^-1 b.  counter must be 0 at
// launch; it counts the completed positions of the sweep order.
//
// CTA s owns block row v(s).  It folds in the positions before the last D =
// kSweepDepth ones as they complete, M[v][u] x_u, and forms
// c = inv(T_vv) (b_v - that sum).  The last D positions enter through the
// precomputed products W_d = inv(T_vv) T_{v,u} (next_tile_kernel):
// x_v = c - sum_d W_d x_{s-d}, each taken as soon as its block arrives, so
// that only W_1 x_{s-1} lies between two blocks of the sweep and the fold-in
// of the earlier positions, which goes through the completion counter, has
// D steps of slack.  Thread 0 alone polls the counter, sleeping longer the
// further the row is from what it needs, and solved blocks known to be
// complete (up to 16 at a time) are staged in shared memory with one load
// per element.  Each thread holds the next tile row quarter in registers
// while it multiplies the current one.  A block x_{s-d} is taken by polling
// its values in global memory until none is still unset (x starts as
// kSweepUnset).  A wait that runs out sets bit 9 of *status; every CTA then
// returns.
//
// CS > 0: launched in clusters of CS CTAs, one position per CTA (grid >=
// the number of blocks).  A block x_{s-d} whose CTA is in the same cluster
// (rank >= d) arrives in this CTA's shared memory instead: its CTA stores
// each value there with one 64-bit store and this CTA polls its own shared
// memory for the unset marker, without the round trip through L2 and
// without fences.  All CTAs of a cluster
// meet at a cluster barrier before they exit, so none exits while a peer
// may still write to it.
template <bool LOWER, int CS = 0>
__global__ void __launch_bounds__(kInvSweepThreads, 2) inv_sweep_kernel(const float2* M, int64_t ld, int64_t n,
                                                                     const float2* tinv, const float2* wnext,
                                                                     const float2* b, float2* x, unsigned* counter,
                                                                     int* status) {
  constexpr int NB = kBlk, QW = NB / 4, KX = kInvSweepChunk, D = kSweepDepth;  // four column quarters of 16
  __shared__ float2 part[4][NB];
  __shared__ float2 part2[4][NB];  // the last products' partial sums (part may still be read)
  __shared__ float2 sv[NB];
  __shared__ float2 sx[KX * NB];
  __shared__ float2 sinv[NB][NB + 1];  // inv(T_vv), rows padded against bank conflicts
  __shared__ float2 xin[D][NB];        // x_{s-d} from cluster peers (CS > 0), unset until written
  __shared__ int s_avail;
  const int t = threadIdx.x;
  const int r = t & (NB - 1), q = t >> 6;  // row in the block, column quarter
  const int nblk = (int)((n + NB - 1) / NB);
  unsigned rank = 0;
  if constexpr (CS > 0) {
    rank = cluster_rank();
    for (int e = t; e < D * NB; e += kInvSweepThreads)
      xin[e / NB][e % NB] = make_float2(__uint_as_float(kSweepUnset), __uint_as_float(kSweepUnset));
    cluster_sync_all();  // no peer writes before every buffer is unset
  }
  // one position of the sweep order; false when a wait ran out
  auto position = [&](int s) -> bool {
    const int v = LOWER ? s : nblk - 1 - s;
    const int64_t r0 = (int64_t)v * NB;
    const int bs = (int)min((int64_t)NB, n - r0);
    const bool rowok = r < bs;
    // independent of the sweep: inv(T_vv) into shared memory and the
    // right-hand side
    const int64_t bbase = ((int64_t)v * 2 + (LOWER ? 0 : 1)) * NB * NB;
    const int64_t wbase = ((int64_t)v * 2 + (LOWER ? 0 : 1)) * D * NB * NB + r * NB + q * QW;
    __syncthreads();  // the previous block's reads of sinv are done
    for (int e = t; e < NB * NB; e += kInvSweepThreads) sinv[e / NB][e % NB] = tinv[bbase + e];
    // this thread's row quarters of the W_d (128-byte lines) into L2, late
    // enough that the tiles streamed meanwhile do not evict them: at the
    // last pass of the fold-in, or now when there is none
    auto prefetch_w = [&]() {
#pragma unroll
      for (int d = 1; d <= D; d++)
        if (s >= d) asm volatile("prefetch.global.L2 [%0];" ::"l"(wnext + wbase + (d - 1) * NB * NB));
    };
    if (s - D <= 0) prefetch_w();
    const float2 bb = t < bs ? b[r0 + t] : make_float2(0.f, 0.f);
    // the quarter row of the tile at sweep position i
    auto load_tile = [&](float2 (&m)[QW], int i) {
      const int u = LOWER ? i : nblk - 1 - i;
      const int64_t c0 = (int64_t)u * NB + q * QW;
      if (rowok && c0 + QW <= n) {
        const float4* mp = reinterpret_cast<const float4*>(M + (r0 + r) * ld + c0);
#pragma unroll
        for (int k = 0; k < QW / 2; k++) {
          const float4 w = mp[k];
          m[2 * k] = make_float2(w.x, w.y);
          m[2 * k + 1] = make_float2(w.z, w.w);
        }
      } else {
#pragma unroll
        for (int k = 0; k < QW; k++)
          m[k] = (rowok && c0 + k < n) ? M[(r0 + r) * ld + c0 + k] : make_float2(0.f, 0.f);
      }
    };
    const int lim = s - D;  // positions folded in through the counter: 0 .. lim - 1
    int avail = 0;          // positions known complete (the same in every thread)
    // thread 0 waits until position `need` is complete; false when a wait ran out
    auto wait_for = [&](int need) -> bool {
      if (t == 0) {
        const unsigned long long t0 = global_ns();
        long long spins = 0;
        int c = (int)ld_acquire_u32(counter);
        while (c <= need) {
          if (((++spins & 63) == 0 && (*(volatile int*)status & (1 << 9))) || spins > kSweepSpinLimit ||
              global_ns() - t0 > kSweepWaitNs) {
            atomicOr(status, 1 << 9);
            c = -1;
            break;
          }
          // the row needs position lim - 1 only after lim - 1 - c more blocks
          const int ahead = lim - 1 - c;
          __nanosleep(ahead <= 1 ? 20u : (unsigned)min(ahead * 64, 1024));
          c = (int)ld_acquire_u32(counter);
        }
        s_avail = c;
      }
      __syncthreads();  // orders thread 0's acquire before the x reads that follow
      avail = s_avail;
      return avail >= 0;
    };
    float2 m[QW];
    if (lim > 0) load_tile(m, 0);
    float accr = 0.f, acci = 0.f;
    bool ok = true;
    for (int i0 = 0; i0 < lim;) {
      if (avail <= i0 && !(ok = wait_for(i0))) break;
      const int i1 = min(lim, min(avail, i0 + KX));
      if (i1 == lim) prefetch_w();
      for (int e = t; e < (i1 - i0) * NB; e += kInvSweepThreads) {
        const int i = i0 + e / NB;
        const int64_t col = (int64_t)(LOWER ? i : nblk - 1 - i) * NB + (e % NB);
        sx[e] = col < n ? __ldcg(x + col) : make_float2(0.f, 0.f);
      }
      __syncthreads();
#pragma unroll 1
      for (int i = i0; i < i1; i++) {
        float2 mn[QW];
        if (i + 1 < lim) load_tile(mn, i + 1);  // in flight during this tile's products
        const float2* xs = sx + (i - i0) * NB + q * QW;
#pragma unroll
        for (int k = 0; k < QW; k++) {
          const float2 xv = xs[k];
          accr += m[k].x * xv.x - m[k].y * xv.y;
          acci += m[k].x * xv.y + m[k].y * xv.x;
        }
        if (i + 1 < lim) {
#pragma unroll
          for (int k = 0; k < QW; k++) m[k] = mn[k];
        }
      }
      __syncthreads();  // sx is reused by the next pass
      i0 = i1;
    }
    if (!ok) return false;
    // W_1's quarter row in registers ahead of the wait for x_{s-1}
    float4 wv[QW / 2];
    if (s > 0) {
      const float4* wp = reinterpret_cast<const float4*>(wnext + wbase);
#pragma unroll
      for (int k = 0; k < QW / 2; k++) wv[k] = ld_early_f4(wp + k);
    }
    // c = inv(T_vv) (b_v - sum so far), row r held by thread r
    part[q][r] = make_float2(accr, acci);
    __syncthreads();
    if (t < NB) {
      float2 a = make_float2(0.f, 0.f);
      if (t < bs) {
        a.x = bb.x - (part[0][t].x + part[1][t].x + part[2][t].x + part[3][t].x);
        a.y = bb.y - (part[0][t].y + part[1][t].y + part[2][t].y + part[3][t].y);
      }
      sv[t] = a;
    }
    __syncthreads();
    accr = 0.f;
    acci = 0.f;
#pragma unroll
    for (int k = 0; k < QW; k++) {
      const float2 a = sv[q * QW + k], w = sinv[r][q * QW + k];
      accr += w.x * a.x - w.y * a.y;
      acci += w.x * a.y + w.y * a.x;
    }
    part[q][r] = make_float2(accr, acci);
    __syncthreads();
    float2 xval = make_float2(0.f, 0.f);  // x_v, row t (t < NB)
    if (t < NB)
      xval = make_float2(part[0][t].x + part[1][t].x + part[2][t].x + part[3][t].x,
                         part[0][t].y + part[1][t].y + part[2][t].y + part[3][t].y);
    // this thread's quarter of x_{s-d} in xin[d - 1]: stored there by the
    // cluster peer (each thread polls its quarter, read only), or polled in
    // global memory by one thread per value, which stores it there, and a
    // barrier before anyone reads them (that branch is the same in every
    // thread of the CTA, and its iterations come before the peer ones)
    float2* xq_base = &xin[0][q * QW];
    auto acquire = [&](int d) -> bool {
      const unsigned long long t0 = global_ns();
      long long spins = 0;
      float2* xq = xq_base + (d - 1) * NB;
      if (CS > 0 && rank >= (unsigned)d) {
        // the peer's 64-bit stores land in this CTA's shared memory: poll
        // them until none is still unset
        while (true) {
          bool ready = true;
#pragma unroll
          for (int k = 0; k < QW; k++) {
            const float2 v = ld_volatile_shared_f2(xq + k);
            ready = ready && __float_as_uint(v.x) != kSweepUnset && __float_as_uint(v.y) != kSweepUnset;
          }
          if (ready) return true;
          if (((++spins & 63) == 0 && (*(volatile int*)status & (1 << 9))) || spins > kSweepSpinLimit ||
              global_ns() - t0 > kSweepWaitNs) {
            atomicOr(status, 1 << 9);
            return false;
          }
        }
      }
      bool ok = true;
      if (r < QW) {  // value q * QW + r of x_{s-d}
        const int sp = s - d;
        const int64_t cp = (int64_t)(LOWER ? sp : nblk - 1 - sp) * NB + q * QW + r;
        while (true) {
          const float2 v = cp < n ? ld_relaxed_f2(x + cp) : make_float2(0.f, 0.f);
          if (__float_as_uint(v.x) != kSweepUnset && __float_as_uint(v.y) != kSweepUnset) {
            xq[r] = v;
            break;
          }
          if (((++spins & 63) == 0 && (*(volatile int*)status & (1 << 9))) || spins > kSweepSpinLimit ||
              global_ns() - t0 > kSweepWaitNs) {
            atomicOr(status, 1 << 9);
            ok = false;
            break;
          }
          __nanosleep(20u);
        }
      }
      return !__syncthreads_or(!ok);
    };
    // the last D positions, the oldest first: x_v = c - sum_d W_d x_{s-d}
    float pr = 0.f, pi = 0.f;
    int timed_out = 0;
    for (int d = min(D, s); d >= 1 && !timed_out; d--) {
      if (CS > 0 && d >= 2 && rank >= (unsigned)d) continue;  // the peer sends W_d x_{s-d} itself
      // W_d's quarter row (d >= 2) requested before the wait for its block
      float4 wd[QW / 2];
      if (d >= 2) {
        const float4* wp = reinterpret_cast<const float4*>(wnext + wbase + (d - 1) * NB * NB);
#pragma unroll
        for (int k = 0; k < QW / 2; k++) wd[k] = ld_early_f4(wp + k);
      }
      if (!acquire(d)) {
        timed_out = 1;
        break;
      }
      const float4* xq = reinterpret_cast<const float4*>(xq_base + (d - 1) * NB);
#pragma unroll
      for (int k = 0; k < QW / 2; k++) {
        const float4 w = d == 1 ? wv[k] : wd[k];
        const float4 xx = xq[k];
        pr += w.x * xx.x - w.y * xx.y + w.z * xx.z - w.w * xx.w;
        pi += w.x * xx.y + w.y * xx.x + w.z * xx.w + w.w * xx.z;
      }
    }
    part2[q][r] = make_float2(pr, pi);
    if (__syncthreads_or(timed_out)) return false;  // a wait ran out: every thread leaves
    if (t < NB && s > 0) {
      xval.x -= part2[0][t].x + part2[1][t].x + part2[2][t].x + part2[3][t].x;
      xval.y -= part2[0][t].y + part2[1][t].y + part2[2][t].y + part2[3][t].y;
    }
    if constexpr (CS > 0) {
      // W_d x_{s-d} (d >= 2) computed and sent by the peer: row t of it in
      // xin[d - 1], polled until set
      if (t < NB) {
        for (int d = 2; d <= min(D, s); d++) {
          if (rank < (unsigned)d) continue;
          const unsigned long long t0 = global_ns();
          long long spins = 0;
          while (true) {
            const float2 y = ld_volatile_shared_f2(&xin[d - 1][t]);
            if (__float_as_uint(y.x) != kSweepUnset && __float_as_uint(y.y) != kSweepUnset) {
              xval.x -= y.x;
              xval.y -= y.y;
              break;
            }
            if (((++spins & 63) == 0 && (*(volatile int*)status & (1 << 9))) || spins > kSweepSpinLimit ||
                global_ns() - t0 > kSweepWaitNs) {
              atomicOr(status, 1 << 9);
              break;
            }
          }
        }
      }
      // the next position's CTA in this cluster takes x_v from here: each
      // value is one 64-bit store that the receiver polls, so no fence
      if (t < NB && rank + 1 < (unsigned)CS && s + 1 < nblk)
        st_peer_f2(peer_addr(smem_addr(&xin[0][t]), rank + 1), t < bs ? xval : make_float2(0.f, 0.f));
    }
    if (t < bs) x[r0 + t] = xval;
    // the block's stores are ordered before the counter by the barrier and
    // thread 0's release at device scope
    __syncthreads();
    if (t == 0) st_release_u32(counter, (unsigned)(s + 1));
    if constexpr (CS > 0) {
      // for the CTAs d = 2 .. D positions on in this cluster: W_d of their
      // block times x_v, formed here after the block is out (its rows
      // fetched now, off the chain) and stored into their xin[d - 1]
      if (t < NB) sv[t] = t < bs ? xval : make_float2(0.f, 0.f);
      __syncthreads();
      for (int d = 2; d <= D; d++) {
        if (rank + d >= (unsigned)CS || s + d >= nblk) continue;  // the same in every thread
        const int vs = LOWER ? s + d : nblk - 1 - (s + d);
        const float4* wp = reinterpret_cast<const float4*>(
            wnext + (((int64_t)vs * 2 + (LOWER ? 0 : 1)) * D + (d - 1)) * NB * NB + r * NB + q * QW);
        const float4* xs4 = reinterpret_cast<const float4*>(sv + q * QW);
        float hr = 0.f, hi = 0.f;
#pragma unroll
        for (int k = 0; k < QW / 2; k++) {
          const float4 w = wp[k], xx = xs4[k];
          hr += w.x * xx.x - w.y * xx.y + w.z * xx.z - w.w * xx.w;
          hi += w.x * xx.y + w.y * xx.x + w.z * xx.w + w.w * xx.z;
        }
        part[q][r] = make_float2(hr, hi);
        __syncthreads();
        if (t < NB)
          st_peer_f2(peer_addr(smem_addr(&xin[d - 1][t]), rank + d),
                     make_float2(part[0][t].x + part[1][t].x + part[2][t].x + part[3][t].x,
                                 part[0][t].y + part[1][t].y + part[2][t].y + part[3][t].y));
        __syncthreads();
      }
    }
    return true;
  };
  if constexpr (CS > 0) {
    if ((int)blockIdx.x < nblk) position((int)blockIdx.x);
    cluster_sync_all();
  } else {
    for (int s = blockIdx.x; s < nblk; s += gridDim.x)  // s: position in sweep order
      if (!position(s)) return;
  }
}

// ---------------------------------------------------------------------------
// Adjoint (transposed) solves on the same factors.  With P A = L U,
//   A^T w = phi  <=>  U^T L^T (P w) = phi,
// so the transposed factors M^T (lower part U^T, upper part L^T) and the
// transposed inverted diagonal blocks drive the same sweeps, and the result
// is scattered back through the permutation.

// B = A^T for the n x n leading block (row-major, leading dims lda, ldb)
template <typename T>
__global__ void __launch_bounds__(256) transpose_kernel(const T* A, int64_t lda, T* B, int64_t ldb, int64_t n) {
  __shared__ T tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.y * 32, c0 = (int64_t)blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int r = ty; r < 32; r += 8)
    if (r0 + r < n && c0 + tx < n) tile[r][tx] = A[(r0 + r) * lda + c0 + tx];
  __syncthreads();
  for (int c = ty; c < 32; c += 8)
    if (c0 + c < n && r0 + tx < n) B[(c0 + c) * ldb + r0 + tx] = tile[tx][c];
}

// tinvT[2b] = (U_bb^-1)^T, tinvT[2b+1] = (L_bb^-1)^T: the lower- and
// upper-triangle inverses of the transposed factors
__global__ void __launch_bounds__(256) tinv_transpose_kernel(const float2* tinv, float2* tinvT) {
  constexpr int NB = kBlk;
  const float2* in = tinv + (int64_t)blockIdx.x * 2 * NB * NB;
  float2* out = tinvT + (int64_t)blockIdx.x * 2 * NB * NB;
  for (int e = threadIdx.x; e < NB * NB; e += 256) {
    const int r = e / NB, c = e % NB;
    out[e] = in[NB * NB + c * NB + r];
    out[NB * NB + e] = in[c * NB + r];
  }
}

// x[perm[i]] += d[i]   (x += P^T d)
__global__ void axpy_scatter_kernel(double2* x, const float2* d, const int* perm, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double2 v = x[perm[i]];
  v.x += (double)d[i].x;
  v.y += (double)d[i].y;
  x[perm[i]] = v;
}

// Impedance loading (src/nec_context.cpp:2127-2142): row j of Z loses
// (a + c) * zload[j] at every basis function with support on segment j.
// One thread per segment; rows are distinct, so no two threads meet.
__global__ void load_kernel(int64_t n, const int32_t* cptr, const int32_t* cbasis, const double* ca,
                            const double* cc, const double2* zload, double2* Z, int64_t ld) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const double2 zl = zload[j];
  if (zl.x == 0.0 && zl.y == 0.0) return;
  for (int e = cptr[j]; e < cptr[j + 1]; e++) {
    const double w = ca[e] + cc[e];
    double2* p = Z + j * ld + cbasis[e];
    p->x -= w * zl.x;
    p->y -= w * zl.y;
  }
}

}  // namespace necb
