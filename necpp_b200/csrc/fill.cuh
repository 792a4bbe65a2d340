// Interaction-matrix fill (replaces cmset/cmww, src/nec_context.cpp:2077-2204,
// 2514-2650, for wires).
//
// Z is row-major: Z[obs * ld + basis].  The reference fills the same layout
// (cm[basis + obs*nrow]) by scattering, for each source segment j in turn,
// etk*ax + ets*bx + etc*cx into the <= jsno basis columns that have support
// on j.  Here the scatter is turned into a gather that needs no atomics:
// one CTA owns a tile of TI observation rows x TB basis columns.  The host
// lists, per column tile, the distinct source segments that contribute to
// any of its columns (ascending), and for each such source the (column,
// a, b, c) entries.  Each thread (one observation row) walks that list,
// computes the source's fields once, and accumulates into its row of a
// shared-memory tile.  Because sources are visited in ascending order, every
// element is summed in exactly the reference's order.
#pragma once
#include <cstdint>

#include "field.cuh"

namespace necb {

constexpr int kFillTI = 64;  // observation rows per CTA (= threads)
constexpr int kFillTB = 16;  // basis columns per CTA

struct FillArgs {
  int64_t n, ld;
  // segments (wavelengths)
  const double *x, *y, *z, *s, *b, *cab, *sab, *salp;
  const int32_t *ind1, *ind2;
  // column-tile source lists
  const int32_t* tile_src_ptr;  // [ntiles+1] into tsrc
  const int32_t* tsrc;          // source segment (0-based)
  const int32_t* tsrc_eptr;     // [len(tsrc)+1] into entries
  const uint8_t* ecol;          // column within tile
  const double *ea, *eb, *ec;   // basis coefficients
  FieldParams P;
  double2* Z64;  // row-major FP64 output (may be null)
  float2* Z32;   // row-major FP32 copy (mixed precision; may be null)
  int* status;
};

// Contraction instead of storage (adjoint gradients): out[k] +=
// w_k^T Z x over this structure's Z, for nw vectors w_k (n complex each).
struct ContractArgs {
  const double2* x;  // n
  const double2* w;  // nw x n
  int nw;
  double* out;       // nw complex
};
constexpr int kMaxContract = 4;

// One tile of Z: rows [row0, row0+64) x basis columns of column tile `tile`.
// CONTRACT = false stores the tile (Z64 / Z32); true folds it into C.out.
template <int GROUND, bool EXK, bool CONTRACT>
__device__ __forceinline__ void fill_tile(const FillArgs& A, const ContractArgs& C, int tile, int64_t row0) {
  __shared__ double2 acc[kFillTB][kFillTI + 1];
  const int tid = threadIdx.x;
  const int64_t i = row0 + tid;
  const bool active = i < A.n;
#pragma unroll
  for (int c = 0; c < kFillTB; c++) acc[c][tid] = make_double2(0.0, 0.0);

  double xi = 0, yi = 0, zi = 0, ai = 0, cabi = 0, sabi = 0, salpi = 0;
  if (active) {
    xi = A.x[i];
    yi = A.y[i];
    zi = A.z[i];
    ai = A.b[i];
    cabi = A.cab[i];
    sabi = A.sab[i];
    salpi = A.salp[i];
  }
  int status = 0;
  const int sbeg = A.tile_src_ptr[tile], send = A.tile_src_ptr[tile + 1];
  // the far-pair factor sin(pi s)/pi of the tile's sources, computed once per
  // source by the CTA in chunks of kFillTI instead of once per pair
  __shared__ double sfac[kFillTI];
  for (int sidx = sbeg; sidx < send; sidx++) {
    if ((sidx - sbeg) % kFillTI == 0) {
      __syncthreads();  // the previous chunk's factors are no longer read
      const int q = sidx + tid;
      if (q < send) sfac[tid] = far_sfac(__ldg(A.s + __ldg(A.tsrc + q)));
      __syncthreads();
    }
    const int j = __ldg(A.tsrc + sidx);
    SrcSeg J;
    J.sfac = sfac[(sidx - sbeg) % kFillTI];
    J.x = __ldg(A.x + j);
    J.y = __ldg(A.y + j);
    J.z = __ldg(A.z + j);
    J.s = __ldg(A.s + j);
    J.b = __ldg(A.b + j);
    J.cab = __ldg(A.cab + j);
    J.sab = __ldg(A.sab + j);
    J.salp = __ldg(A.salp + j);
    J.ind1 = EXK ? __ldg(A.ind1 + j) : 0;
    J.ind2 = EXK ? __ldg(A.ind2 + j) : 0;
    if (!active) continue;
    cplx etk, ets, etc;
    pair_field<GROUND, EXK>(J, xi, yi, zi, ai, cabi, sabi, salpi, i != j, A.P, &etk, &ets, &etc,
                            &status, i * A.n + j);
    const int e0 = __ldg(A.tsrc_eptr + sidx), e1 = __ldg(A.tsrc_eptr + sidx + 1);
    for (int e = e0; e < e1; e++) {
      const int c = A.ecol[e];
      const double a = __ldg(A.ea + e), bb = __ldg(A.eb + e), cc = __ldg(A.ec + e);
      cplx v = etk * a + ets * bb + etc * cc;
      double2 t = acc[c][tid];
      t.x += v.re;
      t.y += v.im;
      acc[c][tid] = t;
    }
  }
  if (status) atomicOr(A.status, status);
  __syncthreads();
  const int lane = tid & 31, warp = tid >> 5;
  if (CONTRACT) {
    // row i: t = sum_c Z[i][col0+c] x[col0+c]; out[k] += w_k[i] t
    double tr = 0, ti = 0;
    if (active) {
      const int64_t col0 = (int64_t)tile * kFillTB;
      for (int c = 0; c < kFillTB && col0 + c < A.n; c++) {
        const double2 z = acc[c][tid], xv = C.x[col0 + c];
        tr += z.x * xv.x - z.y * xv.y;
        ti += z.x * xv.y + z.y * xv.x;
      }
    }
    for (int k = 0; k < C.nw; k++) {
      double pr = 0, pi = 0;
      if (active) {
        const double2 wv = C.w[(int64_t)k * A.n + i];
        pr = wv.x * tr - wv.y * ti;
        pi = wv.x * ti + wv.y * tr;
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        pr += __shfl_down_sync(0xffffffffu, pr, off);
        pi += __shfl_down_sync(0xffffffffu, pi, off);
      }
      if (lane == 0) {
        atomicAdd(C.out + 2 * k, pr);
        atomicAdd(C.out + 2 * k + 1, pi);
      }
    }
    return;
  }
  // write out: consecutive threads along a row's (contiguous) columns
  (void)lane;
  (void)warp;
  const int64_t col0 = (int64_t)tile * kFillTB;
  for (int e = tid; e < kFillTI * kFillTB; e += kFillTI) {
    const int r = e / kFillTB, c = e % kFillTB;
    const int64_t row = row0 + r, col = col0 + c;
    if (row < A.n && col < A.n) {
      const double2 v = acc[c][r];
      if (A.Z64) A.Z64[row * A.ld + col] = v;
      if (A.Z32) A.Z32[row * A.ld + col] = make_float2((float)v.x, (float)v.y);
    }
  }
}

// Free space: registers capped so that eight 64-thread CTAs fit an SM (the
// fill is latency-bound at six); the ground variants keep their registers
// (their larger field code spills at the cap).
template <int GROUND, bool EXK>
__global__ void __launch_bounds__(kFillTI, GROUND == 0 ? 8 : 1) fill_kernel(FillArgs A) {
  fill_tile<GROUND, EXK, false>(A, ContractArgs{}, blockIdx.y, (int64_t)blockIdx.x * kFillTI);
}

// Batched fill of perturbed structures (blockIdx.z), each contracted with
// its own output slot: out_s[k] = w_k^T Z_s x.
template <int GROUND, bool EXK>
__global__ void __launch_bounds__(kFillTI) fill_contract_kernel(const FillArgs* __restrict__ As,
                                                                const ContractArgs* __restrict__ Cs) {
  fill_tile<GROUND, EXK, true>(As[blockIdx.z], Cs[blockIdx.z], blockIdx.y, (int64_t)blockIdx.x * kFillTI);
}

}  // namespace necb
