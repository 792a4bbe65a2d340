// Far-field sum (replaces ffld, src/nec_context.cpp:6639-6888, wire part,
// free space and infinite-ground image with reflection coefficients).
//
// One warp per direction; a CTA of PAT_DIRS warps stages segment data and
// current coefficients through shared memory in chunks so each datum is read
// from L2 once per CTA.  Per (direction, segment) the work is two sincos:
// the segment shape factors a, b, c of the sine/cosine/constant current
// components (sin(pi s (1 +- omega)) from the staged sin and cos of pi s by
// the addition formula) and the phase exp(j 2pi r.r_i).
#pragma once
#include <cstdint>

#include "cplx.cuh"

namespace necb {

constexpr int kPatDirs = 8;      // warps (directions) per CTA
constexpr int kPatChunk = 256;   // segments staged per step

struct PatternArgs {
  int64_t n;
  int ndir;
  const double *theta, *phi;
  const double *x, *y, *z, *s, *cab, *sab, *salp;
  const double* abc;  // air aii bir bii cir cii (n each)
  int ksymp;          // 1 free space, 2 image
  int perfect;        // image: perfect ground
  cplx zrati;
  double eta;
  double2 *eth, *eph;
};

struct SegPat {
  double x, y, z, s, cab, sab, salp, air, aii, bir, bii, cir, cii;
  double sel, cel;  // sin and cos of el = pi s (per segment, set when staged)
};

// the per-segment part of a SegPat's shape factors
__device__ __forceinline__ void seg_pat_el(SegPat& g) {
  const double pi = 3.1415926536;
  sincos(pi * g.s, &g.sel, &g.cel);
}

__device__ __forceinline__ void seg_term(const SegPat& g, double rox, double roy, double roz,
                                         cplx* exa) {
  const double pi = 3.1415926536;
  double omega = -(rox * g.cab + roy * g.sab + roz * g.salp);
  double el = pi * g.s;
  double sill = omega * el;
  double top = el + sill;
  double bot = el - sill;
  // one sincos per term: sin(el +- sill) from the segment's sin / cos of el
  double ssill, csill;
  sincos(sill, &ssill, &csill);
  const double stop = g.sel * csill + g.cel * ssill, sbot = g.sel * csill - g.cel * ssill;
  double a, too, boo;
  if (fabs(omega) >= 1.0e-7 && fabs(top) >= 1.0e-7 && fabs(bot) >= 1.0e-7) {
    // the usual case: the three quotients from one reciprocal
    const double ob = omega * bot, r = 1.0 / (ob * top);
    a = 2. * ssill * (top * bot * r);
    too = stop * (ob * r);
    boo = sbot * (omega * top * r);
  } else {
    if (fabs(omega) >= 1.0e-7)
      a = 2. * ssill / omega;
    else
      a = (2. - omega * omega * el * el / 3.) * el;
    if (fabs(top) >= 1.0e-7)
      too = stop / top;
    else
      too = 1. - top * top / 6.;
    if (fabs(bot) >= 1.0e-7)
      boo = sbot / bot;
    else
      boo = 1. - bot * bot / 6.;
  }
  double b = el * (boo - too);
  double c = el * (boo + too);
  double rr = a * g.air + b * g.bii + c * g.cir;
  double ri = a * g.aii - b * g.bir + c * g.cii;
  // the phase 2 pi r.r_i (pi the constant above) as sincospi of
  // r.r_i * 2 pi / pi_exact: the reduction of a multiple of pi is exact
  constexpr double kTwoPiOverPi = 2.0 * 3.1415926536 / 3.141592653589793;
  double sn, cs;
  sincospi(kTwoPiOverPi * (g.x * rox + g.y * roy + g.z * roz), &sn, &cs);
  *exa = mk(cs, sn) * mk(rr, ri);
}

__global__ void __launch_bounds__(kPatDirs * 32) pattern_kernel(PatternArgs A) {
  __shared__ SegPat seg[kPatChunk];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int d = blockIdx.x * kPatDirs + warp;
  const bool active = d < A.ndir;
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
    for (int64_t c0 = 0; c0 < A.n; c0 += kPatChunk) {
      __syncthreads();
      for (int t = threadIdx.x; t < kPatChunk; t += blockDim.x) {
        int64_t i = c0 + t;
        if (i < A.n) {
          SegPat g;
          g.x = A.x[i];
          g.y = A.y[i];
          g.z = A.z[i];
          g.s = A.s[i];
          g.cab = A.cab[i];
          g.sab = A.sab[i];
          g.salp = A.salp[i];
          g.air = A.abc[i];
          g.aii = A.abc[A.n + i];
          g.bir = A.abc[2 * A.n + i];
          g.bii = A.abc[3 * A.n + i];
          g.cir = A.abc[4 * A.n + i];
          g.cii = A.abc[5 * A.n + i];
          seg_pat_el(g);
          seg[t] = g;
        }
      }
      __syncthreads();
      if (active) {
        const int cnt = (int)min((int64_t)kPatChunk, A.n - c0);
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
      const double roz = roz0;
      cplx zrsin = csqrt_(1. - A.zrati * A.zrati * thz * thz);
      rrv = -(roz - A.zrati * zrsin) / (roz + A.zrati * zrsin);
      rrh = (A.zrati * roz - zrsin) / (A.zrati * roz + zrsin);
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
  A.eth[d] = make_double2(e_t.re, e_t.im);
  A.eph[d] = make_double2(e_p.re, e_p.im);
}

// ---------------------------------------------------------------------------
// Far field of one direction as a linear functional of the basis amplitudes
// x (adjoint gradients).  Per segment the sum above adds
//     exa_k = e^{j arg_k} (a_k A - j b_k B + c_k C),  k = direct, image,
// with A = air + j aii, B = bir + j bii, C = cir + j cii the segment's
// current coefficients, and E_theta, E_phi are linear in the exa_k.

struct FarDir {
  double phx, phy, thx, thy, thz, rox, roy, roz0;
  cplx rrv, rrh, C3;
  int ksymp;
};

__host__ __device__ inline FarDir far_dir(double theta, double phi, int ksymp, int perfect, cplx zrati, double eta) {
  FarDir d;
  const double sp = sin(phi), cp = cos(phi), st = sin(theta), ct = cos(theta);
  d.phx = -sp;
  d.phy = cp;
  d.roz0 = ct;
  d.thx = d.roz0 * d.phy;
  d.thy = -d.roz0 * d.phx;
  d.thz = -st;
  d.rox = -d.thz * d.phy;
  d.roy = d.thz * d.phx;
  d.ksymp = ksymp;
  d.rrv = mk(-1.0, -0.0);
  d.rrh = mk(-1.0, -0.0);
  if (ksymp == 2 && !perfect) {
    cplx zrsin = csqrt_(1. - zrati * zrati * d.thz * d.thz);
    d.rrv = -(d.roz0 - zrati * zrsin) / (d.roz0 + zrati * zrsin);
    d.rrh = (zrati * d.roz0 - zrsin) / (zrati * d.roz0 + zrsin);
  }
  d.C3 = mk(0.0, -eta / (4.0 * 3.1415926536));
  return d;
}

// shape factors a, b, c and phase of one segment (the arithmetic of seg_term)
__device__ __forceinline__ void seg_shape(double x, double y, double z, double s, double cab, double sab,
                                          double salp, double rox, double roy, double roz, double* a, double* b,
                                          double* c, cplx* ph) {
  const double pi = 3.1415926536;
  double omega = -(rox * cab + roy * sab + roz * salp);
  double el = pi * s;
  double sill = omega * el;
  double top = el + sill;
  double bot = el - sill;
  double too, boo;
  if (fabs(omega) >= 1.0e-7)
    *a = 2. * sin(sill) / omega;
  else
    *a = (2. - omega * omega * el * el / 3.) * el;
  if (fabs(top) >= 1.0e-7)
    too = sin(top) / top;
  else
    too = 1. - top * top / 6.;
  if (fabs(bot) >= 1.0e-7)
    boo = sin(bot) / bot;
  else
    boo = 1. - bot * bot / 6.;
  *b = el * (boo - too);
  *c = el * (boo + too);
  double sn, cs;
  sincos(2.0 * pi * (x * rox + y * roy + z * roz), &sn, &cs);
  *ph = mk(cs, sn);
}

// d E_theta / d exa_k and d E_phi / d exa_k of a segment with direction
// cosines (cab, sab, salp)
__device__ __forceinline__ void exa_weights(const FarDir& d, double cab, double sab, double salp, cplx wt[2],
                                            cplx wp[2]) {
  wt[0] = d.C3 * (d.thx * cab + d.thy * sab + d.thz * salp);
  wp[0] = d.C3 * (d.phx * cab + d.phy * sab);
  if (d.ksymp == 2) {
    const cplx rd = d.rrh - d.rrv;
    const double dp = cab * d.phx + sab * d.phy;
    const cplx gx = d.rrv * cab + rd * (dp * d.phx);
    const cplx gy = d.rrv * sab + rd * (dp * d.phy);
    const cplx gz = -(d.rrv * salp);
    wt[1] = d.C3 * (gx * d.thx + gy * d.thy + gz * d.thz);
    wp[1] = d.C3 * (gx * d.phx + gy * d.phy);
  } else {
    wt[1] = mk(0, 0);
    wp[1] = mk(0, 0);
  }
}

// phi_t[j], phi_p[j] (zeroed by the caller): E_theta = phi_t^T x and
// E_phi = phi_p^T x.  One thread per segment; scattered to the basis
// functions with support on the segment.
__global__ void pattern_weights_kernel(int64_t n, FarDir d, const double* seg, const int32_t* cptr,
                                       const int32_t* cbasis, const double* ca, const double* cb, const double* cc,
                                       double* phi_t, double* phi_p) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = seg[i], y = seg[n + i], z = seg[2 * n + i], s = seg[3 * n + i];
  const double cab = seg[5 * n + i], sab = seg[6 * n + i], salp = seg[7 * n + i];
  cplx wt[2], wp[2];
  exa_weights(d, cab, sab, salp, wt, wp);
  cplx tA = mk(0, 0), tB = mk(0, 0), tC = mk(0, 0), pA = mk(0, 0), pB = mk(0, 0), pC = mk(0, 0);
  for (int k = 0; k < d.ksymp; k++) {
    double a, b, c;
    cplx ph;
    seg_shape(x, y, z, s, cab, sab, salp, d.rox, d.roy, k == 0 ? d.roz0 : -d.roz0, &a, &b, &c, &ph);
    const cplx eA = ph * a, eB = ph * mk(0.0, -b), eC = ph * c;
    tA += wt[k] * eA;
    tB += wt[k] * eB;
    tC += wt[k] * eC;
    pA += wp[k] * eA;
    pB += wp[k] * eB;
    pC += wp[k] * eC;
  }
  for (int e = cptr[i]; e < cptr[i + 1]; e++) {
    const int64_t j = cbasis[e];
    const cplx vt = tA * ca[e] + tB * cb[e] + tC * cc[e];
    const cplx vp = pA * ca[e] + pB * cb[e] + pC * cc[e];
    atomicAdd(phi_t + 2 * j, vt.re);
    atomicAdd(phi_t + 2 * j + 1, vt.im);
    atomicAdd(phi_p + 2 * j, vp.re);
    atomicAdd(phi_p + 2 * j + 1, vp.im);
  }
}

// Far field of the fixed amplitudes x on each of a batch of structures
// (blockIdx.x = structure; its segments seg_s and coefficients ccoef_s, the
// table layout cptr / cbasis shared): out[s] = (E_theta, E_phi).
constexpr int kFarBatchThreads = 256;
__global__ void __launch_bounds__(kFarBatchThreads) far_batch_kernel(int64_t n, int64_t nc, FarDir d,
                                                                     const double* segs, const int32_t* cptr,
                                                                     const int32_t* cbasis, const double* ccoefs,
                                                                     const double2* x, double2* out) {
  __shared__ cplx red[kFarBatchThreads / 32][2];
  const double* seg = segs + (int64_t)blockIdx.x * 8 * n;
  const double* ca = ccoefs + (int64_t)blockIdx.x * 3 * nc;
  const double* cb = ca + nc;
  const double* cc = ca + 2 * nc;
  cplx et = mk(0, 0), ep = mk(0, 0);
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const double xx = seg[i], yy = seg[n + i], zz = seg[2 * n + i], s = seg[3 * n + i];
    const double cab = seg[5 * n + i], sab = seg[6 * n + i], salp = seg[7 * n + i];
    cplx A = mk(0, 0), B = mk(0, 0), C = mk(0, 0);
    for (int e = cptr[i]; e < cptr[i + 1]; e++) {
      const double2 xv = x[cbasis[e]];
      const cplx v = mk(xv.x, xv.y);
      A += v * ca[e];
      B += v * cb[e];
      C += v * cc[e];
    }
    cplx wt[2], wp[2];
    exa_weights(d, cab, sab, salp, wt, wp);
    for (int k = 0; k < d.ksymp; k++) {
      double a, b, c;
      cplx ph;
      seg_shape(xx, yy, zz, s, cab, sab, salp, d.rox, d.roy, k == 0 ? d.roz0 : -d.roz0, &a, &b, &c, &ph);
      const cplx exa = ph * (A * a + B * mk(0.0, -b) + C * c);
      et += wt[k] * exa;
      ep += wp[k] * exa;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    et.re += __shfl_down_sync(0xffffffffu, et.re, off);
    et.im += __shfl_down_sync(0xffffffffu, et.im, off);
    ep.re += __shfl_down_sync(0xffffffffu, ep.re, off);
    ep.im += __shfl_down_sync(0xffffffffu, ep.im, off);
  }
  if (lane == 0) {
    red[warp][0] = et;
    red[warp][1] = ep;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    cplx t = mk(0, 0), p = mk(0, 0);
    for (int w = 0; w < kFarBatchThreads / 32; w++) {
      t += red[w][0];
      p += red[w][1];
    }
    out[2 * blockIdx.x] = make_double2(t.re, t.im);
    out[2 * blockIdx.x + 1] = make_double2(p.re, p.im);
  }
}

}  // namespace necb
