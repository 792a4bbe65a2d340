// Far-field sum (replaces ffld, src/nec_context.cpp:6639-6888, wire part,
// free space and infinite-ground image with reflection coefficients).
//
// One warp per direction; a CTA of PAT_DIRS warps stages segment data and
// current coefficients through shared memory in chunks so each datum is read
// from L2 once per CTA.  Per (direction, segment) the work is four sines and
// one sincos: the segment shape factors a, b, c of the sine/cosine/constant
// current components and the phase exp(j 2pi r.r_i).
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
};

__device__ __forceinline__ void seg_term(const SegPat& g, double rox, double roy, double roz,
                                         cplx* exa) {
  const double pi = 3.1415926536;
  double omega = -(rox * g.cab + roy * g.sab + roz * g.salp);
  double el = pi * g.s;
  double sill = omega * el;
  double top = el + sill;
  double bot = el - sill;
  double a, too, boo;
  if (fabs(omega) >= 1.0e-7)
    a = 2. * sin(sill) / omega;
  else
    a = (2. - omega * omega * el * el / 3.) * el;
  if (fabs(top) >= 1.0e-7)
    too = sin(top) / top;
  else
    too = 1. - top * top / 6.;
  if (fabs(bot) >= 1.0e-7)
    boo = sin(bot) / bot;
  else
    boo = 1. - bot * bot / 6.;
  double b = el * (boo - too);
  double c = el * (boo + too);
  double rr = a * g.air + b * g.bii + c * g.cir;
  double ri = a * g.aii - b * g.bir + c * g.cii;
  double arg = 2.0 * pi * (g.x * rox + g.y * roy + g.z * roz);
  double sn, cs;
  sincos(arg, &sn, &cs);
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

}  // namespace necb
