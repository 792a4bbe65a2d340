// Near electric and magnetic fields at points in space from the current
// coefficients of the last solve.
//
// Device restatement of NEC2++ src/nec_context.cpp:
//   nefld 4304-4490 (wires), nhfld 5189-5265 (wires), hsfld 3927-4056,
//   hsflx 4059-4133, hfk 3681-3822, gh 3582-3600.
// One warp per point: lanes take the segments, each evaluates the field of
// its segment's constant, sine and cosine currents (the fill's efld, or
// hsfld for H) and weights it with the segment's coefficients; the warp
// sums.  For Sommerfeld ground, the (point, segment) pairs within the table
// limit of the segment's image go through the ordered cache walk of
// near_field_chain_kernel, whose per-point sums are added here.
#pragma once
#include "field.cuh"
#include "somm.cuh"

namespace necb {

constexpr int kNearWarps = 4;  // points per CTA

struct NearFieldArgs {
  int64_t n;
  const double *x, *y, *z, *s, *b, *cab, *sab, *salp;
  const int32_t *ind1, *ind2;
  FieldParams P;
  int ground;           // kGround*
  const double* abc;    // 6n: air aii bir bii cir cii
  int npts;
  const double* pts;    // 3 per point (wavelengths)
  double2* out;         // 3 per point
  const double2* near;  // Sommerfeld: table-limit pairs' part, 3 per point (or null)
  int* status;
};

__device__ __forceinline__ SrcSeg load_seg(const NearFieldArgs& A, int64_t i, bool exk) {
  SrcSeg J;
  J.x = A.x[i];
  J.y = A.y[i];
  J.z = A.z[i];
  J.s = A.s[i];
  J.b = A.b[i];
  J.cab = A.cab[i];
  J.sab = A.sab[i];
  J.salp = A.salp[i];
  J.ind1 = exk ? A.ind1[i] : 0;
  J.sfac = far_sfac(J.s);
  J.ind2 = exk ? A.ind2[i] : 0;
  return J;
}

__device__ __forceinline__ cplx coef(const double* abc, int64_t n, int64_t i, int k) {
  return mk(abc[2 * k * n + i], abc[(2 * k + 1) * n + i]);
}

// Radius of the first segment whose volume holds the point, else 0
// (nefld 4316-4334), rounded as the reference rounds it.
__device__ double point_radius_warp(const NearFieldArgs& A, double xob, double yob, double zob) {
  const int lane = threadIdx.x & 31;
  for (int64_t i0 = 0; i0 < A.n; i0 += 32) {
    const int64_t i = i0 + lane;
    bool hit = false;
    if (i < A.n) {
      const double xj = xob - A.x[i], yj = yob - A.y[i], zj = zob - A.z[i];
      double zp = __dadd_rn(__dadd_rn(__dmul_rn(A.cab[i], xj), __dmul_rn(A.sab[i], yj)), __dmul_rn(A.salp[i], zj));
      if (!(fabs(zp) > __dmul_rn(0.5001, A.s[i]))) {
        const double d2 = __dsub_rn(
            __dadd_rn(__dadd_rn(__dmul_rn(xj, xj), __dmul_rn(yj, yj)), __dmul_rn(zj, zj)), __dmul_rn(zp, zp));
        hit = !(d2 > __dmul_rn(__dmul_rn(0.9, A.b[i]), A.b[i]));
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    if (m) return A.b[i0 + __ffs(m) - 1];
  }
  return 0.0;
}

__device__ __forceinline__ void warp_sum3(cplx f[3]) {
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      f[k].re += __shfl_down_sync(0xffffffffu, f[k].re, off);
      f[k].im += __shfl_down_sync(0xffffffffu, f[k].im, off);
    }
}

template <int GROUND, bool EXK>
__global__ void __launch_bounds__(32 * kNearWarps) near_e_kernel(NearFieldArgs A) {
  const int p = blockIdx.x * kNearWarps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= A.npts) return;
  const double xob = A.pts[3 * p], yob = A.pts[3 * p + 1], zob = A.pts[3 * p + 2];
  const double ax = point_radius_warp(A, xob, yob, zob);
  cplx f[3] = {mk(0, 0), mk(0, 0), mk(0, 0)};
  int status = 0;
  for (int64_t i = lane; i < A.n; i += 32) {
    const SrcSeg J = load_seg(A, i, EXK);
    cplx e[9];
    if (GROUND == kGroundSommerfeld) {
      const double r = image_r2(xob - J.x, yob - J.y, zob + J.z);
      if (r <= .95) {
        if (!A.near) status |= kStatSommerfeldTab;
        continue;  // the ordered walk supplies these pairs
      }
      pair_fields9<GROUND, EXK>(J, xob, yob, zob, ax, true, A.P, e, &status);
      cplx g[9];
      const SommGeom sg = somm_geometry(J, xob, yob, zob, ax);
      norton_field(J, sg, xob - J.x, yob - J.y, zob + J.z, r, ax, A.P, g);
#pragma unroll
      for (int k = 0; k < 9; k++) e[k] = e[k] + g[k];
    } else {
      pair_fields9<GROUND, EXK>(J, xob, yob, zob, ax, true, A.P, e, &status);
    }
    const cplx ac = coef(A.abc, A.n, i, 0), bc = coef(A.abc, A.n, i, 1), cc = coef(A.abc, A.n, i, 2);
    f[0] += e[0] * ac + e[3] * bc + e[6] * cc;
    f[1] += e[1] * ac + e[4] * bc + e[7] * cc;
    f[2] += e[2] * ac + e[5] * bc + e[8] * cc;
  }
  warp_sum3(f);
  if (status) atomicOr(A.status, status);
  if (lane == 0) {
    for (int k = 0; k < 3; k++) {
      cplx v = f[k];
      if (A.near) v += mk(A.near[3 * p + k].x, A.near[3 * p + k].y);
      A.out[3 * p + k] = make_double2(v.re, v.im);
    }
  }
}

// Sommerfeld ground: the (point, segment) pairs within the table limit, in
// the reference's order (points in turn, segments ascending), one thread
// per listed point from the cache `entry[p]`, or (chain) one thread over
// all listed points in order.  Sums into near[3 * p].
template <bool EXK>
__global__ void __launch_bounds__(64) near_field_chain_kernel(NearFieldArgs A, const double* __restrict__ axs,
                                                              const cplx* __restrict__ tab,
                                                              const int* __restrict__ units, int nunits,
                                                              const InterpKey* __restrict__ entry,
                                                              const InterpCache* __restrict__ carried,
                                                              NearRecord* __restrict__ rec, double2* __restrict__ near,
                                                              int chain) {
  int k0, k1;
  if (chain) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    k0 = 0;
    k1 = nunits;
  } else {
    k0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (k0 >= nunits) return;
    k1 = k0 + 1;
  }
  InterpCache S;
  InterpKey key = entry[units[k0]];
  interp_restore(S, key, tab, carried);
  int status = 0;
  for (int k = k0; k < k1; k++) {
    const int p = units[k];
    const double xob = A.pts[3 * p], yob = A.pts[3 * p + 1], zob = A.pts[3 * p + 2], ax = axs[p];
    NearRecord r;
    r.has_near = 0;
    r.used = key;
    r.x1 = r.y1 = 0.0;
    cplx f[3] = {mk(0, 0), mk(0, 0), mk(0, 0)};
    for (int64_t i = 0; i < A.n; i++) {
      const SrcSeg J = load_seg(A, i, EXK);
      if (image_r2(xob - J.x, yob - J.y, zob + J.z) > .95) continue;
      double2 s1;
      cplx e[9];
      near_efld9<EXK>(J, xob, yob, zob, ax, true, A.P, A.n, S, tab, r.has_near ? nullptr : &s1, e, &status);
      if (!r.has_near) {
        r.has_near = 1;
        r.x1 = s1.x;
        r.y1 = s1.y;
      }
      const cplx ac = coef(A.abc, A.n, i, 0), bc = coef(A.abc, A.n, i, 1), cc = coef(A.abc, A.n, i, 2);
      f[0] += e[0] * ac + e[3] * bc + e[6] * cc;
      f[1] += e[1] * ac + e[4] * bc + e[7] * cc;
      f[2] += e[2] * ac + e[5] * bc + e[8] * cc;
    }
    for (int c = 0; c < 3; c++) near[3 * p + c] = make_double2(f[c].re, f[c].im);
    key = InterpKey{S.igrs, S.ix, S.iy, S.carry};
    r.exit = key;
    rec[p] = r;
  }
  if (status) atomicOr(A.status, status);
}

// observer radius of every point (one warp per point)
__global__ void __launch_bounds__(32 * kNearWarps) near_radius_kernel(NearFieldArgs A, double* axs) {
  const int p = blockIdx.x * kNearWarps + (threadIdx.x >> 5);
  if (p >= A.npts) return;
  const double ax = point_radius_warp(A, A.pts[3 * p], A.pts[3 * p + 1], A.pts[3 * p + 2]);
  if ((threadIdx.x & 31) == 0) axs[p] = ax;
}

// ---- magnetic field ----

// H-field integrand of a filament, gh 3582-3600
__device__ __forceinline__ void gh(double zk, double zpka, double rhks, double* hr, double* hi) {
  double rs = zk - zpka;
  rs = rhks + rs * rs;
  const double r = sqrt(rs);
  double skr, ckr;
  sincos(r, &skr, &ckr);
  const double rr2 = 1. / rs, rr3 = rr2 / r;
  *hr = skr * rr2 + ckr * rr3;
  *hi = ckr * rr2 - skr * rr3;
}

// hfk 3681-3822: H of a uniform filament by variable-interval Romberg
// integration (bounded: at most nma halvings, then accepted)
__device__ void hfk(double el1, double el2, double rhk, double zpkx, double* sgr, double* sgi, int* status) {
  const int nx = 1, nma = 65536, nts = 4;
  const double rx = 1.0e-4;
  const double rhks = rhk * rhk;
  double z = el1;
  const double ze = el2, s = ze - z, ep = s / (10. * nma), zend = ze - ep;
  double dz = 0., dzot = 0.;
  double g1r, g1i, g2r, g2i, g3r, g3i, g4r, g4i, g5r, g5i, te1r, te1i, te2r, te2i;
  *sgr = 0.0;
  *sgi = 0.0;
  int ns = nx, nt = 0;
  bool flag = true;
  gh(z, zpkx, rhks, &g1r, &g1i);
  for (int guard = 0; guard < 4 * nma + 64; guard++) {
    if (flag) {
      dz = s / ns;
      if (z + dz > ze) {
        dz = ze - z;
        if (fabs(dz) <= ep) {
          *sgr = *sgr * rhk * .5;
          *sgi = *sgi * rhk * .5;
          return;
        }
      }
      dzot = dz * .5;
      gh(z + dzot, zpkx, rhks, &g3r, &g3i);
      gh(z + dz, zpkx, rhks, &g5r, &g5i);
    }
    const double t00r = (g1r + g5r) * dzot, t00i = (g1i + g5i) * dzot;
    const double t01r = (t00r + dz * g3r) * 0.5, t01i = (t00i + dz * g3i) * 0.5;
    const double t10r = (4.0 * t01r - t00r) / 3.0, t10i = (4.0 * t01i - t00i) / 3.0;
    conv_test(t01r, t10r, &te1r, t01i, t10i, &te1i);
    double addr, addi;
    if ((te1i <= rx) && (te1r <= rx)) {
      addr = t10r;
      addi = t10i;
      nt += 2;
    } else {
      gh(z + dz * 0.25, zpkx, rhks, &g2r, &g2i);
      gh(z + dz * 0.75, zpkx, rhks, &g4r, &g4i);
      const double t02r = (t01r + dzot * (g2r + g4r)) * 0.5, t02i = (t01i + dzot * (g2i + g4i)) * 0.5;
      const double t11r = (4.0 * t02r - t01r) / 3.0, t11i = (4.0 * t02i - t01i) / 3.0;
      const double t20r = (16.0 * t11r - t10r) / 15.0, t20i = (16.0 * t11i - t10i) / 15.0;
      conv_test(t11r, t20r, &te2r, t11i, t20i, &te2i);
      if ((te2i > rx) || (te2r > rx)) {
        nt = 0;
        if (ns < nma) {
          ns = ns * 2;
          dz = s / ns;
          dzot = dz * 0.5;
          g5r = g3r;
          g5i = g3i;
          g3r = g2r;
          g3i = g2i;
          flag = false;
          continue;
        }
        *status |= kStatRombergCap;
      }
      addr = t20r;
      addi = t20i;
      nt++;
    }
    *sgr = *sgr + addr;
    *sgi = *sgi + addi;
    z += dz;
    if (z >= zend) {
      *sgr = *sgr * rhk * .5;
      *sgi = *sgi * rhk * .5;
      return;
    }
    g1r = g5r;
    g1i = g5i;
    if (nt >= nts && ns > nx) {
      ns = ns / 2;
      nt = 1;
    }
    flag = true;
  }
  *status |= kStatIterCap;
}

// hsflx 4059-4133: H of the constant, sine and cosine currents of a segment
__device__ void hsflx(double s, double rh, double zpx, cplx* hpk, cplx* hps, cplx* hpc, int* status) {
  const double pi8 = kPiD * 8.0;
  const cplx fjk = -mk(0.0, kTwoPiD);
  if (rh >= 1.0e-10) {
    double zp, hss;
    if (zpx >= 0.0) {
      zp = zpx;
      hss = 1.;
    } else {
      zp = -zpx;
      hss = -1.;
    }
    const double dh = 0.5 * s, z1 = zp + dh, z2a = zp - dh;
    const double rhz = (z2a >= 1.0e-7) ? rh / z2a : 1.;
    const double dk = kTwoPiD * dh;
    double sdk, cdk;
    sincos(dk, &sdk, &cdk);
    double hkr, hki;
    hfk(-dk, dk, rh * kTwoPiD, zp * kTwoPiD, &hkr, &hki, status);
    *hpk = mk(hkr, hki);
    if (rhz >= 1.0e-3) {
      const double rh2 = rh * rh, r1 = sqrt(rh2 + z1 * z1), r2 = sqrt(rh2 + z2a * z2a);
      const cplx ekr1 = cexp_(fjk * r1), ekr2 = cexp_(fjk * r2);
      const cplx t1 = z1 * ekr1 / r1, t2 = z2a * ekr2 / r2;
      cplx ps = (cdk * (ekr2 - ekr1) - mk(0.0, sdk) * (t2 + t1)) * hss;
      cplx pc = -sdk * (ekr2 + ekr1) - mk(0.0, cdk) * (t2 - t1);
      const cplx cons = -mk(0.0, 1.0) / (2.0 * kTwoPiD * rh);
      *hps = cons * ps;
      *hpc = cons * pc;
      return;
    }
    const cplx ekr1 = mk(cdk, sdk) / (z2a * z2a), ekr2 = mk(cdk, -sdk) / (z1 * z1);
    const double t1 = kTwoPiD * (1.0 / z1 - 1.0 / z2a);
    const cplx t2 = cexp_(fjk * zp) * rh / pi8;
    *hps = t2 * (t1 + (ekr1 + ekr2) * sdk) * hss;
    *hpc = t2 * (-mk(0.0, 1.0) * t1 + (ekr1 - ekr2) * cdk);
    return;
  }
  *hps = mk(0, 0);
  *hpc = mk(0, 0);
  *hpk = mk(0, 0);
}

// hsfld 3927-4056: H of segment J at (xi, yi, zi) with its image (a
// perfect image, or the reflection-coefficient approximation for any
// finite ground)
__device__ void hsfld(const SrcSeg& J, double xi, double yi, double zi, double ai, int ground, cplx zrati,
                      cplx h[9], int* status) {
  const double xij = xi - J.x, yij = yi - J.y;
  const int ksymp = ground != kGroundNone ? 2 : 1;
  double rfl = -1.;
#pragma unroll
  for (int k = 0; k < 9; k++) h[k] = mk(0, 0);
  for (int gl = 0; gl < ksymp; gl++) {
    rfl = -rfl;
    const double salpr = J.salp * rfl, zij = zi - rfl * J.z;
    const double zp = xij * J.cab + yij * J.sab + zij * salpr;
    double rhox = xij - J.cab * zp, rhoy = yij - J.sab * zp, rhoz = zij - salpr * zp;
    const double rh = sqrt(rhox * rhox + rhoy * rhoy + rhoz * rhoz + ai * ai);
    if (rh <= 1.0e-10) {
#pragma unroll
      for (int k = 0; k < 9; k++) h[k] = mk(0, 0);
      continue;
    }
    rhox = rhox / rh;
    rhoy = rhoy / rh;
    rhoz = rhoz / rh;
    const double phx = J.sab * rhoz - salpr * rhoy, phy = salpr * rhox - J.cab * rhoz,
                 phz = J.cab * rhoy - J.sab * rhox;
    cplx hp[3];
    hsflx(J.s, rh, zp, &hp[0], &hp[1], &hp[2], status);
    if (gl == 1) {
      if (ground != kGroundPerfect) {
        const cplx zratx = zrati;
        const double rmag = sqrt(zp * zp + rh * rh), xymag = sqrt(xij * xij + yij * yij);
        double px, py, cth;
        cplx rrv, rrh;
        if (xymag <= 1.0e-6) {
          px = 0.;
          py = 0.;
          cth = 1.;
          rrv = mk(1.0, 0.0);
        } else {
          px = -yij / xymag;
          py = xij / xymag;
          cth = zij / rmag;
          rrv = csqrt_(1. - zratx * zratx * (1. - cth * cth));
        }
        rrh = zratx * cth;
        rrh = -(rrh - rrv) / (rrh + rrv);
        rrv = zratx * rrv;
        rrv = (cth - rrv) / (cth + rrv);
        cplx qy = (phx * px + phy * py) * (rrv - rrh);
        const cplx qx = qy * px + phx * rrh;
        qy = qy * py + phy * rrh;
        const cplx qz = phz * rrh;
#pragma unroll
        for (int k = 0; k < 3; k++) {
          h[3 * k] = h[3 * k] - hp[k] * qx;
          h[3 * k + 1] = h[3 * k + 1] - hp[k] * qy;
          h[3 * k + 2] = h[3 * k + 2] - hp[k] * qz;
        }
        continue;
      }
#pragma unroll
      for (int k = 0; k < 3; k++) {
        h[3 * k] = h[3 * k] - hp[k] * phx;
        h[3 * k + 1] = h[3 * k + 1] - hp[k] * phy;
        h[3 * k + 2] = h[3 * k + 2] - hp[k] * phz;
      }
      continue;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
      h[3 * k] = hp[k] * phx;
      h[3 * k + 1] = hp[k] * phy;
      h[3 * k + 2] = hp[k] * phz;
    }
  }
}

__global__ void __launch_bounds__(32 * kNearWarps) near_h_kernel(NearFieldArgs A) {
  const int p = blockIdx.x * kNearWarps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= A.npts) return;
  const double xob = A.pts[3 * p], yob = A.pts[3 * p + 1], zob = A.pts[3 * p + 2];
  const double ax = point_radius_warp(A, xob, yob, zob);
  cplx f[3] = {mk(0, 0), mk(0, 0), mk(0, 0)};
  int status = 0;
  for (int64_t i = lane; i < A.n; i += 32) {
    const SrcSeg J = load_seg(A, i, false);
    cplx h[9];
    hsfld(J, xob, yob, zob, ax, A.ground, A.P.zrati, h, &status);
    const cplx ac = coef(A.abc, A.n, i, 0), bc = coef(A.abc, A.n, i, 1), cc = coef(A.abc, A.n, i, 2);
    f[0] += h[0] * ac + h[3] * bc + h[6] * cc;
    f[1] += h[1] * ac + h[4] * bc + h[7] * cc;
    f[2] += h[2] * ac + h[5] * bc + h[8] * cc;
  }
  warp_sum3(f);
  if (status) atomicOr(A.status, status);
  if (lane == 0)
    for (int k = 0; k < 3; k++) A.out[3 * p + k] = make_double2(f[k].re, f[k].im);
}

}  // namespace necb
