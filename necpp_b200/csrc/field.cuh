// Electric field of the constant, sine and cosine current filaments of one
// source segment at one observation point: the per-pair work of the fill.
//
// Device restatement of NEC2++ src/nec_context.cpp:
//   efld_compute 2777-2843, efld 2845-3045, eksc 3051-3104, ekscx 3108-3188,
//   gf 3553-3578, gx 3605-3620, gxx 3623-3676, intx 4135-4300,
//   sflds (Norton branch) 6024-6141;
// src/c_ggrid.cpp: fbar 291-350, gwave 351-432; src/c_evlcom.cpp: test 845-868.
// The adaptive Romberg integration keeps the reference's decision sequence
// (3-point then 5-point tests, step doubling after nts accepted steps,
// halving down to s/65536) so near-pair elements agree to rounding.
#pragma once
#include "cplx.cuh"

namespace necb {

constexpr double kPiD = 3.1415926536;  // pi() of math_util.h:72-74
constexpr double kTwoPiD = 2.0 * kPiD;
constexpr double kC1 = 4.771341189;  // __const1 = j*4.771341189

// status bits reported by the fill
enum : int {
  kStatRombergCap = 1,     // intx hit the step-size limit ("STEP SIZE LIMITED")
  kStatIterCap = 2,        // a quadrature exceeded its iteration bound
  kStatSommerfeldTab = 4,  // a pair needs the Sommerfeld table path (r <= 0.95)
};

struct SrcSeg {
  double x, y, z, s, b, cab, sab, salp;
  int ind1, ind2;
  double sfac;  // far_sfac(s): set by whoever builds the SrcSeg
};

// sin(pi s) / pi of efld_compute's far branch (2815), once per source
__device__ __forceinline__ double far_sfac(double s) { return sin(kPiD * s) / kPiD; }

struct FieldParams {
  double rkh;
  double eta;       // wave impedance of the medium
  cplx zrati;       // 1/sqrt(eps_c)
  cplx frati;       // image scale factor
  cplx u, u2;       // ground-wave constants (u = zrati)
  // Sommerfeld ground: projected fields (etk, ets, etc) of the pairs closer
  // than the table limit to their image, precomputed in the reference's
  // order by near_ground_kernel; [(obs * near_n + src) * 3 + k], or null
  const cplx* near_g;
  int64_t near_n;
};

// Squared distance from an observation point to a source's image (the
// table / Norton switch of efld, 2993-2995), rounded as the reference rounds
// it (no fused multiply-add) so every kernel takes the same branch.
__device__ __forceinline__ double image_r2(double xij, double yij, double zij) {
  return __dadd_rn(__dadd_rn(__dmul_rn(xij, xij), __dmul_rn(yij, yij)), __dmul_rn(zij, zij));
}

// c_evlcom.cpp:845-868
__device__ __forceinline__ void conv_test(double f1r, double f2r, double* tr, double f1i,
                                          double f2i, double* ti) {
  double den = fabs(f2r);
  double t = fabs(f2i);
  if (den < t) den = t;
  if (den < 1.0e-37) {
    *tr = 0.0;
    *ti = 0.0;
    return;
  }
  *tr = fabs((f1r - f2r) / den);
  *ti = fabs((f1i - f2i) / den);
}

// exp(jkr)/(kr) integrand, nec_context.cpp:3553-3578
__device__ __forceinline__ void gf(double zk, double zpk, double rkb2, bool ija, double* co,
                                   double* si) {
  double zdk = zk - zpk;
  double rk = sqrt(rkb2 + zdk * zdk);
  double s, c;
  sincos(rk, &s, &c);
  *si = s / rk;
  if (ija) {
    *co = c / rk;
    return;
  }
  if (rk >= .2) {
    *co = (c - 1.0) / rk;
    return;
  }
  double rks = rk * rk;
  *co = ((-1.38888889e-3 * rks + 4.16666667e-2) * rks - 0.5) * rk;
}

// Variable-interval Romberg integration of exp(jkr)/r, nec_context.cpp:4135-4300
__device__ void intx(double el1, double el2, double b, bool ij, double zpk, double rkb2,
                     double* sgr, double* sgi, int* status) {
  const int nx = 1, nma = 65536, nts = 4;
  const double rx = 1.0e-4;
  double z = el1, ze = el2;
  if (!ij) ze = 0.;
  const double s = ze - z;
  const double fnm = nma;
  const double ep = s / (10. * fnm);
  const double zend = ze - ep;
  double sr = 0., si = 0.;
  int ns = nx, nt = 0;
  double g1r, g1i, g2r = 0, g2i = 0, g3r = 0, g3i = 0, g4r, g4i, g5r = 0, g5i = 0;
  double dz = 0., dzot = 0.;
  gf(z, zpk, rkb2, ij, &g1r, &g1i);
  bool flag = true;
  // bound: every accepted step advances z by at least s/nma and every
  // rejected one halves dz (at most log2(nma) times per position)
  for (int guard = 0; guard < 8 * nma; guard++) {
    if (flag) {
      double fns = ns;
      dz = s / fns;
      double zp = z + dz;
      if (zp > ze) {
        dz = ze - z;
        if (fabs(dz) <= ep) goto done;
      }
      dzot = dz * .5;
      zp = z + dzot;
      gf(zp, zpk, rkb2, ij, &g3r, &g3i);
      zp = z + dz;
      gf(zp, zpk, rkb2, ij, &g5r, &g5i);
    }
    {
      double t00r = (g1r + g5r) * dzot;
      double t00i = (g1i + g5i) * dzot;
      double t01r = (t00r + dz * g3r) * 0.5;
      double t01i = (t00i + dz * g3i) * 0.5;
      double t10r = (4.0 * t01r - t00r) / 3.0;
      double t10i = (4.0 * t01i - t00i) / 3.0;
      double te1r, te1i;
      conv_test(t01r, t10r, &te1r, t01i, t10i, &te1i);
      if (te1i <= rx && te1r <= rx) {
        sr = sr + t10r;
        si = si + t10i;
        nt += 2;
        z += dz;
        if (z >= zend) goto done;
        g1r = g5r;
        g1i = g5i;
        if (nt >= nts && ns > nx) {
          ns = ns / 2;
          nt = 1;
        }
        flag = true;
        continue;
      }
      double zp = z + dz * 0.25;
      gf(zp, zpk, rkb2, ij, &g2r, &g2i);
      zp = z + dz * 0.75;
      gf(zp, zpk, rkb2, ij, &g4r, &g4i);
      double t02r = (t01r + dzot * (g2r + g4r)) * 0.5;
      double t02i = (t01i + dzot * (g2i + g4i)) * 0.5;
      double t11r = (4.0 * t02r - t01r) / 3.0;
      double t11i = (4.0 * t02i - t01i) / 3.0;
      double t20r = (16.0 * t11r - t10r) / 15.0;
      double t20i = (16.0 * t11i - t10i) / 15.0;
      double te2r, te2i;
      conv_test(t11r, t20r, &te2r, t11i, t20i, &te2i);
      if (te2i > rx || te2r > rx) {
        nt = 0;
        if (ns >= nma) {
          *status |= kStatRombergCap;
        } else {
          ns = ns * 2;
          double fns = ns;
          dz = s / fns;
          dzot = dz * 0.5;
          g5r = g3r;
          g5i = g3i;
          g3r = g2r;
          g3i = g2i;
          flag = false;
          continue;
        }
      }
      sr = sr + t20r;
      si = si + t20i;
      nt++;
      z += dz;
      if (z >= zend) goto done;
      g1r = g5r;
      g1i = g5i;
      if (nt >= nts && ns > nx) {
        ns = ns / 2;
        nt = 1;
      }
      flag = true;
    }
  }
  *status |= kStatIterCap;
done:
  if (!ij) {
    sr = 2. * (sr + log((sqrt(b * b + s * s) + s) / b));
    si = 2. * si;
  }
  *sgr = sr;
  *sgi = si;
}

// segment-end terms, nec_context.cpp:3605-3620
__device__ __forceinline__ void gx(double zz, double rh, double xk, cplx* gz, cplx* gzp) {
  double r2 = zz * zz + rh * rh;
  double r = sqrt(r2);
  double rkz = xk * r;
  double s, c;
  sincos(rkz, &s, &c);
  cplx temp = mk(c, -s) / r;
  *gz = temp;
  *gzp = -mk(1.0, rkz) * temp / r2;
}

// extended-kernel segment-end terms, nec_context.cpp:3623-3676
__device__ void gxx(double zz, double rh, double a, double a2, double xk, int ira, cplx* g1,
                    cplx* g1p, cplx* g2, cplx* g2p, cplx* g3, cplx* gzp) {
  double r2 = zz * zz + rh * rh;
  double r = sqrt(r2);
  double r4 = r2 * r2;
  double rk = xk * r;
  double rk2 = rk * rk;
  double rh2 = rh * rh;
  double t1 = .25 * a2 * rh2 / r4;
  double t2 = .5 * a2 / r2;
  cplx c1 = mk(1.0, rk);
  cplx c2 = 3. * c1 - rk2;
  cplx c3 = mk(6.0, rk) * rk2 - 15. * c1;
  double s, c;
  sincos(rk, &s, &c);
  cplx gz = mk(c, -s) / r;
  *g2 = gz * (1. + t1 * c2);
  *g1 = *g2 - t2 * c1 * gz;
  gz = gz / r2;
  *g2p = gz * (t1 * c3 - c1);
  *gzp = t2 * c2 * gz;
  *g3 = *g2p + *gzp;
  *g1p = *g3 * zz;
  if (ira != 1) {
    *g3 = (*g3 + *gzp) * rh;
    *gzp = -zz * c1 * gz;
    if (rh <= 1.0e-10) {
      *g2 = mk(0., 0.);
      *g2p = mk(0., 0.);
      return;
    }
    *g2 = *g2 / rh;
    *g2p = *g2p * zz / rh;
    return;
  }
  t2 = .5 * a;
  *g2 = -t2 * c1 * gz;
  *g2p = t2 * gz * c2 / r2;
  *g3 = rh2 * *g2p - a * gz * c1;
  *g2p = *g2p * zz;
  *gzp = -zz * c1 * gz;
}

// thin-wire (reduced) kernel, nec_context.cpp:3051-3104
__device__ void eksc(double s, double z, double rh, double xk, bool ij, cplx* ezs, cplx* ers,
                     cplx* ezc, cplx* erc, cplx* ezk, cplx* erk, int* status) {
  const cplx C1 = mk(0.0, kC1);
  double zpk = xk * z;
  double rhk = xk * rh;
  double rkb2 = rhk * rhk;
  double sh = .5 * s;
  double shk = xk * sh;
  double ss, cs;
  sincos(shk, &ss, &cs);
  double z2a = sh - z;
  double z1a = -(sh + z);
  cplx gz1, gz2, gp1, gp2;
  gx(z1a, rh, xk, &gz1, &gp1);
  gx(z2a, rh, xk, &gz2, &gp2);
  cplx gzp1 = gp1 * z1a;
  cplx gzp2 = gp2 * z2a;
  *ezs = C1 * ((gz2 - gz1) * cs * xk - (gzp2 + gzp1) * ss);
  *ezc = -C1 * ((gz2 + gz1) * ss * xk + (gzp2 - gzp1) * cs);
  *erk = C1 * (gp2 - gp1) * rh;
  double cint, sint;
  intx(-shk, shk, rhk, ij, zpk, rkb2, &cint, &sint, status);
  *ezk = -C1 * (gzp2 - gzp1 + xk * xk * mk(cint, -sint));
  if (rh >= 1.0e-10) {
    gzp1 = gzp1 * z1a;
    gzp2 = gzp2 * z2a;
    *ers = -C1 * ((gzp2 + gzp1 + gz2 + gz1) * ss - (z2a * gz2 - z1a * gz1) * cs * xk) / rh;
    *erc = -C1 * ((gzp2 - gzp1 + gz2 - gz1) * cs + (z2a * gz2 + z1a * gz1) * ss * xk) / rh;
    return;
  }
  *ers = mk(0., 0.);
  *erc = mk(0., 0.);
}

// extended thin-wire kernel, nec_context.cpp:3108-3188
__device__ void ekscx(double bx, double s, double z, double rhx, double xk, bool ij, int inx1,
                      int inx2, cplx* ezs, cplx* ers, cplx* ezc, cplx* erc, cplx* ezk,
                      cplx* erk, int* status) {
  const cplx C1 = mk(0.0, kC1);
  double b, rh;
  int ira;
  if (rhx >= bx) {
    rh = rhx;
    b = bx;
    ira = 0;
  } else {
    rh = bx;
    b = rhx;
    ira = 1;
  }
  double sh = .5 * s;
  double zpk = xk * z;
  double rhk = xk * rh;
  double rkb2 = rhk * rhk;
  double shk = xk * sh;
  double ss, cs;
  sincos(shk, &ss, &cs);
  double z2a = sh - z;
  double z1a = -(sh + z);
  double a2 = b * b;
  cplx gz1, gz2, gzp1, gzp2, gr1, gr2, grp1, grp2, grk1, grk2, gzz1, gzz2;
  if (inx1 != 2) {
    gxx(z1a, rh, b, a2, xk, ira, &gz1, &gzp1, &gr1, &grp1, &grk1, &gzz1);
  } else {
    gx(z1a, rhx, xk, &gz1, &grk1);
    gzp1 = grk1 * z1a;
    gr1 = gz1 / rhx;
    grp1 = gzp1 / rhx;
    grk1 = grk1 * rhx;
    gzz1 = mk(0., 0.);
  }
  if (inx2 != 2) {
    gxx(z2a, rh, b, a2, xk, ira, &gz2, &gzp2, &gr2, &grp2, &grk2, &gzz2);
  } else {
    gx(z2a, rhx, xk, &gz2, &grk2);
    gzp2 = grk2 * z2a;
    gr2 = gz2 / rhx;
    grp2 = gzp2 / rhx;
    grk2 = grk2 * rhx;
    gzz2 = mk(0., 0.);
  }
  *ezs = C1 * ((gz2 - gz1) * cs * xk - (gzp2 + gzp1) * ss);
  *ezc = -C1 * ((gz2 + gz1) * ss * xk + (gzp2 - gzp1) * cs);
  *ers = -C1 * ((z2a * grp2 + z1a * grp1 + gr2 + gr1) * ss - (z2a * gr2 - z1a * gr1) * cs * xk);
  *erc = -C1 * ((z2a * grp2 - z1a * grp1 + gr2 - gr1) * cs + (z2a * gr2 + z1a * gr1) * ss * xk);
  *erk = C1 * (grk2 - grk1);
  double cint, sint;
  intx(-shk, shk, rhk, ij, zpk, rkb2, &cint, &sint, status);
  double bk = b * xk;
  double bk2 = bk * bk * .25;
  *ezk = -C1 * (gzp2 - gzp1 + xk * xk * (1. - bk2) * mk(cint, -sint) - bk2 * (gzz2 - gzz1));
}

// Fields of one source segment (direct or image) at a displacement:
// nec_context.cpp:2777-2843.  e[0..8] = (xk,yk,zk, xs,ys,zs, xc,yc,zc).
// Returns r, the distance used for the far-pair decision.
template <bool EXK>
__device__ double efld_compute(const SrcSeg& J, double xij, double yij, double ai,
                               double salpr, double zij, bool ijx, const FieldParams& P,
                               cplx e[9], int* status) {
  const double cabj = J.cab, sabj = J.sab;
  cplx tezs, ters, tezc, terc, tezk, terk;
  double zp = xij * cabj + yij * sabj + zij * salpr;
  double rhox = xij - cabj * zp;
  double rhoy = yij - sabj * zp;
  double rhoz = zij - salpr * zp;
  double rh = sqrt(rhox * rhox + rhoy * rhoy + rhoz * rhoz + ai * ai);
  double r = sqrt(zp * zp + rh * rh);
  const bool far = r >= P.rkh;
  // the FP64 divide is the costliest operation of a far pair: 1 / rh for
  // the three components and, for a far pair, 1 / r come from one
  // reciprocal of rh r
  double rinv = 0.0;
  if (rh <= 1.e-10) {
    rhox = 0.0;
    rhoy = 0.0;
    rhoz = 0.0;
    if (far) rinv = 1.0 / r;
  } else {
    double rhinv;
    if (far) {
      const double q = 1.0 / (rh * r);
      rhinv = r * q;
      rinv = rh * q;
    } else {
      rhinv = 1.0 / rh;
    }
    rhox *= rhinv;
    rhoy *= rhinv;
    rhoz *= rhinv;
  }
  if (far) {
    // lumped current element, 2798-2819, with the divisions by r, rmag and
    // py = 2 pi r^2 folded into that reciprocal
    double rmag = kTwoPiD * r;
    double cth = zp * rinv;
    double px = rh * rinv;
    // exp(-j rmag) as sincospi of r * 2 pi / pi_exact (exact reduction)
    constexpr double kTwoPiOverPi = kTwoPiD / 3.141592653589793;
    double sn, cs;
    sincospi(kTwoPiOverPi * r, &sn, &cs);
    cplx e0 = mk(cs, -sn);
    const double rminv = rinv * (1.0 / kTwoPiD);
    const double pyinv = rminv * rinv;  // 1 / py
    cplx e1 = (P.eta * cth * pyinv) * e0 * mk(1.0, -rminv);
    cplx e2 = (0.5 * P.eta * px * pyinv) * e0 * mk(1.0, rmag - rminv);
    tezk = e1 * cth - e2 * px;
    terk = e1 * px + e2 * cth;
    const double sfac = J.sfac;
    tezc = tezk * sfac;
    terc = terk * sfac;
    tezk = tezk * J.s;
    terk = terk * J.s;
    e[3] = mk(0., 0.);
    e[4] = mk(0., 0.);
    e[5] = mk(0., 0.);
  } else {
    if (!EXK)
      eksc(J.s, zp, rh, kTwoPiD, ijx, &tezs, &ters, &tezc, &terc, &tezk, &terk, status);
    else
      ekscx(J.b, J.s, zp, rh, kTwoPiD, ijx, J.ind1, J.ind2, &tezs, &ters, &tezc, &terc, &tezk,
            &terk, status);
    e[3] = tezs * cabj + ters * rhox;
    e[4] = tezs * sabj + ters * rhoy;
    e[5] = tezs * salpr + ters * rhoz;
  }
  e[0] = tezk * cabj + terk * rhox;
  e[1] = tezk * sabj + terk * rhoy;
  e[2] = tezk * salpr + terk * rhoz;
  e[6] = tezc * cabj + terc * rhox;
  e[7] = tezc * sabj + terc * rhoy;
  e[8] = tezc * salpr + terc * rhoz;
  return r;
}

// Sommerfeld attenuation function, c_ggrid.cpp:291-350
__device__ cplx fbar(cplx p) {
  const double sqrt_pi = sqrt(kPiD);
  const double tosp = 2.0 / sqrt_pi;
  cplx z = mk(0.0, 1.0) * csqrt_(p);
  if (cabs_(z) <= 3.) {
    cplx zs = z * z;
    cplx sum = z, pw = z;
    for (int i = 1; i <= 100; i++) {
      pw = -pw * zs / static_cast<double>(i);
      cplx term = pw / (2. * i + 1.);
      sum = sum + term;
      if (cnorm(term) / cnorm(sum) < 1.E-12) break;
    }
    return 1. - (1. - sum * tosp) * z * cexp_(zs) * sqrt_pi;
  }
  bool minus = false;
  if (z.re < 0.) {
    minus = true;
    z = -z;
  }
  cplx zs = .5 / (z * z);
  cplx sum = mk(0., 0.), term = mk(1., 0.);
  for (int i = 1; i <= 6; i++) {
    term = -term * (2. * i - 1.) * zs;
    sum += term;
  }
  if (minus) sum -= 2.0 * sqrt_pi * z * cexp_(z * z);
  return -sum;
}

// Norton ground wave of a current element, c_ggrid.cpp:351-432, with the
// source term of sflds (isnor=2): r1=1, zmh=1, xx1=0.
__device__ void gwave(double r2, double zph, cplx xx2, cplx u, cplx u2, double eta, cplx* erv,
                      cplx* ezv, cplx* erh, cplx* ezh, cplx* eph) {
  const cplx C4 = mk(0.0, eta / 2.0);
  const double r1 = 1.0, zmh = 1.0;
  const cplx xx1 = mk(0., 0.);
  double sppp = zmh / r1;
  double sppp2 = sppp * sppp;
  double cppp2 = 1. - sppp2;
  if (cppp2 < 1.0e-20) cppp2 = 1.0e-20;
  double cppp = sqrt(cppp2);
  double spp = zph / r2;
  double spp2 = spp * spp;
  double cpp2 = 1. - spp2;
  if (cpp2 < 1.0e-20) cpp2 = 1.0e-20;
  double cpp = sqrt(cpp2);
  const cplx two_pi_j = mk(0.0, kTwoPiD);
  cplx rk1 = -two_pi_j * r1;
  cplx rk2 = -two_pi_j * r2;
  cplx t1 = 1. - u2 * cpp2;
  cplx t2 = csqrt_(t1);
  cplx t3 = (1. - 1. / rk1) / rk1;
  cplx t4 = (1. - 1. / rk2) / rk2;
  cplx p1 = rk2 * u2 * t1 / (2. * cpp2);
  cplx rv = (spp - u * t2) / (spp + u * t2);
  cplx omr = 1. - rv;
  cplx w = 1. / omr;
  w = mk(4.0, 0.0) * p1 * w * w;
  cplx f = fbar(w);
  cplx q1 = rk2 * t1 / (2. * u2 * cpp2);
  cplx rh = (t2 - u * spp) / (t2 + u * spp);
  cplx v = 1. / (1. + rh);
  v = mk(4.0, 0.0) * q1 * v * v;
  cplx g = fbar(v);
  cplx xr1 = xx1 / r1;
  cplx xr2 = xx2 / r2;
  cplx x1 = cppp2 * xr1;
  cplx x2 = rv * cpp2 * xr2;
  cplx x3 = omr * cpp2 * f * xr2;
  cplx x4 = u * t2 * spp * 2. * xr2 / rk2;
  cplx x5 = xr1 * t3 * (1. - 3. * sppp2);
  cplx x6 = xr2 * t4 * (1. - 3. * spp2);
  const cplx nC4 = -C4;
  *ezv = (x1 + x2 + x3 - x4 - x5 - x6) * nC4;
  x1 = sppp * cppp * xr1;
  x2 = rv * spp * cpp * xr2;
  x3 = cpp * omr * u * t2 * f * xr2;
  x4 = spp * cpp * omr * xr2 / rk2;
  x5 = 3. * sppp * cppp * t3 * xr1;
  x6 = cpp * u * t2 * omr * xr2 / rk2 * .5;
  cplx x7 = 3. * spp * cpp * t4 * xr2;
  *erv = -(x1 + x2 - x3 + x4 - x5 + x6 - x7) * nC4;
  *ezh = -(x1 - x2 + x3 - x4 - x5 - x6 + x7) * nC4;
  x1 = sppp2 * xr1;
  x2 = rv * spp2 * xr2;
  x4 = u2 * t1 * omr * f * xr2;
  x5 = t3 * (1. - 3. * cppp2) * xr1;
  x6 = t4 * (1. - 3. * cpp2) * (1. - u2 * (1. + rv) - u2 * omr * f) * xr2;
  x7 = u2 * cpp2 * omr * (1. - 1. / rk2) * (f * (u2 * t1 - spp2 - 1. / rk2) + 1. / rk2) * xr2;
  *erh = (x1 - x2 - x4 - x5 + x6 + x7) * nC4;
  x1 = xr1;
  x2 = rh * xr2;
  x3 = (rh + 1.) * g * xr2;
  x4 = t3 * xr1;
  x5 = t4 * (1. - u2 * (1. + rv) - u2 * omr * f) * xr2;
  x6 = .5 * u2 * omr * (f * (u2 * t1 - spp2 - 1. / rk2) + 1. / rk2) * xr2 / rk2;
  *eph = -(x1 - x2 + x3 - x4 + x5 + x6) * nC4;
}

enum { kGroundNone = 0, kGroundPerfect = 1, kGroundReflection = 2, kGroundSommerfeld = 3 };

// Fields of source J at observation point i, direct plus (for a ground)
// image: efld (2845-2956) up to the Sommerfeld/Norton part.
template <int GROUND, bool EXK>
__device__ __forceinline__ void pair_fields9(const SrcSeg& J, double xi, double yi, double zi, double ai,
                                             bool ij, const FieldParams& P, cplx ex[9], int* status) {
  cplx e[9];
  const double xij = xi - J.x;
  const double yij = yi - J.y;
  efld_compute<EXK>(J, xij, yij, ai, J.salp, zi - J.z, ij, P, ex, status);
  if (GROUND != kGroundNone) {
    const double zij = zi + J.z;
    double r = efld_compute<EXK>(J, xij, yij, ai, -J.salp, zij, true, P, e, status);
    if (GROUND == kGroundReflection) {
      // reflection-coefficient approximation, 2893-2944
      cplx zratx = P.zrati;
      double xymag = sqrt(xij * xij + yij * yij);
      double px, py, cth;
      cplx zrsin;
      if (xymag <= 1.0e-6) {
        px = 0.;
        py = 0.;
        cth = 1.;
        zrsin = mk(1., 0.);
      } else {
        px = -yij / xymag;
        py = xij / xymag;
        cth = zij / r;
        zrsin = csqrt_(1.0 - zratx * zratx * (1.0 - cth * cth));
      }
      cplx refs = (cth - zratx * zrsin) / (cth + zratx * zrsin);
      cplx refps = -(zratx * cth - zrsin) / (zratx * cth + zrsin);
      refps = refps - refs;
#pragma unroll
      for (int k = 0; k < 9; k += 3) {
        cplx epy = px * e[k] + py * e[k + 1];
        cplx epx = px * epy;
        epy = py * epy;
        e[k] = refs * e[k] + refps * epx;
        e[k + 1] = refs * e[k + 1] + refps * epy;
        e[k + 2] = refs * e[k + 2];
      }
    }
#pragma unroll
    for (int k = 0; k < 9; k++) ex[k] -= e[k] * P.frati;
  }
}

// Horizontal direction of the source and the observation point displaced
// by the observer's radius for the thin-wire approximation (2958-3000).
struct SommGeom {
  double xsn, ysn, sn, xo, yo, zo, rhox, rhoy, rhoz, rh;
};

__device__ __forceinline__ SommGeom somm_geometry(const SrcSeg& J, double xi, double yi, double zi, double ai) {
  SommGeom g;
  const double cabj = J.cab, sabj = J.sab, salpj = J.salp;
  g.sn = sqrt(cabj * cabj + sabj * sabj);
  if (g.sn >= 1.0e-5) {
    g.xsn = cabj / g.sn;
    g.ysn = sabj / g.sn;
  } else {
    g.sn = 0.0;
    g.xsn = 1.0;
    g.ysn = 0.0;
  }
  const double xij = xi - J.x, yij = yi - J.y, zij = zi + J.z;
  const double salpr = -salpj;
  g.rhox = sabj * zij - salpr * yij;
  g.rhoy = salpr * xij - cabj * zij;
  g.rhoz = cabj * yij - sabj * xij;
  g.rh = sqrt(g.rhox * g.rhox + g.rhoy * g.rhoy + g.rhoz * g.rhoz);
  if (g.rh <= 1.e-10) {
    g.xo = xi - ai * g.ysn;
    g.yo = yi + ai * g.xsn;
    g.zo = zi;
  } else {
    // the reference takes sqrt of the already-rooted norm here
    double rr = ai / sqrt(g.rh);
    if (g.rhoz < 0.0) rr = -rr;
    g.xo = xi + rr * g.rhox;
    g.yo = yi + rr * g.rhoy;
    g.zo = zi + rr * g.rhoz;
  }
  return g;
}

// Norton ground field of a source lumped at its centre (sflds, isnor = 2,
// 6024-6098) with the thin-wire correction of efld (3009-3032).
__device__ void norton_field(const SrcSeg& J, const SommGeom& g, double xij, double yij, double zij, double r,
                             double ai, const FieldParams& P, cplx e[9]) {
  const double cabj = J.cab, sabj = J.sab, salpj = J.salp, salpr = -salpj;
  const double xsn = g.xsn, ysn = g.ysn, sn = g.sn;
  double xt = J.x + 0. * cabj, yt = J.y + 0. * sabj, zt = J.z + 0. * salpj;
  double rhx = g.xo - xt, rhy = g.yo - yt;
  double rhs = rhx * rhx + rhy * rhy;
  double rho = sqrt(rhs);
  double phx, phy;
  if (rho <= 0.0) {
    rhx = 1.0;
    rhy = 0.0;
    phx = 0.0;
    phy = 1.0;
  } else {
    rhx = rhx / rho;
    rhy = rhy / rho;
    phx = -rhy;
    phy = rhx;
  }
  double cph = rhx * xsn + rhy * ysn;
  double sph = rhy * xsn - rhx * ysn;
  if (fabs(cph) < 1.0e-10) cph = 0.0;
  if (fabs(sph) < 1.0e-10) sph = 0.0;
  double zph = g.zo + zt;
  double zphs = zph * zph;
  double r2s = rhs + zphs;
  double r2 = sqrt(r2s);
  double rk = r2 * kTwoPiD;
  double s_, c_;
  sincos(rk, &s_, &c_);
  cplx xx2 = mk(c_, -s_);
  cplx erv, ezv, erh, ezh, eph;
  gwave(r2, zph, xx2, P.u, P.u2, P.eta, &erv, &ezv, &erh, &ezh, &eph);
  const cplx C1 = mk(0.0, kC1);
  cplx et = -C1 * P.frati * xx2 / (r2s * r2);
  cplx er = 2. * et * mk(1.0, rk);
  et = et * mk(1.0 - rk * rk, rk);
  cplx hrv = (er + et) * rho * zph / r2s;
  cplx hzv = (zphs * er - rhs * et) / r2s;
  cplx hrh = (rhs * er - zphs * et) / r2s;
  erv = erv - hrv;
  ezv = ezv - hzv;
  erh = erh + hrh;
  ezh = ezh + hrv;
  eph = eph + et;
  erv = erv * salpj;
  ezv = ezv * salpj;
  erh = erh * sn * cph;
  ezh = ezh * sn * cph;
  eph = eph * sn * sph;
  erh = erv + erh;
  e[0] = (erh * rhx + eph * phx) * J.s;
  e[1] = (erh * rhy + eph * phy) * J.s;
  e[2] = (ezv + ezh) * J.s;
  e[3] = mk(0., 0.);
  e[4] = mk(0., 0.);
  e[5] = mk(0., 0.);
  double sfac = kPiD * J.s;
  sfac = sin(sfac) / sfac;
  e[6] = e[0] * sfac;
  e[7] = e[1] * sfac;
  e[8] = e[2] * sfac;
  // thin-wire correction, 3009-3032
  double zp = xij * cabj + yij * sabj + zij * salpr;
  double rh = r - zp * zp;
  double dmin = (rh <= 1.e-10) ? 0.0 : sqrt(rh / (rh + ai * ai));
  if (dmin <= .95) {
    double pxx = 1. - dmin;
#pragma unroll
    for (int k = 0; k < 9; k += 3) {
      cplx t = (e[k] * cabj + e[k + 1] * sabj + e[k + 2] * salpr) * pxx;
      e[k] = dmin * e[k] + t * cabj;
      e[k + 1] = dmin * e[k + 1] + t * sabj;
      e[k + 2] = dmin * e[k + 2] + t * salpr;
    }
  }
}

// Tangential projection of cmww, 2617-2619
__device__ __forceinline__ void project_fields(const cplx ex[9], double cabi, double sabi, double salpi, cplx* etk,
                                               cplx* ets, cplx* etc) {
  *etk = ex[0] * cabi + ex[1] * sabi + ex[2] * salpi;
  *ets = ex[3] * cabi + ex[4] * sabi + ex[5] * salpi;
  *etc = ex[6] * cabi + ex[7] * sabi + ex[8] * salpi;
}

// Projected fields (etk, ets, etc) of source J on observation segment i:
// efld (2845-3045) followed by the tangential projection of cmww (2617-2619).
// For Sommerfeld ground, a pair within the table limit of its image is read
// from P.near_g at pair_index (obs * n + src) when those fields exist, and
// is reported (kStatSommerfeldTab) otherwise.
template <int GROUND, bool EXK>
__device__ void pair_field(const SrcSeg& J, double xi, double yi, double zi, double ai,
                           double cabi, double sabi, double salpi, bool ij,
                           const FieldParams& P, cplx* etk, cplx* ets, cplx* etc,
                           int* status, int64_t pair_index = -1) {
  const double xij = xi - J.x, yij = yi - J.y;
  double r_img = 0.0;
  if (GROUND == kGroundSommerfeld) {
    r_img = image_r2(xij, yij, zi + J.z);
    if (r_img <= .95 && P.near_g != nullptr && pair_index >= 0) {
      const cplx* g = P.near_g + pair_index * 3;
      *etk = g[0];
      *ets = g[1];
      *etc = g[2];
      return;
    }
  }
  cplx ex[9];
  pair_fields9<GROUND, EXK>(J, xi, yi, zi, ai, ij, P, ex, status);
  if (GROUND == kGroundSommerfeld) {
    cplx e[9];
    if (r_img <= .95) {
      *status |= kStatSommerfeldTab;
      for (int k = 0; k < 9; k++) e[k] = mk(0., 0.);
    } else {
      const SommGeom g = somm_geometry(J, xi, yi, zi, ai);
      norton_field(J, g, xij, yij, zi + J.z, r_img, ai, P, e);
    }
#pragma unroll
    for (int k = 0; k < 9; k++) ex[k] = ex[k] + e[k];
  }
  project_fields(ex, cabi, sabi, salpi, etk, ets, etc);
}

}  // namespace necb
