// Sommerfeld ground on the device: the interpolation tables of the
// reflected field and the near-ground field of a source segment read from
// them.
//
// Device restatement of NEC2++
//   src/c_evlcom.cpp: bessel 640-733, hankel 738-840, saoa 382-488,
//     rom1 218-379, gshank 47-214, evlua 491-637;
//   src/c_ggrid.cpp: sommerfeld 164-288, interpolate 38-162;
//   src/nec_context.cpp: rom2 5589-5834, sflds (table branch) 6024-6066,
//     6108-6137.
// The tables are three grids in (R, theta) of the image distance and
// elevation: 11 x 10 points from R = 0 in steps of 0.02 wavelength, 17 x 5
// and 9 x 8 points from R = 0.2 (theta below / above 20 degrees); four
// functions per point (erv, ezv, erh, eph), scaled by the image spherical
// wave.  One thread evaluates the Sommerfeld integrals of one grid point.
//
// The interpolation keeps the reference's cache: the last 4 x 4 patch and
// its cell, reused for a point that lies below the start of the patch's
// grid.  Results therefore depend on the order of the points, and the
// near-ground fill reproduces that order (see near_ground_kernel).
#pragma once
#include "cplx.cuh"
#include "field.cuh"
#include "fill.cuh"

namespace necb {

constexpr int kSommPoints = 1068;  // 440 + 340 + 288 complex values
// grid points whose integrals are evaluated (R = 0 of the first grid has a
// closed form)
constexpr int kSommEvalPoints = 100 + 85 + 72;

__host__ __device__ __forceinline__ cplx conj_(cplx a) { return {a.re, -a.im}; }
__device__ __forceinline__ cplx clog_(cplx z) { return {log(hypot(z.re, z.im)), atan2(z.im, z.re)}; }
__device__ __forceinline__ cplx mul_i(cplx a) { return cplx{0.0, 1.0} * a; }

// grid geometry, c_ggrid.cpp:27-34
__host__ __device__ __forceinline__ int somm_nx(int g) { return g == 0 ? 11 : (g == 1 ? 17 : 9); }
__host__ __device__ __forceinline__ int somm_ny(int g) { return g == 0 ? 10 : (g == 1 ? 5 : 8); }
__host__ __device__ __forceinline__ double somm_dx(int g) { return g == 0 ? .02 : (g == 1 ? .05 : .1); }
__host__ __device__ __forceinline__ double somm_dy(int g) {
  return g == 1 ? .0872664626 : .1745329252;
}
__host__ __device__ __forceinline__ double somm_xs(int g) { return g == 0 ? 0. : .2; }
__host__ __device__ __forceinline__ double somm_ys(int g) { return g == 2 ? .3490658504 : 0.; }
__host__ __device__ __forceinline__ int somm_off(int g) { return g == 0 ? 0 : (g == 1 ? 440 : 780); }

// Series-length tables of bessel / hankel (the reference builds them on
// first use; here each thread block builds them in shared memory).
struct BesselTables {
  int bes_m[101], han_m[101];
  double bes_a1[25], bes_a2[25], han_a1[25], han_a2[25], han_a3[25], han_a4[25];
};

__device__ void build_bessel_tables(BesselTables& t) {
  for (int k = 1; k <= 25; k++) {
    t.bes_a1[k - 1] = -0.25 / (k * k);
    t.bes_a2[k - 1] = 1.0 / (k + 1.0);
  }
  for (int i = 1; i <= 101; i++) {
    double tst = 1.0;
    int init = 0;
    for (int k = 0; k < 24; k++) {
      init = k;
      tst *= -i * t.bes_a1[k];
      if (tst < 1.0e-6) break;
    }
    t.bes_m[i - 1] = init + 1;
  }
  double psi = -.5772156649;
  for (int k = 1; k <= 25; k++) {
    int i = k - 1;
    t.han_a1[i] = -.25 / (k * k);
    t.han_a2[i] = 1.0 / (k + 1.0);
    psi += 1.0 / k;
    t.han_a3[i] = psi + psi;
    t.han_a4[i] = (psi + psi + 1.0 / (k + 1.0)) / (k + 1.0);
  }
  for (int i = 1; i <= 101; i++) {
    double tt = 1.0;
    int init = 0;
    for (int k = 0; k < 24; k++) {
      init = k;
      tt *= -i * t.han_a1[k];
      if ((tt * t.han_a3[k]) < 1.e-6) break;
    }
    t.han_m[i - 1] = init + 1;
  }
}

// asymptotic-series constants, c_evlcom.cpp:627-637
constexpr double kP10 = .0703125, kP20 = .1121520996, kQ10 = .125, kQ20 = .0732421875;
constexpr double kP11 = .1171875, kP21 = .1441955566, kQ11 = .375, kQ21 = .1025390625;
constexpr double kPOF = .7853981635, kC3 = .7978845608;

// J0 and its derivative, complex argument
__device__ void bessel_j0(const BesselTables& T, cplx z, cplx* j0, cplx* j0p) {
  double zms = cnorm(z);
  if (zms <= 1.e-12) {
    *j0 = mk(1.0, 0.0);
    *j0p = -0.5 * z;
    return;
  }
  cplx j0x = mk(0, 0), j0px = mk(0, 0);
  int ib = 0;
  if (zms <= 37.21) {
    if (zms > 36.0) ib = 1;
    int miz = T.bes_m[(int)floor(zms)];
    cplx a = mk(1.0, 0.0), ap = mk(1.0, 0.0), zk = mk(1.0, 0.0), zi = z * z;
    for (int k = 0; k < miz; k++) {
      zk = zk * (T.bes_a1[k] * zi);
      a += zk;
      ap += T.bes_a2[k] * zk;
    }
    ap = ap * (-0.5 * z);
    *j0 = a;
    *j0p = ap;
    if (ib == 0) return;
    j0x = a;
    j0px = ap;
  }
  cplx zi = 1.0 / z;
  cplx zi2 = zi * zi;
  cplx p0z = 1.0 + (kP20 * zi2 - kP10) * zi2;
  cplx p1z = 1.0 + (kP11 - kP21 * zi2) * zi2;
  cplx q0z = (kQ20 * zi2 - kQ10) * zi;
  cplx q1z = (kQ11 - kQ21 * zi2) * zi;
  cplx zk = cexp_(mul_i(z - kPOF));
  zi2 = 1.0 / zk;
  cplx cz = 0.5 * (zk + zi2);
  cplx sz = mk(0.0, 0.5) * (zi2 - zk);
  zk = kC3 * csqrt_(zi);
  *j0 = zk * (p0z * cz - q0z * sz);
  *j0p = -zk * (p1z * sz + q1z * cz);
  if (ib == 0) return;
  zms = cos((sqrt(zms) - 6.0) * (kPiD * 10.0));
  *j0 = 0.5 * (j0x * (1.0 + zms) + *j0 * (1.0 - zms));
  *j0p = 0.5 * (j0px * (1.0 + zms) + *j0p * (1.0 - zms));
}

// H0(1) and its derivative, complex argument (z != 0)
__device__ bool hankel_h0(const BesselTables& T, cplx z, cplx* h0, cplx* h0p) {
  double zms = cnorm(z);
  if (zms == 0.0) return false;
  cplx y0 = mk(0, 0), y0p = mk(0, 0);
  int ib = 0;
  if (zms <= 16.81) {
    if (zms > 16.) ib = 1;
    int miz = T.han_m[(int)zms];
    cplx j0 = mk(1.0, 0.0), j0p = mk(1.0, 0.0), zk = mk(1.0, 0.0), zi = z * z;
    for (int k = 0; k < miz; k++) {
      zk = zk * (T.han_a1[k] * zi);
      j0 += zk;
      j0p += T.han_a2[k] * zk;
      y0 += T.han_a3[k] * zk;
      y0p += T.han_a4[k] * zk;
    }
    j0p = j0p * (-.5 * z);
    cplx clogz = clog_(.5 * z);
    y0 = (2.0 * j0 * clogz - y0) / kPiD + .3674669052;
    y0p = (2.0 / z + 2.0 * j0p * clogz + 0.5 * y0p * z) / kPiD + -.02457850915 * z;
    *h0 = j0 + mul_i(y0);
    *h0p = j0p + mul_i(y0p);
    if (ib == 0) return true;
    y0 = *h0;
    y0p = *h0p;
  }
  cplx zi = 1. / z;
  cplx zi2 = zi * zi;
  cplx p0z = 1. + (kP20 * zi2 - kP10) * zi2;
  cplx p1z = 1. + (kP11 - kP21 * zi2) * zi2;
  cplx q0z = (kQ20 * zi2 - kQ10) * zi;
  cplx q1z = (kQ11 - kQ21 * zi2) * zi;
  cplx zk = cexp_(mul_i(z - kPOF)) * csqrt_(zi) * kC3;
  *h0 = zk * (p0z + mul_i(q0z));
  *h0p = mul_i(zk) * (p1z + mul_i(q1z));
  if (ib == 0) return true;
  zms = cos((sqrt(zms) - 4.) * 31.41592654);
  *h0 = .5 * (y0 * (1. + zms) + *h0 * (1. - zms));
  *h0p = .5 * (y0p * (1. + zms) + *h0p * (1. - zms));
  return true;
}

// State of the contour integration of one grid point (c_evlcom members).
struct Evl {
  double ck2, ck2sq, tkmag, tsmag, ck1r, zph, rho;
  cplx ct1, ct2, ct3, ck1, ck1sq, cksm;
  cplx a, b;  // contour segment
  bool bessel_form;
  int fail;
};

constexpr int kSommNM = 131072, kSommMaxH = 20;
constexpr double kSommCrit = 1.0E-4, kSommPTP = .6283185308;

// integrands of the six Sommerfeld integrals at contour parameter t
__device__ void saoa(const BesselTables& T, Evl& E, double t, cplx ans[6]) {
  cplx dxl = E.b - E.a;
  cplx xl = E.a + dxl * t;
  cplx b0 = mk(0, 0), b0p = mk(0, 0), cgam1, cgam2, com, dgam;
  if (E.bessel_form) {
    bessel_j0(T, xl * E.rho, &b0, &b0p);
    b0 = b0 * 2.;
    b0p = b0p * 2.;
    cgam1 = csqrt_(xl * xl - E.ck1sq);
    cgam2 = csqrt_(xl * xl - E.ck2sq);
    if (cgam1.re == 0.0) cgam1 = mk(0.0, -fabs(cgam1.im));
    if (cgam2.re == 0.) cgam2 = mk(0.0, -fabs(cgam2.im));
  } else {
    if (!hankel_h0(T, xl * E.rho, &b0, &b0p)) E.fail = 1;
    com = xl - E.ck1;
    cgam1 = csqrt_(xl + E.ck1) * csqrt_(com);
    if (com.re < 0. && com.im >= 0.) cgam1 = -cgam1;
    com = xl - E.ck2;
    cgam2 = csqrt_(xl + E.ck2) * csqrt_(com);
    if (com.re < 0. && com.im >= 0.) cgam2 = -cgam2;
  }
  bool direct = true;
  double sign = 1.0;
  if (cnorm(xl) >= E.tsmag) {
    direct = false;
    if (xl.im >= 0.0) {
      if (xl.re >= E.ck2) {
        if (xl.re <= E.ck1r) direct = true;
      } else {
        sign = -1.0;
      }
    }
  }
  if (direct) {
    dgam = cgam2 - cgam1;
  } else {
    dgam = 1.0 / (xl * xl);
    dgam = sign * ((E.ct3 * dgam + E.ct2) * dgam + E.ct1) / xl;
  }
  cplx den2 = E.cksm * dgam / (cgam2 * (E.ck1sq * cgam2 + E.ck2sq * cgam1));
  cplx den1 = 1. / (cgam1 + cgam2) - E.cksm / cgam2;
  com = dxl * xl * cexp_(-cgam2 * E.zph);
  ans[5] = com * b0 * den1 / E.ck1;
  com = com * den2;
  if (E.rho != 0.) {
    b0p = b0p / E.rho;
    ans[0] = -com * xl * (b0p + b0 * xl);
    ans[3] = com * xl * b0p;
  } else {
    ans[0] = -com * xl * xl * .5;
    ans[3] = ans[0];
  }
  ans[1] = com * cgam2 * cgam2 * b0;
  ans[2] = -ans[3] * cgam2 * E.rho;
  ans[4] = com * b0;
}

// variable-interval Romberg integration of the six integrands over [a, b]
__device__ void rom1(const BesselTables& T, Evl& E, cplx sum[6], int nx) {
  const double s = 1.0, ze = 1.0, ep = s / (1.0e4 * kSommNM), zend = ze - ep;
  double z = 0.0, dz = 0.0, dzot = 0.0, tr, ti;
  cplx g1[6], g2[6], g3[6], g4[6], g5[6], t01[6], t10[6], t20[6];
  for (int i = 0; i < 6; i++) sum[i] = mk(0, 0);
  int ns = nx, nt = 0;
  saoa(T, E, z, g1);
  bool jump = false;
  for (int guard = 0; guard < (1 << 20); guard++) {
    if (!jump) {
      dz = s / ns;
      if ((z + dz) > ze) {
        dz = ze - z;
        if (dz <= ep) return;
      }
      dzot = dz * .5;
      saoa(T, E, z + dzot, g3);
      saoa(T, E, z + dz, g5);
    }
    bool nogo = false;
    for (int i = 0; i < 6; i++) {
      cplx t00 = (g1[i] + g5[i]) * dzot;
      t01[i] = (t00 + dz * g3[i]) * .5;
      t10[i] = (4. * t01[i] - t00) / 3.;
      conv_test(t01[i].re, t10[i].re, &tr, t01[i].im, t10[i].im, &ti);
      if ((tr > kSommCrit) || (ti > kSommCrit)) nogo = true;
    }
    bool accept5 = false;
    if (!nogo) {
      for (int i = 0; i < 6; i++) sum[i] += t10[i];
      nt += 2;
    } else {
      saoa(T, E, z + dz * .25, g2);
      saoa(T, E, z + dz * .75, g4);
      nogo = false;
      for (int i = 0; i < 6; i++) {
        cplx t02 = (t01[i] + dzot * (g2[i] + g4[i])) * .5;
        cplx t11 = (4. * t02 - t01[i]) / 3.;
        t20[i] = (16. * t11 - t10[i]) / 15.;
        conv_test(t11.re, t20[i].re, &tr, t11.im, t20[i].im, &ti);
        if ((tr > kSommCrit) || (ti > kSommCrit)) nogo = true;
      }
      if (nogo) {
        nt = 0;
        if (ns < kSommNM) {
          ns *= 2;
          dz = s / ns;
          dzot = dz * .5;
          for (int i = 0; i < 6; i++) {
            g5[i] = g3[i];
            g3[i] = g2[i];
          }
          jump = true;
          continue;
        }
      }
      accept5 = true;
    }
    if (accept5) {
      for (int i = 0; i < 6; i++) sum[i] += t20[i];
      nt++;
    }
    z += dz;
    if (z > zend) return;
    for (int i = 0; i < 6; i++) g1[i] = g5[i];
    if ((nt >= 4) && (ns > nx)) {
      ns = ns / 2;
      nt = 1;
    }
    jump = false;
  }
  E.fail = 1;
}

// integration from `start` to infinity with Shanks' transformation; at the
// break point bk (when ibk != 0) the step changes from dela to delb
__device__ void gshank(const BesselTables& T, Evl& E, cplx start, cplx dela, cplx sum[6], const cplx seed[6],
                       int ibk, cplx bk, cplx delb) {
  cplx q1[6][kSommMaxH], q2[6][kSommMaxH], ans1[6], ans2[6];
  const double rbk = bk.re;
  cplx del = dela;
  int ibx = (ibk == 0) ? 1 : 0;
  for (int i = 0; i < 6; i++) ans2[i] = seed[i];
  E.b = start;
  int restarts = 0;
  for (int intx = 1; intx <= kSommMaxH; intx++) {
    const int inx = intx - 1;
    E.a = E.b;
    E.b = E.b + del;
    if ((ibx == 0) && (E.b.re >= rbk)) {
      ibx = 1;
      E.b = bk;
      del = delb;
      rom1(T, E, sum, 2);
      for (int i = 0; i < 6; i++) ans2[i] += sum[i];
      intx = 0;
      if (++restarts > 2) break;
      continue;
    }
    rom1(T, E, sum, 2);
    for (int i = 0; i < 6; i++) ans1[i] = ans2[i] + sum[i];
    E.a = E.b;
    E.b = E.b + del;
    if ((ibx == 0) && (E.b.re >= rbk)) {
      ibx = 2;
      E.b = bk;
      del = delb;
      rom1(T, E, sum, 2);
      for (int i = 0; i < 6; i++) ans2[i] = ans1[i] + sum[i];
      intx = 0;
      if (++restarts > 2) break;
      continue;
    }
    rom1(T, E, sum, 2);
    for (int i = 0; i < 6; i++) ans2[i] = ans1[i] + sum[i];
    double den = 0.;
    for (int i = 0; i < 6; i++) {
      cplx as1 = ans1[i], as2 = ans2[i];
      for (int j = 1; j < intx; j++) {
        const int jm = j - 1;
        cplx aa = q2[i][jm];
        cplx a1 = q1[i][jm] + as1 - 2. * aa;
        if ((a1.re != 0.) || (a1.im != 0.)) {
          cplx a2 = aa - q1[i][jm];
          a1 = q1[i][jm] - a2 * a2 / a1;
        } else {
          a1 = q1[i][jm];
        }
        cplx a2 = aa + as2 - 2. * as1;
        if ((a2.re != 0.) || (a2.im != 0.))
          a2 = aa - (as1 - aa) * (as1 - aa) / a2;
        else
          a2 = aa;
        q1[i][jm] = as1;
        q2[i][jm] = as2;
        as1 = a1;
        as2 = a2;
      }
      q1[i][intx - 1] = as1;
      q2[i][intx - 1] = as2;
      double amg = fabs(as2.re) + fabs(as2.im);
      if (amg > den) den = amg;
    }
    const double denm = 1.e-3 * den * kSommCrit;
    int jm = intx - 3;
    if (jm < 1) jm = 1;
    bool brk = false;
    for (int j = jm - 1; j < intx && !brk; j++) {
      for (int i = 0; i < 6; i++) {
        cplx a1 = q2[i][j];
        double d = (fabs(a1.re) + fabs(a1.im)) * kSommCrit;
        if (d < denm) d = denm;
        a1 = q1[i][j] - a1;
        if (fabs(a1.re) + fabs(a1.im) > d) {
          brk = true;
          break;
        }
      }
    }
    if (!brk) {
      for (int i = 0; i < 6; i++) sum[i] = .5 * (q1[i][inx] + q2[i][inx]);
      return;
    }
  }
  E.fail = 1;
}

// The four field functions at the current (rho, zph): contour choice of evlua
__device__ void evlua(const BesselTables& T, Evl& E, cplx* erv, cplx* ezv, cplx* erh, cplx* eph) {
  cplx sum[6], ans[6];
  double del = E.zph;
  if (E.rho > del) del = E.rho;
  if (E.zph >= 2. * E.rho) {
    // Bessel-function form
    E.bessel_form = true;
    E.a = mk(0.0, 0.0);
    del = 1.0 / del;
    if (del > E.tkmag) {
      E.b = mk(0.1 * E.tkmag, -0.1 * E.tkmag);
      rom1(T, E, sum, 2);
      E.a = E.b;
      E.b = mk(del, -del);
      rom1(T, E, ans, 2);
      for (int i = 0; i < 6; i++) sum[i] += ans[i];
    } else {
      E.b = mk(del, -del);
      rom1(T, E, sum, 2);
    }
    const cplx delta = mk(kSommPTP * del, 0.0);
    gshank(T, E, E.b, delta, ans, sum, 0, E.b, E.b);
  } else {
    // Hankel-function form
    E.bessel_form = false;
    cplx cp1 = mk(0.0, .4 * E.ck2), cp2 = mk(.6 * E.ck2, -.2 * E.ck2), cp3 = mk(1.02 * E.ck2, -.2 * E.ck2);
    E.a = cp1;
    E.b = cp2;
    rom1(T, E, sum, 2);
    E.a = cp2;
    E.b = cp3;
    rom1(T, E, ans, 2);
    for (int i = 0; i < 6; i++) sum[i] = -(sum[i] + ans[i]);
    const double slope = (E.zph > .001 * E.rho) ? E.rho / E.zph : 1000.;
    del = kSommPTP / del;
    cplx delta = mk(-1.0, slope) * del / sqrt(1. + slope * slope);
    const cplx delta2 = -conj_(delta);
    cplx bk = mk(0, 0);
    gshank(T, E, cp1, delta, ans, sum, 0, bk, bk);
    double rmis = E.rho * (E.ck1.re - E.ck2);
    bool below;
    if ((rmis < 2. * E.ck2) || (E.rho < 1.e-10)) {
      below = true;
    } else if (E.zph < 1.e-10) {
      below = false;
    } else {
      bk = mk(-E.zph, E.rho) * (E.ck1 - cp3);
      rmis = -bk.re / fabs(bk.im);
      below = rmis > 4. * E.rho / E.zph;
    }
    if (!below) {
      // up between the branch cuts, then to +infinity
      cp1 = E.ck1 - mk(0.1, +0.2);
      cp2 = cp1 + .2;
      bk = mk(0., del);
      gshank(T, E, cp1, bk, sum, ans, 0, bk, bk);
      E.a = cp1;
      E.b = cp2;
      rom1(T, E, ans, 1);
      for (int i = 0; i < 6; i++) ans[i] -= sum[i];
      gshank(T, E, cp3, bk, sum, ans, 0, bk, bk);
      gshank(T, E, cp2, delta2, ans, sum, 0, bk, bk);
    } else {
      // below the branch points, then to +infinity
      for (int i = 0; i < 6; i++) sum[i] = -ans[i];
      rmis = E.ck1.re * 1.01;
      if ((E.ck2 + 1.) > rmis) rmis = E.ck2 + 1.;
      bk = mk(rmis, .99 * E.ck1.im);
      delta = bk - cp3;
      delta = delta * (del / cabs_(delta));
      gshank(T, E, cp3, delta, ans, sum, 1, bk, delta2);
    }
  }
  ans[5] = ans[5] * E.ck1;
  // conjugates: the integrals use exp(-jwt)
  *erv = conj_(E.ck1sq * ans[2]);
  *ezv = conj_(E.ck1sq * (ans[1] + E.ck2sq * ans[4]));
  *erh = conj_(E.ck2sq * (ans[0] + ans[5]));
  *eph = -conj_(E.ck2sq * (ans[3] + ans[5]));
}

// One thread per grid point (257), plus the R = 0 column of the first grid
// from the closed form (thread 0).  eps: complex permittivity (the reference's epscf).
__global__ void __launch_bounds__(32) somm_table_kernel(cplx eps, double eta, cplx* tables, int* status) {
  __shared__ BesselTables T;
  if (threadIdx.x == 0) build_bessel_tables(T);
  __syncthreads();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kSommEvalPoints) {
    Evl E;
    E.fail = 0;
    E.ck2 = kTwoPiD;
    E.ck2sq = E.ck2 * E.ck2;
    E.ck1sq = E.ck2sq * conj_(eps);
    E.ck1 = csqrt_(E.ck1sq);
    E.ck1r = E.ck1.re;
    E.tkmag = 100.0 * cabs_(E.ck1);
    E.tsmag = 100.0 * cnorm(E.ck1);
    E.cksm = E.ck2sq / (E.ck1sq + E.ck2sq);
    E.ct1 = .5 * (E.ck1sq - E.ck2sq);
    cplx erv = E.ck1sq * E.ck1sq, ezv = mk(E.ck2sq * E.ck2sq, 0.0), erh, eph;
    E.ct2 = .125 * (erv - ezv);
    erv = erv * E.ck1sq;
    ezv = ezv * E.ck2sq;
    E.ct3 = .0625 * (erv - ezv);
    // grid, radius and angle index of this point (grid 1 starts at R index 1)
    int g = 0, q = p;
    if (q >= 100) {
      q -= 100;
      g = 1;
      if (q >= 85) {
        q -= 85;
        g = 2;
      }
    }
    const int nr = somm_nx(g), nth = somm_ny(g);
    const int ir = (g == 0) ? 1 + q % (nr - 1) : q % nr;
    const int ith = (g == 0) ? q / (nr - 1) : q / nr;
    // r and theta stepped from the grid start as the reference steps them
    const double dr = somm_dx(g), dth = somm_dy(g);
    double r = (g == 0) ? somm_xs(g) : somm_xs(g) - dr;
    const int irs = (g == 0) ? 1 : 0;
    for (int k = irs; k <= ir; k++) r += dr;
    double thet = somm_ys(g) - dth;
    for (int k = 0; k <= ith; k++) thet += dth;
    E.rho = r * cos(thet);
    E.zph = r * sin(thet);
    if (E.rho < 1.e-7) E.rho = 1.e-8;
    if (E.zph < 1.e-7) E.zph = 0.;
    evlua(T, E, &erv, &ezv, &erh, &eph);
    const double rk = E.ck2 * r;
    double sr, cr;
    sincos(rk, &sr, &cr);
    const cplx con = (-mk(0.0, 4.771341189)) * r / mk(cr, -sr);
    const int nd = nr * nth;
    cplx* o = tables + somm_off(g) + ir + ith * nr;
    o[0] = erv * con;
    o[nd] = ezv * con;
    o[2 * nd] = erh * con;
    o[3 * nd] = eph * con;
    if (E.fail) atomicOr(status, kStatIterCap);
  }
  if (p == 0) {
    // R = 0 of grid 1 from the static limit, c_ggrid.cpp:262-287
    const cplx c4 = mk(0.0, eta / 2.0);
    const cplx cl2 = -c4 * (eps - 1.) / (eps + 1.);
    const cplx cl1 = cl2 / (eps + 1.);
    const cplx ezv = eps * cl1;
    const double dth = somm_dy(2);
    double thet = -dth;
    for (int ith = 0; ith < 10; ith++) {
      thet += dth;
      cplx erv, erh, eph;
      if ((ith + 1) != 10) {
        double tfac2 = cos(thet);
        double tfac1 = (1. - sin(thet)) / tfac2;
        tfac2 = tfac1 / tfac2;
        erv = eps * cl1 * tfac1;
        erh = cl1 * (tfac2 - 1.) + cl2;
        eph = cl1 * tfac2 - cl2;
      } else {
        erv = mk(0., 0.);
        erh = cl2 - .5 * cl1;
        eph = -erh;
      }
      tables[ith * 11 + 0] = erv;
      tables[ith * 11 + 110] = ezv;
      tables[ith * 11 + 220] = erh;
      tables[ith * 11 + 330] = eph;
    }
  }
}

// ---- interpolation with the reference's patch cache ----

// Within one fill the cache is fully described by the cell of its last
// recomputation: grid (or kInterpFresh) and the point's cell indices in
// that grid.  A cache carried over from an earlier fill also holds patch
// coefficients of the earlier tables, which a reuse reads as they are
// (the reference recomputes its tables per frequency and keeps the cache):
// `carry` marks such a cache, whose coefficients live in the engine's
// carried copy until the first recomputation.
constexpr int kInterpFresh = -10;
struct InterpKey {
  int igrs, ix, iy, carry;
};

struct InterpCache {
  int igrs, ix, iy, ixs, iys, ixeg, iyeg, nxm2, nym2, nxms, nyms, nd, ndp;
  int carry;  // coefficients come from a previous fill's tables
  double dx, dy, xs, ys, xz, yz;
  cplx a[4][4], b[4][4], c[4][4], d[4][4];
};

__host__ __device__ inline void interp_cell(int igr, int ix, int iy, int* ixs, int* iys, int* ixeg, int* iyeg) {
  const int nxm2 = somm_nx(igr) - 2, nym2 = somm_ny(igr) - 2;
  *ixs = ((ix - 1) / 3) * 3 + 2;
  if (*ixs < 2) *ixs = 2;
  *ixeg = -10000;
  if (*ixs > nxm2) {
    *ixs = nxm2;
    *ixeg = ((nxm2 + 1) / 3) * 3 + 1;
  }
  *iys = ((iy - 1) / 3) * 3 + 2;
  if (*iys < 2) *iys = 2;
  *iyeg = -10000;
  if (*iys > nym2) {
    *iys = nym2;
    *iyeg = ((nym2 + 1) / 3) * 3 + 1;
  }
}

// Whether a point (x, y) met with cache `k` reuses the cached patch instead
// of recomputing (c_ggrid.cpp:44-54): below the grid start and the cached
// cell passes the region test.
__host__ __device__ inline bool interp_reuses(InterpKey k, double x, double y) {
  if (k.igrs == kInterpFresh) return false;
  if (x >= somm_xs(k.igrs) && y >= somm_ys(k.igrs)) return false;
  int ixs, iys, ixeg, iyeg;
  interp_cell(k.igrs, k.ix, k.iy, &ixs, &iys, &ixeg, &iyeg);
  return (k.ix >= ixeg && k.iy >= iyeg) && (abs(k.ix - ixs) < 2 && abs(k.iy - iys) < 2);
}

__device__ void interp_coefficients(InterpCache& s, const cplx* tables) {
  const cplx* ar = tables + somm_off(s.igrs);
  int iadz = s.ixs + (s.iys - 3) * s.nd - s.ndp;
  for (int k = 0; k < 4; k++) {
    iadz += s.ndp;
    int iadd = iadz;
    for (int i = 0; i < 4; i++) {
      iadd += s.nd;
      const cplx p1 = ar[iadd - 2], p2 = ar[iadd - 1], p3 = ar[iadd], p4 = ar[iadd + 1];
      s.a[i][k] = (p4 - p1 + 3.0 * (p2 - p3)) * 0.1666666667;
      s.b[i][k] = (p1 - 2.0 * p2 + p3) * 0.5;
      s.c[i][k] = p3 - (2.0 * p1 + 3.0 * p2 + p4) * 0.1666666667;
      s.d[i][k] = p2;
    }
  }
  s.xz = (s.ixs - 1) * s.dx + s.xs;
  s.yz = (s.iys - 1) * s.dy + s.ys;
}

__device__ void interp_set_grid(InterpCache& s, int igr) {
  s.igrs = igr;
  s.dx = somm_dx(igr);
  s.dy = somm_dy(igr);
  s.xs = somm_xs(igr);
  s.ys = somm_ys(igr);
  s.nxm2 = somm_nx(igr) - 2;
  s.nym2 = somm_ny(igr) - 2;
  s.nxms = ((s.nxm2 + 1) / 3) * 3 + 1;
  s.nyms = ((s.nym2 + 1) / 3) * 3 + 1;
  s.nd = somm_nx(igr);
  s.ndp = somm_nx(igr) * somm_ny(igr);
}

// Rebuild a cache from its key (c_ggrid::initialize for a fresh one) with
// coefficients from `tables`, or take the carried cache.
__device__ void interp_restore(InterpCache& s, InterpKey k, const cplx* tables, const InterpCache* carried) {
  s.carry = 0;
  if (k.igrs != kInterpFresh && k.carry) {
    s = *carried;
    s.carry = 1;
    return;
  }
  if (k.igrs == kInterpFresh) {
    s.ixs = -10;
    s.iys = -10;
    s.igrs = kInterpFresh;
    s.ixeg = 0;
    s.iyeg = 0;
    s.dx = 1.0;
    s.dy = 1.0;
    s.xs = 0.0;
    s.ys = 0.0;
    s.ix = 0;
    s.iy = 0;
    return;
  }
  interp_set_grid(s, k.igrs);
  s.ix = k.ix;
  s.iy = k.iy;
  interp_cell(k.igrs, k.ix, k.iy, &s.ixs, &s.iys, &s.ixeg, &s.iyeg);
  interp_coefficients(s, tables);
}

// c_ggrid::interpolate: the four functions at R = x, theta = y
__device__ void interp_eval(InterpCache& s, const cplx* tables, double x, double y, cplx f[4]) {
  bool recalc = true;
  if ((x >= s.xs) && (y >= s.ys)) {
    s.ix = (int)((x - s.xs) / s.dx) + 1;
    s.iy = (int)((y - s.ys) / s.dy) + 1;
  } else if (((s.ix >= s.ixeg) && (s.iy >= s.iyeg)) && ((abs(s.ix - s.ixs) < 2) && (abs(s.iy - s.iys) < 2))) {
    recalc = false;
  }
  if (recalc) {
    int igr;
    if (x <= somm_xs(1))
      igr = 0;
    else
      igr = (y > somm_ys(2)) ? 2 : 1;
    if (igr != s.igrs) {
      interp_set_grid(s, igr);
      s.ix = (int)((x - s.xs) / s.dx) + 1;
      s.iy = (int)((y - s.ys) / s.dy) + 1;
    }
    s.ixs = ((s.ix - 1) / 3) * 3 + 2;
    if (s.ixs < 2) s.ixs = 2;
    s.ixeg = -10000;
    if (s.ixs > s.nxm2) {
      s.ixs = s.nxm2;
      s.ixeg = s.nxms;
    }
    s.iys = ((s.iy - 1) / 3) * 3 + 2;
    if (s.iys < 2) s.iys = 2;
    s.iyeg = -10000;
    if (s.iys > s.nym2) {
      s.iys = s.nym2;
      s.iyeg = s.nyms;
    }
    interp_coefficients(s, tables);
    s.carry = 0;
  }
  const double xx = (x - s.xz) / s.dx, yy = (y - s.yz) / s.dy;
  for (int k = 0; k < 4; k++) {
    cplx fx1 = ((s.a[0][k] * xx + s.b[0][k]) * xx + s.c[0][k]) * xx + s.d[0][k];
    cplx fx2 = ((s.a[1][k] * xx + s.b[1][k]) * xx + s.c[1][k]) * xx + s.d[1][k];
    cplx fx3 = ((s.a[2][k] * xx + s.b[2][k]) * xx + s.c[2][k]) * xx + s.d[2][k];
    cplx fx4 = ((s.a[3][k] * xx + s.b[3][k]) * xx + s.c[3][k]) * xx + s.d[3][k];
    cplx p1 = fx4 - fx1 + 3.0 * (fx2 - fx3);
    cplx p2 = 3.0 * (fx1 - 2.0 * fx2 + fx3);
    cplx p3 = 6.0 * fx3 - 2.0 * fx1 - 3.0 * fx2 - fx4;
    f[k] = ((p1 * yy + p2) * yy + p3) * yy * 0.1666666667 + fx2;
  }
}

// ---- near-ground field: rom2 over the source segment ----

struct NearSrc {
  double xj, yj, zj, cabj, sabj, salpj;
  SommGeom g;
};

// sflds, isnor = 1 (6024-6066, 6108-6137): field due to ground of a
// current element at t from the source centre, from the tables.  The
// positions that steer the interpolation are rounded as the reference
// rounds them.  `first` (if set) receives the point (R, theta).
__device__ void sflds_table(const NearSrc& N, double t, InterpCache& S, const cplx* tab, cplx e[9],
                            double2* first) {
  const SommGeom& g = N.g;
  const double xt = __dadd_rn(N.xj, __dmul_rn(t, N.cabj));
  const double yt = __dadd_rn(N.yj, __dmul_rn(t, N.sabj));
  const double zt = __dadd_rn(N.zj, __dmul_rn(t, N.salpj));
  double rhx = g.xo - xt, rhy = g.yo - yt;
  const double rhs = __dadd_rn(__dmul_rn(rhx, rhx), __dmul_rn(rhy, rhy));
  const double rho = sqrt(rhs);
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
  double cph = __dadd_rn(__dmul_rn(rhx, g.xsn), __dmul_rn(rhy, g.ysn));
  double sph = __dsub_rn(__dmul_rn(rhy, g.xsn), __dmul_rn(rhx, g.ysn));
  if (fabs(cph) < 1.0e-10) cph = 0.0;
  if (fabs(sph) < 1.0e-10) sph = 0.0;
  const double zph = g.zo + zt;
  const double r2s = __dadd_rn(rhs, __dmul_rn(zph, zph));
  const double r2 = sqrt(r2s);
  const double rk = r2 * kTwoPiD;
  double sr, cr;
  sincos(rk, &sr, &cr);
  const double thet = (rho >= 1.0e-12) ? atan(zph / rho) : kPiD / 2.0;
  if (first) *first = make_double2(r2, thet);
  cplx f[4];
  interp_eval(S, tab, r2, thet, f);
  const cplx xx2 = mk(cr, -sr) / r2;
  const double sfac = g.sn * cph;
  const cplx erh = xx2 * (N.salpj * f[0] + sfac * f[2]);
  const cplx ezh = xx2 * (N.salpj * f[1] - sfac * f[0]);
  const cplx eph = g.sn * sph * xx2 * f[3];
  e[0] = erh * rhx + eph * phx;
  e[1] = erh * rhy + eph * phy;
  e[2] = ezh;
  double st, ct;
  sincos(kTwoPiD * t, &st, &ct);
  e[3] = e[0] * st;
  e[4] = e[1] * st;
  e[5] = e[2] * st;
  e[6] = e[0] * ct;
  e[7] = e[1] * ct;
  e[8] = e[2] * ct;
}

__device__ __forceinline__ double test_simple(double f1r, double f2r, double dmin) {
  double den = fabs(f2r);
  if (den < dmin) den = dmin;
  if (den < 1.0e-37) return 0.0;
  return fabs((f1r - f2r) / den);
}

// rom2, 5589-5834: Romberg integration of the table field over [a, b]; the
// finest step is (b - a) / nseg (nseg: segments of the structure).
__device__ void rom2_table(const NearSrc& N, double a, double b, cplx sum[9], double dmin, int64_t nseg,
                           InterpCache& S, const cplx* tab, double2* first, int* status) {
  const int n = 9, nts = 4, nx = 1;
  const double rx = 1e-4;
  double z = a, dz = 0.0, dzot = 0.0;
  const double ze = b, s = b - a;
  cplx g1[9], g2[9], g3[9], g4[9], g5[9], t01[9], t10[9], t20[9];
  const double ep = s / (1.0e4 * (double)nseg);
  const double zend = ze - ep;
  for (int i = 0; i < n; i++) sum[i] = mk(0, 0);
  int64_t ns = nx;
  int nt = 0;
  sflds_table(N, z, S, tab, g1, first);
  // every accepted step advances z by at least s / nseg
  for (int64_t guard = 0; guard < 4 * nseg + 64; guard++) {
    dz = s / (double)ns;
    if (__dadd_rn(z, dz) >= ze) {
      dz = ze - z;
      if (dz <= ep) return;
    }
    dzot = dz * .5;
    sflds_table(N, __dadd_rn(z, dzot), S, tab, g3, nullptr);
    sflds_table(N, __dadd_rn(z, dz), S, tab, g5, nullptr);
    bool five = false;
    for (;;) {
      for (int i = 0; i < n; i++) {
        const cplx t00 = (g1[i] + g5[i]) * dzot;
        t01[i] = (t00 + dz * g3[i]) * 0.5;
        t10[i] = (4.0 * t01[i] - t00) / 3.;
      }
      double tmag1 = sqrt(cnorm(t01[0]) + cnorm(t01[1]) + cnorm(t01[2]));
      double tmag2 = sqrt(cnorm(t10[0]) + cnorm(t10[1]) + cnorm(t10[2]));
      if (test_simple(tmag1, tmag2, dmin) <= rx) {
        for (int i = 0; i < n; i++) sum[i] += t10[i];
        nt += 2;
        break;
      }
      sflds_table(N, __dadd_rn(z, __dmul_rn(dz, .25)), S, tab, g2, nullptr);
      sflds_table(N, __dadd_rn(z, __dmul_rn(dz, .75)), S, tab, g4, nullptr);
      cplx t11[9];
      for (int i = 0; i < n; i++) {
        const cplx t02 = (t01[i] + dzot * (g2[i] + g4[i])) * 0.5;
        t11[i] = (4.0 * t02 - t01[i]) / 3.0;
        t20[i] = (16. * t11[i] - t10[i]) / 15.0;
      }
      tmag1 = sqrt(cnorm(t11[0]) + cnorm(t11[1]) + cnorm(t11[2]));
      tmag2 = sqrt(cnorm(t20[0]) + cnorm(t20[1]) + cnorm(t20[2]));
      if (test_simple(tmag1, tmag2, dmin) <= rx) {
        five = true;
        break;
      }
      nt = 0;
      if (ns >= nseg) {
        *status |= kStatRombergCap;
        five = true;
        break;
      }
      ns = ns * 2;
      dz = s / (double)ns;
      dzot = dz * .5;
      for (int i = 0; i < n; i++) {
        g5[i] = g3[i];
        g3[i] = g2[i];
      }
    }
    if (five) {
      for (int i = 0; i < n; i++) sum[i] += t20[i];
      nt = nt + 1;
    }
    z = z + dz;
    if (z > zend) return;
    for (int i = 0; i < n; i++) g1[i] = g5[i];
    if ((nt >= nts) && (ns > nx)) {
      ns = ns / 2;
      nt = 1;
    }
  }
  *status |= kStatIterCap;
}

// Fields of source J at a point within the table limit of J's image:
// direct and image fields plus the table field integrated over the source
// (efld, 2993-3001).
template <bool EXK>
__device__ void near_efld9(const SrcSeg& J, double xi, double yi, double zi, double ai, bool ij,
                           const FieldParams& P, int64_t nseg, InterpCache& S, const cplx* tab, double2* first,
                           cplx ex[9], int* status) {
  pair_fields9<kGroundSommerfeld, EXK>(J, xi, yi, zi, ai, ij, P, ex, status);
  double dmin = cnorm(ex[0]) + cnorm(ex[1]) + cnorm(ex[2]);
  dmin = 0.01 * sqrt(dmin);
  NearSrc N;
  N.xj = J.x;
  N.yj = J.y;
  N.zj = J.z;
  N.cabj = J.cab;
  N.sabj = J.sab;
  N.salpj = J.salp;
  N.g = somm_geometry(J, xi, yi, zi, ai);
  const double shaf = 0.5 * J.s;
  cplx e[9];
  rom2_table(N, -shaf, shaf, e, dmin, nseg, S, tab, first, status);
#pragma unroll
  for (int k = 0; k < 9; k++) ex[k] = ex[k] + e[k];
}

// One near-ground pair of the fill, projected (cmww 2617-2619).
template <bool EXK>
__device__ void near_pair(const SrcSeg& J, double xi, double yi, double zi, double ai, double cabi, double sabi,
                          double salpi, bool ij, const FieldParams& P, int64_t nseg, InterpCache& S,
                          const cplx* tab, double2* first, cplx out[3], int* status) {
  cplx ex[9];
  near_efld9<EXK>(J, xi, yi, zi, ai, ij, P, nseg, S, tab, first, ex, status);
  project_fields(ex, cabi, sabi, salpi, &out[0], &out[1], &out[2]);
}

// Per source column j: whether it has near pairs, the cache it was
// computed from, the cache it leaves, and the first table point it reads.
struct NearRecord {
  int has_near;
  InterpKey used, exit;
  double x1, y1;
};

// The near-ground pairs of the listed source columns.  The reference fills
// source by source (cmset, 2077-2204) and, per source, observation points in
// order; each pair's integration reads the tables through the cache left by
// the previous pair.  One thread follows that order down one column from
// the cache `entry[j]`; with `chain` set a single thread walks all listed
// columns in order, each starting from the cache the previous one left.
// Writes the projected fields of every near pair to G[(i * n + j) * 3 + k].
template <bool EXK>
__global__ void __launch_bounds__(64) near_ground_kernel(FillArgs A, const cplx* __restrict__ tab,
                                                         const int* __restrict__ cols, int ncols,
                                                         const InterpKey* __restrict__ entry,
                                                         const InterpCache* __restrict__ carried,
                                                         NearRecord* __restrict__ rec, cplx* __restrict__ G,
                                                         int chain) {
  int k0, k1;
  if (chain) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    k0 = 0;
    k1 = ncols;
  } else {
    k0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (k0 >= ncols) return;
    k1 = k0 + 1;
  }
  const int64_t n = A.n;
  InterpCache S;
  InterpKey key = entry[cols[k0]];
  interp_restore(S, key, tab, carried);
  int status = 0;
  for (int k = k0; k < k1; k++) {
    const int j = cols[k];
    NearRecord r;
    r.has_near = 0;
    r.used = key;
    r.x1 = r.y1 = 0.0;
    SrcSeg J;
    J.x = A.x[j];
    J.y = A.y[j];
    J.z = A.z[j];
    J.s = A.s[j];
    J.b = A.b[j];
    J.cab = A.cab[j];
    J.sab = A.sab[j];
    J.salp = A.salp[j];
    J.ind1 = EXK ? A.ind1[j] : 0;
    J.ind2 = EXK ? A.ind2[j] : 0;
    J.sfac = far_sfac(J.s);
    for (int64_t i = 0; i < n; i++) {
      const double xi = A.x[i], yi = A.y[i], zi = A.z[i];
      if (image_r2(xi - J.x, yi - J.y, zi + J.z) > .95) continue;
      double2 s1;
      cplx out[3];
      near_pair<EXK>(J, xi, yi, zi, A.b[i], A.cab[i], A.sab[i], A.salp[i], i != j, A.P, n, S, tab,
                     r.has_near ? nullptr : &s1, out, &status);
      if (!r.has_near) {
        r.has_near = 1;
        r.x1 = s1.x;
        r.y1 = s1.y;
      }
      cplx* o = G + (i * n + j) * 3;
      o[0] = out[0];
      o[1] = out[1];
      o[2] = out[2];
    }
    key = InterpKey{S.igrs, S.ix, S.iy, S.carry};
    r.exit = key;
    rec[j] = r;
  }
  if (status) atomicOr(A.status, status);
}

// The cache a fill leaves, with coefficients of this fill's tables, kept
// for the next fill (one thread).
__global__ void interp_store_kernel(InterpKey key, const cplx* __restrict__ tab, InterpCache* __restrict__ out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  InterpCache S;
  key.carry = 0;
  interp_restore(S, key, tab, nullptr);
  *out = S;
}

}  // namespace necb
