/*
 * somm_oracle.c -- CPU restatement of NEC2++'s Sommerfeld ground tables and
 * their interpolation (the near-ground branch of the fill).
 * TEST INFRASTRUCTURE ONLY (see mom_oracle.h).
 *
 * Follows NEC2++ src/c_evlcom.cpp (bessel, hankel, saoa, rom1, gshank,
 * evlua, test) and src/c_ggrid.cpp (sommerfeld, interpolate).  Plain C99
 * complex arithmetic, no contraction, so it rounds as the reference does.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "mom_oracle.h"

typedef double complex cx;

static const double PI = 3.1415926536;
static const double TWO_PI = 2.0 * 3.1415926536;

/* c_evlcom.cpp:28-31 */
#define NM 131072
#define MAXH 20
#define CRIT 1.0E-4
#define PTP .6283185308

/* ---- Bessel / Hankel functions of order zero (c_evlcom.cpp:640-840) ---- */

static int bes_m[101], han_m[101];
static double bes_a1[25], bes_a2[25], han_a1[25], han_a2[25], han_a3[25], han_a4[25];
static int fun_init = 0;

static void init_functions(void) {
  if (fun_init) return;
  for (int k = 1; k <= 25; k++) {
    bes_a1[k - 1] = -0.25 / (k * k);
    bes_a2[k - 1] = 1.0 / (k + 1.0);
  }
  for (int i = 1; i <= 101; i++) {
    double tst = 1.0;
    int init = 0;
    for (int k = 0; k < 24; k++) {
      init = k;
      tst *= -i * bes_a1[k];
      if (tst < 1.0e-6) break;
    }
    bes_m[i - 1] = init + 1;
  }
  double psi = -.5772156649;
  for (int k = 1; k <= 25; k++) {
    int i = k - 1;
    han_a1[i] = -.25 / (k * k);
    han_a2[i] = 1.0 / (k + 1.0);
    psi += 1.0 / k;
    han_a3[i] = psi + psi;
    han_a4[i] = (psi + psi + 1.0 / (k + 1.0)) / (k + 1.0);
  }
  for (int i = 1; i <= 101; i++) {
    double t = 1.0;
    int init = 0;
    for (int k = 0; k < 24; k++) {
      init = k;
      t *= -i * han_a1[k];
      if ((t * han_a3[k]) < 1.e-6) break;
    }
    han_m[i - 1] = init + 1;
  }
  fun_init = 1;
}

#define P10 .0703125
#define P20 .1121520996
#define Q10 .125
#define Q20 .0732421875
#define P11 .1171875
#define P21 .1441955566
#define Q11 .375
#define Q21 .1025390625
#define POF .7853981635
#define C3 .7978845608

static void bessel(cx z, cx* j0, cx* j0p) {
  double zms = creal(z) * creal(z) + cimag(z) * cimag(z);
  if (zms <= 1.e-12) {
    *j0 = 1.0;
    *j0p = -0.5 * z;
    return;
  }
  cx j0x = 0, j0px = 0;
  int ib = 0;
  if (zms <= 37.21) {
    if (zms > 36.0) ib = 1;
    int iz = (int)floor(zms);
    int miz = bes_m[iz];
    *j0 = 1.0;
    *j0p = 1.0;
    cx zk = 1.0, zi = z * z;
    for (int k = 0; k < miz; k++) {
      zk *= bes_a1[k] * zi;
      *j0 += zk;
      *j0p += bes_a2[k] * zk;
    }
    *j0p *= -0.5 * z;
    if (ib == 0) return;
    j0x = *j0;
    j0px = *j0p;
  }
  cx zi = 1.0 / z;
  cx zi2 = zi * zi;
  cx p0z = 1.0 + (P20 * zi2 - P10) * zi2;
  cx p1z = 1.0 + (P11 - P21 * zi2) * zi2;
  cx q0z = (Q20 * zi2 - Q10) * zi;
  cx q1z = (Q11 - Q21 * zi2) * zi;
  cx zk = cexp(I * (z - POF));
  zi2 = 1.0 / zk;
  cx cz = 0.5 * (zk + zi2);
  cx sz = I * 0.5 * (zi2 - zk);
  zk = C3 * csqrt(zi);
  *j0 = zk * (p0z * cz - q0z * sz);
  *j0p = -zk * (p1z * sz + q1z * cz);
  if (ib == 0) return;
  double pi_10 = PI * 10.0;
  zms = cos((sqrt(zms) - 6.0) * pi_10);
  *j0 = 0.5 * (j0x * (1.0 + zms) + *j0 * (1.0 - zms));
  *j0p = 0.5 * (j0px * (1.0 + zms) + *j0p * (1.0 - zms));
}

static int hankel(cx z, cx* h0, cx* h0p) {
  double zms = creal(z) * creal(z) + cimag(z) * cimag(z);
  if (zms == 0.0) return 1;
  cx y0 = 0, y0p = 0;
  int ib = 0;
  if (zms <= 16.81) {
    if (zms > 16.) ib = 1;
    int iz = (int)zms;
    int miz = han_m[iz];
    cx j0 = 1.0, j0p = 1.0, zk = 1.0, zi = z * z;
    for (int k = 0; k < miz; k++) {
      zk *= han_a1[k] * zi;
      j0 += zk;
      j0p += han_a2[k] * zk;
      y0 += han_a3[k] * zk;
      y0p += han_a4[k] * zk;
    }
    j0p *= -.5 * z;
    cx clogz = clog(.5 * z);
    y0 = (2.0 * j0 * clogz - y0) / PI + .3674669052;
    y0p = (2.0 / z + 2.0 * j0p * clogz + 0.5 * y0p * z) / PI + -.02457850915 * z;
    *h0 = j0 + I * y0;
    *h0p = j0p + I * y0p;
    if (ib == 0) return 0;
    y0 = *h0;
    y0p = *h0p;
  }
  cx zi = 1. / z;
  cx zi2 = zi * zi;
  cx p0z = 1. + (P20 * zi2 - P10) * zi2;
  cx p1z = 1. + (P11 - P21 * zi2) * zi2;
  cx q0z = (Q20 * zi2 - Q10) * zi;
  cx q1z = (Q11 - Q21 * zi2) * zi;
  cx zk = cexp(I * (z - POF)) * csqrt(zi) * C3;
  *h0 = zk * (p0z + I * q0z);
  *h0p = I * zk * (p1z + I * q1z);
  if (ib == 0) return 0;
  zms = cos((sqrt(zms) - 4.) * 31.41592654);
  *h0 = .5 * (y0 * (1. + zms) + *h0 * (1. - zms));
  *h0p = .5 * (y0p * (1. + zms) + *h0p * (1. - zms));
  return 0;
}

/* ---- Sommerfeld integrals (c_evlcom.cpp:35-637) ---- */

typedef struct {
  double ck2, ck2sq, tkmag, tsmag, ck1r, zph, rho;
  cx ct1, ct2, ct3, ck1, ck1sq, cksm;
  cx a, b; /* contour end points */
  int bessel_form;
  int fail;
} evl_t;

/* c_evlcom.cpp:847-868 */
static void ctest(double f1r, double f2r, double* tr, double f1i, double f2i, double* ti) {
  double den = fabs(f2r), t = fabs(f2i);
  if (den < t) den = t;
  if (den < 0.0) den = 0.0;
  if (den < 1.0e-37) {
    *tr = 0.0;
    *ti = 0.0;
    return;
  }
  *tr = fabs((f1r - f2r) / den);
  *ti = fabs((f1i - f2i) / den);
}

/* saoa, 382-488 */
static void saoa(evl_t* E, double t, cx ans[6]) {
  cx dxl = E->b - E->a;
  cx xl = E->a + dxl * t;
  cx b0 = 0, b0p = 0, cgam1, cgam2, com, dgam;
  if (E->bessel_form) {
    bessel(xl * E->rho, &b0, &b0p);
    b0 *= 2.;
    b0p *= 2.;
    cgam1 = csqrt(xl * xl - E->ck1sq);
    cgam2 = csqrt(xl * xl - E->ck2sq);
    if (creal(cgam1) == 0.0) cgam1 = CMPLX(0.0, -fabs(cimag(cgam1)));
    if (creal(cgam2) == 0.) cgam2 = CMPLX(0.0, -fabs(cimag(cgam2)));
  } else {
    if (hankel(xl * E->rho, &b0, &b0p)) E->fail = 1;
    com = xl - E->ck1;
    cgam1 = csqrt(xl + E->ck1) * csqrt(com);
    if (creal(com) < 0. && cimag(com) >= 0.) cgam1 = -cgam1;
    com = xl - E->ck2;
    cgam2 = csqrt(xl + E->ck2) * csqrt(com);
    if (creal(com) < 0. && cimag(com) >= 0.) cgam2 = -cgam2;
  }
  double nxl = creal(xl) * creal(xl) + cimag(xl) * cimag(xl);
  if (nxl >= E->tsmag) {
    double sign = 1.0;
    if (cimag(xl) >= 0.0) {
      double xlr = creal(xl);
      if (xlr >= E->ck2) {
        if (xlr <= E->ck1r) {
          dgam = cgam2 - cgam1;
          goto have_dgam;
        }
      } else {
        sign = -1.0;
      }
    }
    dgam = 1.0 / (xl * xl);
    dgam = sign * ((E->ct3 * dgam + E->ct2) * dgam + E->ct1) / xl;
  } else {
    dgam = cgam2 - cgam1;
  }
have_dgam:;
  cx den2 = E->cksm * dgam / (cgam2 * (E->ck1sq * cgam2 + E->ck2sq * cgam1));
  cx den1 = 1. / (cgam1 + cgam2) - E->cksm / cgam2;
  com = dxl * xl * cexp(-cgam2 * E->zph);
  ans[5] = com * b0 * den1 / E->ck1;
  com *= den2;
  if (E->rho != 0.) {
    b0p = b0p / E->rho;
    ans[0] = -com * xl * (b0p + b0 * xl);
    ans[3] = com * xl * b0p;
  } else {
    ans[0] = -com * xl * xl * .5;
    ans[3] = ans[0];
  }
  ans[1] = com * cgam2 * cgam2 * b0;
  ans[2] = -ans[3] * cgam2 * E->rho;
  ans[4] = com * b0;
}

/* rom1, 218-379: Romberg integration from a to b in lambda */
static void rom1(evl_t* E, cx sum[6], int nx) {
  const int n = 6;
  double z = 0.0, ze = 1.0, s = 1.0, ep = s / (1.0e4 * NM), zend = ze - ep, dz = 0.0, dzot = 0.0;
  double tr, ti;
  cx g1[6], g2[6], g3[6], g4[6], g5[6], t01[6], t10[6], t20[6], t00, t11, t02;
  for (int i = 0; i < n; i++) sum[i] = 0;
  int ns = nx, nt = 0;
  saoa(E, z, g1);
  int jump = 0;
  while (1) {
    if (!jump) {
      dz = s / ns;
      if ((z + dz) > ze) {
        dz = ze - z;
        if (dz <= ep) return;
      }
      dzot = dz * .5;
      saoa(E, z + dzot, g3);
      saoa(E, z + dz, g5);
    }
    int nogo = 0;
    for (int i = 0; i < n; i++) {
      t00 = (g1[i] + g5[i]) * dzot;
      t01[i] = (t00 + dz * g3[i]) * .5;
      t10[i] = (4. * t01[i] - t00) / 3.;
      ctest(creal(t01[i]), creal(t10[i]), &tr, cimag(t01[i]), cimag(t10[i]), &ti);
      if ((tr > CRIT) || (ti > CRIT)) nogo = 1;
    }
    if (!nogo) {
      for (int i = 0; i < n; i++) sum[i] += t10[i];
      nt += 2;
      z += dz;
      if (z > zend) return;
      for (int i = 0; i < n; i++) g1[i] = g5[i];
      if ((nt >= 4) && (ns > nx)) {
        ns = ns / 2;
        nt = 1;
      }
      jump = 0;
      continue;
    }
    saoa(E, z + dz * .25, g2);
    saoa(E, z + dz * .75, g4);
    nogo = 0;
    for (int i = 0; i < n; i++) {
      t02 = (t01[i] + dzot * (g2[i] + g4[i])) * .5;
      t11 = (4. * t02 - t01[i]) / 3.;
      t20[i] = (16. * t11 - t10[i]) / 15.;
      ctest(creal(t11), creal(t20[i]), &tr, cimag(t11), cimag(t20[i]), &ti);
      if ((tr > CRIT) || (ti > CRIT)) nogo = 1;
    }
    if (!nogo) {
      for (int i = 0; i < n; i++) sum[i] += t20[i];
      nt++;
      z += dz;
      if (z > zend) return;
      for (int i = 0; i < n; i++) g1[i] = g5[i];
      if ((nt >= 4) && (ns > nx)) {
        ns = ns / 2;
        nt = 1;
      }
      jump = 0;
      continue;
    }
    nt = 0;
    if (ns < NM) {
      ns *= 2;
      dz = s / ns;
      dzot = dz * .5;
      for (int i = 0; i < n; i++) {
        g5[i] = g3[i];
        g3[i] = g2[i];
      }
      jump = 1;
      continue;
    }
    for (int i = 0; i < n; i++) sum[i] += t20[i];
    nt++;
    z += dz;
    if (z > zend) return;
    for (int i = 0; i < n; i++) g1[i] = g5[i];
    if ((nt >= 4) && (ns > nx)) {
      ns /= 2;
      nt = 1;
    }
    jump = 0;
  }
}

/* gshank, 47-214: integration to infinity with Shanks' transformation */
static void gshank(evl_t* E, cx start, cx dela, cx sum[6], const cx seed[6], int ibk, cx bk, cx delb) {
  const int nans = 6;
  cx q1[6][MAXH], q2[6][MAXH], ans1[6], ans2[6], a1, a2, as1, as2, aa;
  double rbk = creal(bk), amg, den, denm;
  cx del = dela;
  int ibx = (ibk == 0) ? 1 : 0;
  for (int i = 0; i < nans; i++) ans2[i] = seed[i];
  E->b = start;
  for (int intx = 1; intx <= MAXH; intx++) {
    int inx = intx - 1;
    E->a = E->b;
    E->b += del;
    if ((ibx == 0) && (creal(E->b) >= rbk)) {
      ibx = 1;
      E->b = bk;
      del = delb;
      rom1(E, sum, 2);
      for (int i = 0; i < nans; i++) ans2[i] += sum[i];
      intx = 0;
      continue;
    }
    rom1(E, sum, 2);
    for (int i = 0; i < nans; i++) ans1[i] = ans2[i] + sum[i];
    E->a = E->b;
    E->b += del;
    if ((ibx == 0) && (creal(E->b) >= rbk)) {
      ibx = 2;
      E->b = bk;
      del = delb;
      rom1(E, sum, 2);
      for (int i = 0; i < nans; i++) ans2[i] = ans1[i] + sum[i];
      intx = 0;
      continue;
    }
    rom1(E, sum, 2);
    for (int i = 0; i < nans; i++) ans2[i] = ans1[i] + sum[i];
    den = 0.;
    for (int i = 0; i < nans; i++) {
      as1 = ans1[i];
      as2 = ans2[i];
      if (intx >= 2) {
        for (int j = 1; j < intx; j++) {
          int jm = j - 1;
          aa = q2[i][jm];
          a1 = q1[i][jm] + as1 - 2. * aa;
          if ((creal(a1) != 0.) || (cimag(a1) != 0.)) {
            a2 = aa - q1[i][jm];
            a1 = q1[i][jm] - a2 * a2 / a1;
          } else {
            a1 = q1[i][jm];
          }
          a2 = aa + as2 - 2. * as1;
          if ((creal(a2) != 0.) || (cimag(a2) != 0.))
            a2 = aa - (as1 - aa) * (as1 - aa) / a2;
          else
            a2 = aa;
          q1[i][jm] = as1;
          q2[i][jm] = as2;
          as1 = a1;
          as2 = a2;
        }
      }
      q1[i][intx - 1] = as1;
      q2[i][intx - 1] = as2;
      amg = fabs(creal(as2)) + fabs(cimag(as2));
      if (amg > den) den = amg;
    }
    denm = 1.e-3 * den * CRIT;
    int jm = intx - 3;
    if (jm < 1) jm = 1;
    int brk = 0;
    for (int j = jm - 1; j < intx; j++) {
      brk = 0;
      for (int i = 0; i < nans; i++) {
        a1 = q2[i][j];
        den = (fabs(creal(a1)) + fabs(cimag(a1))) * CRIT;
        if (den < denm) den = denm;
        a1 = q1[i][j] - a1;
        amg = fabs(creal(a1)) + fabs(cimag(a1));
        if (amg > den) {
          brk = 1;
          break;
        }
      }
      if (brk) break;
    }
    if (!brk) {
      for (int i = 0; i < nans; i++) sum[i] = .5 * (q1[i][inx] + q2[i][inx]);
      return;
    }
  }
  E->fail = 1; /* no convergence */
}

/* evlua, 491-637 */
static void evlua(evl_t* E, cx* erv, cx* ezv, cx* erh, cx* eph) {
  cx sum[6], ans[6], cp1, cp2, cp3, bk = 0, delta, delta2;
  double del = E->zph, slope, rmis;
  if (E->rho > del) del = E->rho;
  if (E->zph >= 2. * E->rho) {
    E->bessel_form = 1;
    E->a = 0.0;
    del = 1.0 / del;
    if (del > E->tkmag) {
      E->b = CMPLX(0.1 * E->tkmag, -0.1 * E->tkmag);
      rom1(E, sum, 2);
      E->a = E->b;
      E->b = CMPLX(del, -del);
      rom1(E, ans, 2);
      for (int i = 0; i < 6; i++) sum[i] += ans[i];
    } else {
      E->b = CMPLX(del, -del);
      rom1(E, sum, 2);
    }
    delta = PTP * del;
    gshank(E, E->b, delta, ans, sum, 0, E->b, E->b);
    ans[5] *= E->ck1;
    *erv = conj(E->ck1sq * ans[2]);
    *ezv = conj(E->ck1sq * (ans[1] + E->ck2sq * ans[4]));
    *erh = conj(E->ck2sq * (ans[0] + ans[5]));
    *eph = -conj(E->ck2sq * (ans[3] + ans[5]));
    return;
  }
  E->bessel_form = 0;
  cp1 = CMPLX(0.0, .4 * E->ck2);
  cp2 = CMPLX(.6 * E->ck2, -.2 * E->ck2);
  cp3 = CMPLX(1.02 * E->ck2, -.2 * E->ck2);
  E->a = cp1;
  E->b = cp2;
  rom1(E, sum, 2);
  E->a = cp2;
  E->b = cp3;
  rom1(E, ans, 2);
  for (int i = 0; i < 6; i++) sum[i] = -(sum[i] + ans[i]);
  if (E->zph > .001 * E->rho)
    slope = E->rho / E->zph;
  else
    slope = 1000.;
  del = PTP / del;
  delta = CMPLX(-1.0, slope) * del / sqrt(1. + slope * slope);
  delta2 = -conj(delta);
  gshank(E, cp1, delta, ans, sum, 0, bk, bk);
  rmis = E->rho * (creal(E->ck1) - E->ck2);
  int jump;
  if ((rmis < 2. * E->ck2) || (E->rho < 1.e-10))
    jump = 1;
  else if (E->zph < 1.e-10)
    jump = 0;
  else {
    bk = CMPLX(-E->zph, E->rho) * (E->ck1 - cp3);
    rmis = -creal(bk) / fabs(cimag(bk));
    jump = (rmis > 4. * E->rho / E->zph) ? 1 : 0;
  }
  if (!jump) {
    cp1 = E->ck1 - CMPLX(0.1, +0.2);
    cp2 = cp1 + .2;
    bk = CMPLX(0., del);
    gshank(E, cp1, bk, sum, ans, 0, bk, bk);
    E->a = cp1;
    E->b = cp2;
    rom1(E, ans, 1);
    for (int i = 0; i < 6; i++) ans[i] -= sum[i];
    gshank(E, cp3, bk, sum, ans, 0, bk, bk);
    gshank(E, cp2, delta2, ans, sum, 0, bk, bk);
  } else {
    for (int i = 0; i < 6; i++) sum[i] = -ans[i];
    rmis = creal(E->ck1) * 1.01;
    if ((E->ck2 + 1.) > rmis) rmis = E->ck2 + 1.;
    bk = CMPLX(rmis, .99 * cimag(E->ck1));
    delta = bk - cp3;
    delta *= del / cabs(delta);
    gshank(E, cp3, delta, ans, sum, 1, bk, delta2);
  }
  ans[5] *= E->ck1;
  *erv = conj(E->ck1sq * ans[2]);
  *ezv = conj(E->ck1sq * (ans[1] + E->ck2sq * ans[4]));
  *erh = conj(E->ck2sq * (ans[0] + ans[5]));
  *eph = -conj(E->ck2sq * (ans[3] + ans[5]));
}

/* Grid layout (c_ggrid.cpp:27-34): three regions in (R, theta). */
static const int nxa[3] = {11, 17, 9}, nya[3] = {10, 5, 8};
static const double dxa[3] = {.02, .05, .1}, dya[3] = {.1745329252, .0872664626, .1745329252};
static const double xsa[3] = {0., .2, .2}, ysa[3] = {0., 0., .3490658504};
static const int grid_off[3] = {0, 440, 780}; /* complex offsets of ar1, ar2, ar3 */

/* sommerfeld (SOMNEC), c_ggrid.cpp:164-288.  tables: 1068 complex
   (ar1 440 | ar2 340 | ar3 288), interleaved re/im.  Returns 0, or 1 when
   an integral did not converge. */
int mo_sommerfeld(double epr, double sig, double wavelength, double eta, double* tables, double* epscf) {
  init_functions();
  cx* ar = (cx*)tables;
  evl_t E;
  memset(&E, 0, sizeof(E));
  const cx const1_neg = -CMPLX(0.0, 4.771341189);
  const cx CONST4 = CMPLX(0.0, eta / 2.0);
  cx eps;
  if (sig >= 0.0)
    eps = CMPLX(epr, -sig * wavelength * (eta / TWO_PI));
  else
    eps = CMPLX(epr, sig);
  epscf[0] = creal(eps);
  epscf[1] = cimag(eps);
  E.ck2 = TWO_PI;
  E.ck2sq = E.ck2 * E.ck2;
  E.ck1sq = E.ck2sq * conj(eps);
  E.ck1 = csqrt(E.ck1sq);
  E.ck1r = creal(E.ck1);
  E.tkmag = 100.0 * cabs(E.ck1);
  E.tsmag = 100.0 * (creal(E.ck1) * creal(E.ck1) + cimag(E.ck1) * cimag(E.ck1));
  E.cksm = E.ck2sq / (E.ck1sq + E.ck2sq);
  E.ct1 = .5 * (E.ck1sq - E.ck2sq);
  cx erv = E.ck1sq * E.ck1sq, ezv = E.ck2sq * E.ck2sq, erh, eph;
  E.ct2 = .125 * (erv - ezv);
  erv *= E.ck1sq;
  ezv *= E.ck2sq;
  E.ct3 = .0625 * (erv - ezv);
  double dth = 0;
  for (int k = 0; k < 3; k++) {
    int nr = nxa[k], nth = nya[k];
    double dr = dxa[k];
    dth = dya[k];
    double r = xsa[k] - dr;
    int irs = 1;
    if (k == 0) {
      r = xsa[k];
      irs = 2;
    }
    for (int ir = irs - 1; ir < nr; ir++) {
      r += dr;
      double thet = ysa[k] - dth;
      for (int ith = 0; ith < nth; ith++) {
        thet += dth;
        E.rho = r * cos(thet);
        E.zph = r * sin(thet);
        if (E.rho < 1.e-7) E.rho = 1.e-8;
        if (E.zph < 1.e-7) E.zph = 0.;
        evlua(&E, &erv, &ezv, &erh, &eph);
        double rk = E.ck2 * r;
        cx con = const1_neg * r / CMPLX(cos(rk), -sin(rk));
        const int nd = nr * nth;
        cx* g = ar + grid_off[k] + ir + ith * nr;
        g[0] = erv * con;
        g[nd] = ezv * con;
        g[2 * nd] = erh * con;
        g[3 * nd] = eph * con;
      }
    }
  }
  cx cl2 = -CONST4 * (eps - 1.) / (eps + 1.);
  cx cl1 = cl2 / (eps + 1.);
  ezv = eps * cl1;
  double thet = -dth;
  int nth = nya[0];
  for (int ith = 0; ith < nth; ith++) {
    thet += dth;
    if ((ith + 1) != nth) {
      double tfac2 = cos(thet);
      double tfac1 = (1. - sin(thet)) / tfac2;
      tfac2 = tfac1 / tfac2;
      erv = eps * cl1 * tfac1;
      erh = cl1 * (tfac2 - 1.) + cl2;
      eph = cl1 * tfac2 - cl2;
    } else {
      erv = 0.;
      erh = cl2 - .5 * cl1;
      eph = -erh;
    }
    ar[0 + ith * 11 + 0] = erv;
    ar[0 + ith * 11 + 110] = ezv;
    ar[0 + ith * 11 + 220] = erh;
    ar[0 + ith * 11 + 330] = eph;
  }
  return E.fail;
}

/* ---- interpolate (was intrp), c_ggrid.cpp:38-162 ----
   The reference keeps the last 4x4 patch between calls.  With `stateful`
   set this restatement reproduces that cache exactly, including its reuse
   of the previous patch when the new point lies below the previous grid's
   start; otherwise every point takes the patch of its own grid cell. */
int64_t mo_interp_size(void) { return (int64_t)sizeof(mo_interp); }

void mo_interp_init(mo_interp* s) {
  memset(s, 0, sizeof(*s));
  s->ixs = -10;
  s->iys = -10;
  s->igrs = -10;
  s->ixeg = 0;
  s->iyeg = 0;
  s->dx = 1.0;
  s->dy = 1.0;
  s->xs = 0.0;
  s->ys = 0.0;
}

void mo_interpolate(mo_interp* s, const double* tables, double x, double y, int stateful, double* f_) {
  static const int nda[3] = {11, 17, 9}, ndpa[3] = {110, 85, 72};
  const cx* tab = (const cx*)tables;
  cx* f = (cx*)f_;
  cx(*A)[4] = (cx(*)[4])s->a;
  cx(*B)[4] = (cx(*)[4])s->b;
  cx(*C)[4] = (cx(*)[4])s->c;
  cx(*D)[4] = (cx(*)[4])s->d;
  int recalc = 1;
  if (!stateful) {
    s->igrs = -10;
    s->xs = 0.0;
    s->ys = 0.0;
  }
  if ((x >= s->xs) && (y >= s->ys)) {
    s->ix = (int)((x - s->xs) / s->dx) + 1;
    s->iy = (int)((y - s->ys) / s->dy) + 1;
  } else if (((s->ix >= s->ixeg) && (s->iy >= s->iyeg)) && ((abs(s->ix - s->ixs) < 2) && (abs(s->iy - s->iys) < 2))) {
    recalc = 0;
  }
  if (recalc) {
    int igr;
    if (x <= xsa[1])
      igr = 0;
    else
      igr = (y > ysa[2]) ? 2 : 1;
    if (igr != s->igrs) {
      s->igrs = igr;
      s->dx = dxa[igr];
      s->dy = dya[igr];
      s->xs = xsa[igr];
      s->ys = ysa[igr];
      s->nxm2 = nxa[igr] - 2;
      s->nym2 = nya[igr] - 2;
      s->nxms = ((s->nxm2 + 1) / 3) * 3 + 1;
      s->nyms = ((s->nym2 + 1) / 3) * 3 + 1;
      s->nd = nda[igr];
      s->ndp = ndpa[igr];
      s->ix = (int)((x - s->xs) / s->dx) + 1;
      s->iy = (int)((y - s->ys) / s->dy) + 1;
    }
    s->ixs = ((s->ix - 1) / 3) * 3 + 2;
    if (s->ixs < 2) s->ixs = 2;
    s->ixeg = -10000;
    if (s->ixs > s->nxm2) {
      s->ixs = s->nxm2;
      s->ixeg = s->nxms;
    }
    s->iys = ((s->iy - 1) / 3) * 3 + 2;
    if (s->iys < 2) s->iys = 2;
    s->iyeg = -10000;
    if (s->iys > s->nym2) {
      s->iys = s->nym2;
      s->iyeg = s->nyms;
    }
    const cx* ar = tab + grid_off[s->igrs];
    int iadz = s->ixs + (s->iys - 3) * s->nd - s->ndp;
    for (int k = 0; k < 4; k++) {
      iadz += s->ndp;
      int iadd = iadz;
      for (int i = 0; i < 4; i++) {
        iadd += s->nd;
        cx p1 = ar[iadd - 2], p2 = ar[iadd - 1], p3 = ar[iadd], p4 = ar[iadd + 1];
        A[i][k] = (p4 - p1 + 3.0 * (p2 - p3)) * 0.1666666667;
        B[i][k] = (p1 - 2.0 * p2 + p3) * 0.5;
        C[i][k] = p3 - (2.0 * p1 + 3.0 * p2 + p4) * 0.1666666667;
        D[i][k] = p2;
      }
    }
    s->xz = (s->ixs - 1) * s->dx + s->xs;
    s->yz = (s->iys - 1) * s->dy + s->ys;
  }
  double xx = (x - s->xz) / s->dx, yy = (y - s->yz) / s->dy;
  for (int k = 0; k < 4; k++) {
    cx fx1 = ((A[0][k] * xx + B[0][k]) * xx + C[0][k]) * xx + D[0][k];
    cx fx2 = ((A[1][k] * xx + B[1][k]) * xx + C[1][k]) * xx + D[1][k];
    cx fx3 = ((A[2][k] * xx + B[2][k]) * xx + C[2][k]) * xx + D[2][k];
    cx fx4 = ((A[3][k] * xx + B[3][k]) * xx + C[3][k]) * xx + D[3][k];
    cx p1 = fx4 - fx1 + 3.0 * (fx2 - fx3);
    cx p2 = 3.0 * (fx1 - 2.0 * fx2 + fx3);
    cx p3 = 6.0 * fx3 - 2.0 * fx1 - 3.0 * fx2 - fx4;
    f[k] = ((p1 * yy + p2) * yy + p3) * yy * 0.1666666667 + fx2;
  }
}
