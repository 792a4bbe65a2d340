/*
 * mom_oracle.c -- CPU restatement of the NEC2++ thin-wire hot path.
 * TEST INFRASTRUCTURE ONLY (see mom_oracle.h).
 *
 * Each function follows the reference routine named beside it
 * (NEC2++ src/nec_context.cpp unless another file is named).
 */
#include "mom_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cx;

static const double PI = 3.1415926536;     /* math_util.h:72-74 */
static const double TWO_PI = 2.0 * 3.1415926536;
static const double C1 = 4.771341189;      /* j*4.771341189, 3055 */

enum { ST_STEP = 1, ST_TABLE = 4 };

/* c_evlcom.cpp:845-868 */
static void test2(double f1r, double f2r, double* tr, double f1i, double f2i, double* ti) {
  double den = fabs(f2r), t = fabs(f2i);
  if (den < t) den = t;
  if (den < 1.0e-37) {
    *tr = 0.0;
    *ti = 0.0;
    return;
  }
  *tr = fabs((f1r - f2r) / den);
  *ti = fabs((f1i - f2i) / den);
}

typedef struct {
  double zpk, rkb2;
  int ija;
} gfstate;

/* gf, 3553-3578 */
static void gf(const gfstate* g, double zk, double* co, double* si) {
  double zdk = zk - g->zpk;
  double rk = sqrt(g->rkb2 + zdk * zdk);
  *si = sin(rk) / rk;
  if (g->ija) {
    *co = cos(rk) / rk;
    return;
  }
  if (rk >= .2) {
    *co = (cos(rk) - 1.0) / rk;
    return;
  }
  double rks = rk * rk;
  *co = ((-1.38888889e-3 * rks + 4.16666667e-2) * rks - 0.5) * rk;
}

/* intx, 4135-4300: variable-interval Romberg integration */
static void intx(const gfstate* g, double el1, double el2, double b, int ij, double* sgr,
                 double* sgi, int* st) {
  const int nx = 1, nma = 65536, nts = 4;
  const double rx = 1.0e-4;
  double z = el1, ze = el2;
  if (ij == 0) ze = 0.;
  double s = ze - z;
  double fnm = nma;
  double ep = s / (10. * fnm);
  double zend = ze - ep;
  double sr = 0., si = 0.;
  int ns = nx, nt = 0, flag = 1;
  double g1r, g1i, g2r = 0, g2i = 0, g3r = 0, g3i = 0, g4r, g4i, g5r = 0, g5i = 0, dz = 0, dzot = 0;
  gf(g, z, &g1r, &g1i);
  for (;;) {
    if (flag) {
      double fns = ns;
      dz = s / fns;
      double zp = z + dz;
      if (zp > ze) {
        dz = ze - z;
        if (fabs(dz) <= ep) break;
      }
      dzot = dz * .5;
      gf(g, z + dzot, &g3r, &g3i);
      gf(g, z + dz, &g5r, &g5i);
    }
    double t00r = (g1r + g5r) * dzot, t00i = (g1i + g5i) * dzot;
    double t01r = (t00r + dz * g3r) * 0.5, t01i = (t00i + dz * g3i) * 0.5;
    double t10r = (4.0 * t01r - t00r) / 3.0, t10i = (4.0 * t01i - t00i) / 3.0;
    double te1r, te1i;
    test2(t01r, t10r, &te1r, t01i, t10i, &te1i);
    if (te1i <= rx && te1r <= rx) {
      sr = sr + t10r;
      si = si + t10i;
      nt += 2;
      z += dz;
      if (z >= zend) break;
      g1r = g5r;
      g1i = g5i;
      if (nt >= nts && ns > nx) {
        ns = ns / 2;
        nt = 1;
      }
      flag = 1;
      continue;
    }
    gf(g, z + dz * 0.25, &g2r, &g2i);
    gf(g, z + dz * 0.75, &g4r, &g4i);
    double t02r = (t01r + dzot * (g2r + g4r)) * 0.5, t02i = (t01i + dzot * (g2i + g4i)) * 0.5;
    double t11r = (4.0 * t02r - t01r) / 3.0, t11i = (4.0 * t02i - t01i) / 3.0;
    double t20r = (16.0 * t11r - t10r) / 15.0, t20i = (16.0 * t11i - t10i) / 15.0;
    double te2r, te2i;
    test2(t11r, t20r, &te2r, t11i, t20i, &te2i);
    if (te2i > rx || te2r > rx) {
      nt = 0;
      if (ns >= nma) {
        *st |= ST_STEP;
      } else {
        ns = ns * 2;
        double fns = ns;
        dz = s / fns;
        dzot = dz * 0.5;
        g5r = g3r;
        g5i = g3i;
        g3r = g2r;
        g3i = g2i;
        flag = 0;
        continue;
      }
    }
    sr = sr + t20r;
    si = si + t20i;
    nt++;
    z += dz;
    if (z >= zend) break;
    g1r = g5r;
    g1i = g5i;
    if (nt >= nts && ns > nx) {
      ns = ns / 2;
      nt = 1;
    }
    flag = 1;
  }
  if (ij == 0) {
    sr = 2. * (sr + log((sqrt(b * b + s * s) + s) / b));
    si = 2. * si;
  }
  *sgr = sr;
  *sgi = si;
}

/* gx, 3605-3620 */
static void gx(double zz, double rh, double xk, cx* gz, cx* gzp) {
  double r2 = zz * zz + rh * rh;
  double r = sqrt(r2);
  double rkz = xk * r;
  cx temp = cos(rkz) - sin(rkz) * I;
  temp = CMPLX(creal(temp) / r, cimag(temp) / r);
  *gz = temp;
  cx a = -CMPLX(1.0, rkz);
  cx p = a * temp;
  *gzp = CMPLX(creal(p) / r2, cimag(p) / r2);
}

static inline cx rmul(double s, cx a) { return CMPLX(s * creal(a), s * cimag(a)); }
static inline cx rdiv(cx a, double s) { return CMPLX(creal(a) / s, cimag(a) / s); }

/* gxx, 3623-3676 */
static void gxx(double zz, double rh, double a, double a2, double xk, int ira, cx* g1, cx* g1p,
                cx* g2, cx* g2p, cx* g3, cx* gzp) {
  double r2 = zz * zz + rh * rh;
  double r = sqrt(r2);
  double r4 = r2 * r2;
  double rk = xk * r;
  double rk2 = rk * rk;
  double rh2 = rh * rh;
  double t1 = .25 * a2 * rh2 / r4;
  double t2 = .5 * a2 / r2;
  cx c1 = CMPLX(1.0, rk);
  cx c2 = rmul(3., c1) - rk2;
  cx c3 = rmul(rk2, CMPLX(6.0, rk)) - rmul(15., c1);
  cx gz = rdiv(CMPLX(cos(rk), -sin(rk)), r);
  *g2 = gz * (1. + rmul(t1, c2));
  *g1 = *g2 - rmul(t2, c1) * gz;
  gz = rdiv(gz, r2);
  *g2p = gz * (rmul(t1, c3) - c1);
  *gzp = rmul(t2, c2) * gz;
  *g3 = *g2p + *gzp;
  *g1p = rmul(zz, *g3);
  if (ira != 1) {
    *g3 = rmul(rh, *g3 + *gzp);
    *gzp = rmul(-zz, c1) * gz;
    if (rh <= 1.0e-10) {
      *g2 = 0.;
      *g2p = 0.;
      return;
    }
    *g2 = rdiv(*g2, rh);
    *g2p = rdiv(rmul(zz, *g2p), rh);
    return;
  }
  t2 = .5 * a;
  *g2 = rmul(-t2, c1) * gz;
  *g2p = rdiv(rmul(t2, gz) * c2, r2);
  *g3 = rmul(rh2, *g2p) - rmul(a, gz) * c1;
  *g2p = rmul(zz, *g2p);
  *gzp = rmul(-zz, c1) * gz;
}

/* eksc, 3051-3104 */
static void eksc(double s, double z, double rh, double xk, int ij, cx* ezs, cx* ers, cx* ezc,
                 cx* erc, cx* ezk, cx* erk, int* st) {
  const cx K = CMPLX(0.0, C1);
  gfstate g;
  g.ija = ij;
  g.zpk = xk * z;
  double rhk = xk * rh;
  g.rkb2 = rhk * rhk;
  double sh = .5 * s;
  double shk = xk * sh;
  double ss = sin(shk), cs = cos(shk);
  double z2a = sh - z;
  double z1a = -(sh + z);
  cx gz1, gz2, gp1, gp2;
  gx(z1a, rh, xk, &gz1, &gp1);
  gx(z2a, rh, xk, &gz2, &gp2);
  cx gzp1 = rmul(z1a, gp1), gzp2 = rmul(z2a, gp2);
  *ezs = K * (rmul(xk, rmul(cs, gz2 - gz1)) - rmul(ss, gzp2 + gzp1));
  *ezc = -K * (rmul(xk, rmul(ss, gz2 + gz1)) + rmul(cs, gzp2 - gzp1));
  *erk = rmul(rh, K * (gp2 - gp1));
  double cint, sint;
  intx(&g, -shk, shk, rhk, ij, &cint, &sint, st);
  *ezk = -K * (gzp2 - gzp1 + rmul(xk * xk, CMPLX(cint, -sint)));
  if (rh >= 1.0e-10) {
    gzp1 = rmul(z1a, gzp1);
    gzp2 = rmul(z2a, gzp2);
    *ers = rdiv(-K * (rmul(ss, gzp2 + gzp1 + gz2 + gz1) - rmul(xk, rmul(cs, rmul(z2a, gz2) - rmul(z1a, gz1)))), rh);
    *erc = rdiv(-K * (rmul(cs, gzp2 - gzp1 + gz2 - gz1) + rmul(xk, rmul(ss, rmul(z2a, gz2) + rmul(z1a, gz1)))), rh);
    return;
  }
  *ers = 0.;
  *erc = 0.;
}

/* ekscx, 3108-3188 */
static void ekscx(double bx, double s, double z, double rhx, double xk, int ij, int inx1, int inx2,
                  cx* ezs, cx* ers, cx* ezc, cx* erc, cx* ezk, cx* erk, int* st) {
  const cx K = CMPLX(0.0, C1);
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
  gfstate g;
  g.ija = ij;
  g.zpk = xk * z;
  double rhk = xk * rh;
  g.rkb2 = rhk * rhk;
  double shk = xk * sh;
  double ss = sin(shk), cs = cos(shk);
  double z2a = sh - z, z1a = -(sh + z);
  double a2 = b * b;
  cx gz1, gz2, gzp1, gzp2, gr1, gr2, grp1, grp2, grk1, grk2, gzz1, gzz2;
  if (inx1 != 2) {
    gxx(z1a, rh, b, a2, xk, ira, &gz1, &gzp1, &gr1, &grp1, &grk1, &gzz1);
  } else {
    gx(z1a, rhx, xk, &gz1, &grk1);
    gzp1 = rmul(z1a, grk1);
    gr1 = rdiv(gz1, rhx);
    grp1 = rdiv(gzp1, rhx);
    grk1 = rmul(rhx, grk1);
    gzz1 = 0.;
  }
  if (inx2 != 2) {
    gxx(z2a, rh, b, a2, xk, ira, &gz2, &gzp2, &gr2, &grp2, &grk2, &gzz2);
  } else {
    gx(z2a, rhx, xk, &gz2, &grk2);
    gzp2 = rmul(z2a, grk2);
    gr2 = rdiv(gz2, rhx);
    grp2 = rdiv(gzp2, rhx);
    grk2 = rmul(rhx, grk2);
    gzz2 = 0.;
  }
  *ezs = K * (rmul(xk, rmul(cs, gz2 - gz1)) - rmul(ss, gzp2 + gzp1));
  *ezc = -K * (rmul(xk, rmul(ss, gz2 + gz1)) + rmul(cs, gzp2 - gzp1));
  *ers = -K * (rmul(ss, rmul(z2a, grp2) + rmul(z1a, grp1) + gr2 + gr1) -
               rmul(xk, rmul(cs, rmul(z2a, gr2) - rmul(z1a, gr1))));
  *erc = -K * (rmul(cs, rmul(z2a, grp2) - rmul(z1a, grp1) + gr2 - gr1) +
               rmul(xk, rmul(ss, rmul(z2a, gr2) + rmul(z1a, gr1))));
  *erk = K * (grk2 - grk1);
  double cint, sint;
  intx(&g, -shk, shk, rhk, ij, &cint, &sint, st);
  double bk = b * xk;
  double bk2 = bk * bk * .25;
  *ezk = -K * (gzp2 - gzp1 + rmul(xk * xk * (1. - bk2), CMPLX(cint, -sint)) - rmul(bk2, gzz2 - gzz1));
}

typedef struct {
  double x, y, z, s, b, cab, sab, salp;
  int ind1, ind2;
} src_t;

/* efld_compute, 2777-2843: fields e[0..8] of one source (direct or image) */
static double efld_compute(const mo_structure* S, const src_t* J, double xij, double yij, double ai,
                           double salpr, double zij, int ijx, cx e[9], int* st) {
  double cabj = J->cab, sabj = J->sab;
  cx tezs = 0, ters = 0, tezc, terc, tezk, terk;
  double zp = xij * cabj + yij * sabj + zij * salpr;
  double rhox = xij - cabj * zp, rhoy = yij - sabj * zp, rhoz = zij - salpr * zp;
  double rh = sqrt(rhox * rhox + rhoy * rhoy + rhoz * rhoz + ai * ai);
  if (rh <= 1.e-10) {
    rhox = 0.0;
    rhoy = 0.0;
    rhoz = 0.0;
  } else {
    rhox /= rh;
    rhoy /= rh;
    rhoz /= rh;
  }
  double r = sqrt(zp * zp + rh * rh);
  if (r >= S->rkh) {
    double rmag = TWO_PI * r;
    double cth = zp / r;
    double px = rh / r;
    cx e0 = CMPLX(cos(rmag), -sin(rmag));
    double py = TWO_PI * r * r;
    cx e1 = rdiv(rmul(S->eta * cth, e0) * CMPLX(1.0, -1.0 / rmag), py);
    cx e2 = rdiv(rmul(S->eta * px, e0) * CMPLX(1.0, rmag - 1.0 / rmag), 2. * py);
    tezk = rmul(cth, e1) - rmul(px, e2);
    terk = rmul(px, e1) + rmul(cth, e2);
    double sf = sin(PI * J->s) / PI;
    tezc = rmul(sf, tezk);
    terc = rmul(sf, terk);
    tezk = rmul(J->s, tezk);
    terk = rmul(J->s, terk);
    e[3] = 0.;
    e[4] = 0.;
    e[5] = 0.;
  } else {
    if (!S->use_exk)
      eksc(J->s, zp, rh, TWO_PI, ijx, &tezs, &ters, &tezc, &terc, &tezk, &terk, st);
    else
      ekscx(J->b, J->s, zp, rh, TWO_PI, ijx, J->ind1, J->ind2, &tezs, &ters, &tezc, &terc, &tezk,
            &terk, st);
    e[3] = rmul(cabj, tezs) + rmul(rhox, ters);
    e[4] = rmul(sabj, tezs) + rmul(rhoy, ters);
    e[5] = rmul(salpr, tezs) + rmul(rhoz, ters);
  }
  e[0] = rmul(cabj, tezk) + rmul(rhox, terk);
  e[1] = rmul(sabj, tezk) + rmul(rhoy, terk);
  e[2] = rmul(salpr, tezk) + rmul(rhoz, terk);
  e[6] = rmul(cabj, tezc) + rmul(rhox, terc);
  e[7] = rmul(sabj, tezc) + rmul(rhoy, terc);
  e[8] = rmul(salpr, tezc) + rmul(rhoz, terc);
  return r;
}

/* fbar, c_ggrid.cpp:291-350 */
static cx fbar(cx p) {
  const double sp = sqrt(PI);
  const double tosp = 2.0 / sp;
  cx z = I * csqrt(p);
  if (cabs(z) <= 3.) {
    cx zs = z * z, sum = z, pw = z;
    for (int i = 1; i <= 100; i++) {
      pw = -pw * zs / (double)i;
      cx term = pw / (2. * i + 1.);
      sum = sum + term;
      double tms = creal(term) * creal(term) + cimag(term) * cimag(term);
      double sms = creal(sum) * creal(sum) + cimag(sum) * cimag(sum);
      if (tms / sms < 1.E-12) break;
    }
    return 1. - (1. - sum * tosp) * z * cexp(zs) * sp;
  }
  int minus = 0;
  if (creal(z) < 0.) {
    minus = 1;
    z = -z;
  }
  cx zs = .5 / (z * z), sum = 0., term = 1.;
  for (int i = 1; i <= 6; i++) {
    term = -term * (2. * i - 1.) * zs;
    sum += term;
  }
  if (minus) sum -= 2.0 * sp * z * cexp(z * z);
  return -sum;
}

/* gwave, c_ggrid.cpp:351-432 (r1 = zmh = 1, xx1 = 0 as set by sflds) */
static void gwave(double r2, double zph, cx xx2, cx u, cx u2, double eta, cx* erv, cx* ezv,
                  cx* erh, cx* ezh, cx* eph) {
  const cx C4 = CMPLX(0.0, eta / 2.0);
  const double r1 = 1.0, zmh = 1.0;
  const cx xx1 = 0.;
  double sppp = zmh / r1, sppp2 = sppp * sppp, cppp2 = 1. - sppp2;
  if (cppp2 < 1.0e-20) cppp2 = 1.0e-20;
  double cppp = sqrt(cppp2);
  double spp = zph / r2, spp2 = spp * spp, cpp2 = 1. - spp2;
  if (cpp2 < 1.0e-20) cpp2 = 1.0e-20;
  double cpp = sqrt(cpp2);
  const cx tpj = CMPLX(0.0, TWO_PI);
  cx rk1 = -tpj * r1, rk2 = -tpj * r2;
  cx t1 = 1. - u2 * cpp2, t2 = csqrt(t1);
  cx t3 = (1. - 1. / rk1) / rk1, t4 = (1. - 1. / rk2) / rk2;
  cx p1 = rk2 * u2 * t1 / (2. * cpp2);
  cx rv = (spp - u * t2) / (spp + u * t2);
  cx omr = 1. - rv;
  cx w = 1. / omr;
  w = CMPLX(4.0, 0.0) * p1 * w * w;
  cx f = fbar(w);
  cx q1 = rk2 * t1 / (2. * u2 * cpp2);
  cx rh = (t2 - u * spp) / (t2 + u * spp);
  cx v = 1. / (1. + rh);
  v = CMPLX(4.0, 0.0) * q1 * v * v;
  cx g = fbar(v);
  cx xr1 = xx1 / r1, xr2 = xx2 / r2;
  cx x1 = cppp2 * xr1, x2 = rv * cpp2 * xr2, x3 = omr * cpp2 * f * xr2;
  cx x4 = u * t2 * spp * 2. * xr2 / rk2;
  cx x5 = xr1 * t3 * (1. - 3. * sppp2), x6 = xr2 * t4 * (1. - 3. * spp2);
  *ezv = (x1 + x2 + x3 - x4 - x5 - x6) * (-C4);
  x1 = sppp * cppp * xr1;
  x2 = rv * spp * cpp * xr2;
  x3 = cpp * omr * u * t2 * f * xr2;
  x4 = spp * cpp * omr * xr2 / rk2;
  x5 = 3. * sppp * cppp * t3 * xr1;
  x6 = cpp * u * t2 * omr * xr2 / rk2 * .5;
  cx x7 = 3. * spp * cpp * t4 * xr2;
  *erv = -(x1 + x2 - x3 + x4 - x5 + x6 - x7) * (-C4);
  *ezh = -(x1 - x2 + x3 - x4 - x5 - x6 + x7) * (-C4);
  x1 = sppp2 * xr1;
  x2 = rv * spp2 * xr2;
  x4 = u2 * t1 * omr * f * xr2;
  x5 = t3 * (1. - 3. * cppp2) * xr1;
  x6 = t4 * (1. - 3. * cpp2) * (1. - u2 * (1. + rv) - u2 * omr * f) * xr2;
  x7 = u2 * cpp2 * omr * (1. - 1. / rk2) * (f * (u2 * t1 - spp2 - 1. / rk2) + 1. / rk2) * xr2;
  *erh = (x1 - x2 - x4 - x5 + x6 + x7) * (-C4);
  x1 = xr1;
  x2 = rh * xr2;
  x3 = (rh + 1.) * g * xr2;
  x4 = t3 * xr1;
  x5 = t4 * (1. - u2 * (1. + rv) - u2 * omr * f) * xr2;
  x6 = .5 * u2 * omr * (f * (u2 * t1 - spp2 - 1. / rk2) + 1. / rk2) * xr2 / rk2;
  *eph = -(x1 - x2 + x3 - x4 + x5 + x6) * (-C4);
}

/* Geometry of one near-ground pair as sflds sees it (nec_context.cpp:6024-6060). */
typedef struct {
  double xj, yj, zj, cabj, sabj, salpj, xo, yo, zo, xsn, ysn, sn;
} sgeom_t;

/* sflds with isnor = 1, nec_context.cpp:6024-6066, 6108-6137: field due to
   ground of a current element at t from the source centre, read from the
   interpolated Sommerfeld tables. */
static void sflds_table(const mo_structure* S, const sgeom_t* G, double t, cx e[9]) {
  double xt = G->xj + t * G->cabj, yt = G->yj + t * G->sabj, zt = G->zj + t * G->salpj;
  double rhx = G->xo - xt, rhy = G->yo - yt, rhs = rhx * rhx + rhy * rhy, rho = sqrt(rhs), phx, phy;
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
  double cph = rhx * G->xsn + rhy * G->ysn, sph = rhy * G->xsn - rhx * G->ysn;
  if (fabs(cph) < 1.0e-10) cph = 0.0;
  if (fabs(sph) < 1.0e-10) sph = 0.0;
  double zph = G->zo + zt, zphs = zph * zph, r2s = rhs + zphs, r2 = sqrt(r2s), rk = r2 * TWO_PI;
  cx xx2 = CMPLX(cos(rk), -sin(rk));
  double thet = (rho >= 1.0e-12) ? atan(zph / rho) : PI / 2.0;
  cx f[4];
  mo_interpolate(S->interp, S->somm, r2, thet, S->interp_stateful, (double*)f);
  cx erv = f[0], ezv = f[1], erh = f[2], eph = f[3];
  xx2 = xx2 / r2;
  double sfac = G->sn * cph;
  erh = xx2 * (G->salpj * erv + sfac * erh);
  cx ezh = xx2 * (G->salpj * ezv - sfac * erv);
  eph = G->sn * sph * xx2 * eph;
  e[0] = erh * rhx + eph * phx;
  e[1] = erh * rhy + eph * phy;
  e[2] = ezh;
  rk = TWO_PI * t;
  sfac = sin(rk);
  e[3] = e[0] * sfac;
  e[4] = e[1] * sfac;
  e[5] = e[2] * sfac;
  sfac = cos(rk);
  e[6] = e[0] * sfac;
  e[7] = e[1] * sfac;
  e[8] = e[2] * sfac;
}

/* test_simple, c_evlcom.cpp:870-883 */
static double test1(double f1r, double f2r, double dmin) {
  double den = fabs(f2r);
  if (den < dmin) den = dmin;
  if (den < 1.0e-37) return 0.0;
  return fabs((f1r - f2r) / den);
}

/* rom2, nec_context.cpp:5589-5834: Romberg integration of the table field
   over the source segment; the finest step is s / n (n segments). */
static void rom2(const mo_structure* S, const sgeom_t* G, double a, double b, cx sum[9], double dmin,
                 int* st) {
  const int n = 9, nts = 4, nx = 1;
  const double rx = 1e-4;
  double dz = 0.0, dzot = 0.0, z = a, ze = b, s = b - a;
  cx g1[9], g2[9], g3[9], g4[9], g5[9], t01[9], t10[9], t20[9], t11[9];
  const double ep = s / (1.0e4 * (double)S->n);
  const double zend = ze - ep;
  for (int i = 0; i < n; i++) sum[i] = 0;
  int ns = nx, nt = 0;
  sflds_table(S, G, z, g1);
  for (;;) {
    /* 3: next interval */
    dz = s / ns;
    if (z + dz >= ze) {
      dz = ze - z;
      if (dz <= ep) return;
    }
    dzot = dz * .5;
    sflds_table(S, G, z + dzot, g3);
    sflds_table(S, G, z + dz, g5);
    for (;;) {
      /* 5: three-point result */
      for (int i = 0; i < n; i++) {
        cx t00 = (g1[i] + g5[i]) * dzot;
        t01[i] = (t00 + dz * g3[i]) * 0.5;
        t10[i] = (4.0 * t01[i] - t00) / 3.;
      }
      double tmag1 = sqrt(creal(t01[0]) * creal(t01[0]) + cimag(t01[0]) * cimag(t01[0]) +
                          (creal(t01[1]) * creal(t01[1]) + cimag(t01[1]) * cimag(t01[1])) +
                          (creal(t01[2]) * creal(t01[2]) + cimag(t01[2]) * cimag(t01[2])));
      double tmag2 = sqrt(creal(t10[0]) * creal(t10[0]) + cimag(t10[0]) * cimag(t10[0]) +
                          (creal(t10[1]) * creal(t10[1]) + cimag(t10[1]) * cimag(t10[1])) +
                          (creal(t10[2]) * creal(t10[2]) + cimag(t10[2]) * cimag(t10[2])));
      if (test1(tmag1, tmag2, dmin) <= rx) {
        for (int i = 0; i < n; i++) sum[i] += t10[i];
        nt += 2;
        goto advance;
      }
      sflds_table(S, G, z + dz * .25, g2);
      sflds_table(S, G, z + dz * .75, g4);
      for (int i = 0; i < n; i++) {
        cx t02 = (t01[i] + dzot * (g2[i] + g4[i])) * 0.5;
        t11[i] = (4.0 * t02 - t01[i]) / 3.0;
        t20[i] = (16. * t11[i] - t10[i]) / 15.0;
      }
      tmag1 = sqrt(creal(t11[0]) * creal(t11[0]) + cimag(t11[0]) * cimag(t11[0]) +
                   (creal(t11[1]) * creal(t11[1]) + cimag(t11[1]) * cimag(t11[1])) +
                   (creal(t11[2]) * creal(t11[2]) + cimag(t11[2]) * cimag(t11[2])));
      tmag2 = sqrt(creal(t20[0]) * creal(t20[0]) + cimag(t20[0]) * cimag(t20[0]) +
                   (creal(t20[1]) * creal(t20[1]) + cimag(t20[1]) * cimag(t20[1])) +
                   (creal(t20[2]) * creal(t20[2]) + cimag(t20[2]) * cimag(t20[2])));
      if (test1(tmag1, tmag2, dmin) <= rx) break;
      /* 14: halve the step, or accept at the limit */
      nt = 0;
      if (ns >= S->n) {
        *st |= ST_STEP;
        break;
      }
      ns = ns * 2;
      dz = s / ns;
      dzot = dz * .5;
      for (int i = 0; i < n; i++) {
        g5[i] = g3[i];
        g3[i] = g2[i];
      }
    }
    /* 10 */
    for (int i = 0; i < n; i++) sum[i] += t20[i];
    nt = nt + 1;
  advance:
    /* 12 */
    z = z + dz;
    if (z > zend) return;
    for (int i = 0; i < n; i++) g1[i] = g5[i];
    if ((nt >= nts) && (ns > nx)) {
      ns = ns / 2;
      nt = 1;
    }
  }
}

/* efld, 2845-3045 + projection of cmww, 2617-2619 */
/* efld, 2845-3045: the nine field components of source J at (xi, yi, zi)
   with observer radius ai. */
static void efld_point(const mo_structure* S, const src_t* J, double xi, double yi, double zi, double ai, int ij,
                       cx ex[9], int* st) {
  cx e[9];
  double xij = xi - J->x, yij = yi - J->y;
  efld_compute(S, J, xij, yij, ai, J->salp, zi - J->z, ij, e, st);
  memcpy(ex, e, sizeof(e));
  const cx zrati = CMPLX(S->zrati_re, S->zrati_im), frati = CMPLX(S->frati_re, S->frati_im);
  if (S->ground != 0) {
    double zij = zi + J->z;
    double r = efld_compute(S, J, xij, yij, ai, -J->salp, zij, 1, e, st);
    if (S->ground == 2) {
      cx zratx = zrati;
      double xymag = sqrt(xij * xij + yij * yij);
      double px, py, cth;
      cx zrsin;
      if (xymag <= 1.0e-6) {
        px = 0.;
        py = 0.;
        cth = 1.;
        zrsin = 1.;
      } else {
        px = -yij / xymag;
        py = xij / xymag;
        cth = zij / r;
        zrsin = csqrt(1.0 - zratx * zratx * (1.0 - cth * cth));
      }
      cx refs = (cth - zratx * zrsin) / (cth + zratx * zrsin);
      cx refps = -(zratx * cth - zrsin) / (zratx * cth + zrsin);
      refps = refps - refs;
      for (int k = 0; k < 9; k += 3) {
        cx epy = rmul(px, e[k]) + rmul(py, e[k + 1]);
        cx epx = rmul(px, epy);
        epy = rmul(py, epy);
        e[k] = refs * e[k] + refps * epx;
        e[k + 1] = refs * e[k + 1] + refps * epy;
        e[k + 2] = refs * e[k + 2];
      }
    }
    for (int k = 0; k < 9; k++) ex[k] -= e[k] * frati;
  }
  if (S->ground == 3) {
    double cabj = J->cab, sabj = J->sab, salpj = J->salp;
    double sn = sqrt(cabj * cabj + sabj * sabj), xsn, ysn;
    if (sn >= 1.0e-5) {
      xsn = cabj / sn;
      ysn = sabj / sn;
    } else {
      sn = 0.0;
      xsn = 1.0;
      ysn = 0.0;
    }
    double zij = zi + J->z, salpr = -salpj;
    double rhox = sabj * zij - salpr * yij, rhoy = salpr * xij - cabj * zij, rhoz = cabj * yij - sabj * xij;
    double rh = sqrt(rhox * rhox + rhoy * rhoy + rhoz * rhoz), xo, yo, zo;
    if (rh <= 1.e-10) {
      xo = xi - ai * ysn;
      yo = yi + ai * xsn;
      zo = zi;
    } else {
      rh = ai / sqrt(rh);
      if (rhoz < 0.0) rh = -rh;
      xo = xi + rh * rhox;
      yo = yi + rh * rhoy;
      zo = zi + rh * rhoz;
    }
    double r = xij * xij + yij * yij + zij * zij;
    if (r <= .95) {
      if (!S->somm) {
        *st |= ST_TABLE;
        for (int k = 0; k < 9; k++) e[k] = 0.;
      } else {
        /* isnor = 1: the table field integrated over the source segment */
        double dmin = creal(ex[0]) * creal(ex[0]) + cimag(ex[0]) * cimag(ex[0]) +
                      (creal(ex[1]) * creal(ex[1]) + cimag(ex[1]) * cimag(ex[1])) +
                      (creal(ex[2]) * creal(ex[2]) + cimag(ex[2]) * cimag(ex[2]));
        dmin = 0.01 * sqrt(dmin);
        double shaf = 0.5 * J->s;
        sgeom_t G = {J->x, J->y, J->z, cabj, sabj, salpj, xo, yo, zo, xsn, ysn, sn};
        rom2(S, &G, -shaf, shaf, e, dmin, st);
      }
    } else {
      /* sflds(0), isnor = 2: 6024-6098 */
      double xt = J->x + 0. * cabj, yt = J->y + 0. * sabj, zt = J->z + 0. * salpj;
      double rhx = xo - xt, rhy = yo - yt, rhs = rhx * rhx + rhy * rhy, rho = sqrt(rhs), phx, phy;
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
      double cph = rhx * xsn + rhy * ysn, sph = rhy * xsn - rhx * ysn;
      if (fabs(cph) < 1.0e-10) cph = 0.0;
      if (fabs(sph) < 1.0e-10) sph = 0.0;
      double zph = zo + zt, zphs = zph * zph, r2s = rhs + zphs, r2 = sqrt(r2s), rk = r2 * TWO_PI;
      cx xx2 = CMPLX(cos(rk), -sin(rk));
      cx erv, ezv, erh, ezh, eph;
      gwave(r2, zph, xx2, zrati, zrati * zrati, S->eta, &erv, &ezv, &erh, &ezh, &eph);
      const cx K = CMPLX(0.0, C1);
      cx et = -K * frati * xx2 / (r2s * r2);
      cx er = 2. * et * CMPLX(1.0, rk);
      et = et * CMPLX(1.0 - rk * rk, rk);
      cx hrv = (er + et) * rho * zph / r2s;
      cx hzv = (zphs * er - rhs * et) / r2s;
      cx hrh = (rhs * er - zphs * et) / r2s;
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
      e[0] = (erh * rhx + eph * phx) * J->s;
      e[1] = (erh * rhy + eph * phy) * J->s;
      e[2] = (ezv + ezh) * J->s;
      e[3] = e[4] = e[5] = 0.;
      double sfac = PI * J->s;
      sfac = sin(sfac) / sfac;
      e[6] = e[0] * sfac;
      e[7] = e[1] * sfac;
      e[8] = e[2] * sfac;
      double zp = xij * cabj + yij * sabj + zij * salpr;
      rh = r - zp * zp;
      double dmin = (rh <= 1.e-10) ? 0.0 : sqrt(rh / (rh + ai * ai));
      if (dmin <= .95) {
        double px = 1. - dmin;
        for (int k = 0; k < 9; k += 3) {
          cx t = (e[k] * cabj + e[k + 1] * sabj + e[k + 2] * salpr) * px;
          e[k] = dmin * e[k] + t * cabj;
          e[k + 1] = dmin * e[k + 1] + t * sabj;
          e[k + 2] = dmin * e[k + 2] + t * salpr;
        }
      }
    }
    for (int k = 0; k < 9; k++) ex[k] = ex[k] + e[k];
  }
}

static void pair(const mo_structure* S, const src_t* J, int64_t i, int ij, cx* etk, cx* ets, cx* etc,
                 int* st) {
  cx ex[9];
  efld_point(S, J, S->x[i], S->y[i], S->z[i], S->b[i], ij, ex, st);
  double cabi = S->cab[i], sabi = S->sab[i], salpi = S->salp[i];
  *etk = rmul(cabi, ex[0]) + rmul(sabi, ex[1]) + rmul(salpi, ex[2]);
  *ets = rmul(cabi, ex[3]) + rmul(sabi, ex[4]) + rmul(salpi, ex[5]);
  *etc = rmul(cabi, ex[6]) + rmul(sabi, ex[7]) + rmul(salpi, ex[8]);
}

/* cmset/cmww, 2077-2204, 2514-2650: for each source j, scatter-add into the
   basis columns of trio(j), obs rows ascending. */
int mo_fill(const mo_structure* S, double* zout) {
  const int64_t n = S->n;
  cx* z = (cx*)zout;
  memset(z, 0, sizeof(cx) * n * n);
  int st = 0;
  for (int64_t j = 0; j < n; j++) {
    src_t J = {S->x[j], S->y[j], S->z[j], S->s[j], S->b[j], S->cab[j], S->sab[j], S->salp[j],
               S->ind1 ? S->ind1[j] : 0, S->ind2 ? S->ind2[j] : 0};
    for (int64_t i = 0; i < n; i++) {
      cx etk, ets, etc;
      pair(S, &J, i, i != j, &etk, &ets, &etc, &st);
      for (int32_t k = S->trio_ptr[j]; k < S->trio_ptr[j + 1]; k++) {
        int64_t b = S->trio_basis[k];
        z[i * n + b] += rmul(S->trio_a[k], etk) + rmul(S->trio_b[k], ets) + rmul(S->trio_c[k], etc);
      }
    }
    /* loading of row j, after source j's contributions (2127-2142) */
    if (S->zload) {
      cx zaj = CMPLX(S->zload[2 * j], S->zload[2 * j + 1]);
      for (int32_t k = S->trio_ptr[j]; k < S->trio_ptr[j + 1]; k++)
        z[j * n + S->trio_basis[k]] -= rmul(S->trio_a[k] + S->trio_c[k], zaj);
    }
  }
  return st;
}

/* LU with partial pivoting (row interchanges, largest modulus). */
int mo_lu(int64_t n, double* a_, int32_t* piv) {
  cx* a = (cx*)a_;
  int bad = 0;
  for (int64_t k = 0; k < n; k++) {
    int64_t p = k;
    double best = -1.0;
    for (int64_t r = k; r < n; r++) {
      cx v = a[r * n + k];
      double m = creal(v) * creal(v) + cimag(v) * cimag(v);
      if (m > best) {
        best = m;
        p = r;
      }
    }
    piv[k] = (int32_t)p;
    if (best == 0.0) {
      bad = 1;
      continue;
    }
    if (p != k)
      for (int64_t c = 0; c < n; c++) {
        cx t = a[k * n + c];
        a[k * n + c] = a[p * n + c];
        a[p * n + c] = t;
      }
    cx pv = a[k * n + k];
    for (int64_t r = k + 1; r < n; r++) {
      cx l = a[r * n + k] / pv;
      a[r * n + k] = l;
      for (int64_t c = k + 1; c < n; c++) a[r * n + c] -= l * a[k * n + c];
    }
  }
  return bad;
}

void mo_solve(int64_t n, const double* lu_, const int32_t* piv, double* b_) {
  const cx* a = (const cx*)lu_;
  cx* b = (cx*)b_;
  for (int64_t k = 0; k < n; k++) {
    int64_t p = piv[k];
    if (p != k) {
      cx t = b[k];
      b[k] = b[p];
      b[p] = t;
    }
  }
  for (int64_t i = 0; i < n; i++)
    for (int64_t j = 0; j < i; j++) b[i] -= a[i * n + j] * b[j];
  for (int64_t i = n - 1; i >= 0; i--) {
    cx s = 0.;
    for (int64_t j = i + 1; j < n; j++) s += a[i * n + j] * b[j];
    b[i] = (b[i] - s) / a[i * n + i];
  }
}

/* get_current_coefficients, c_geometry.cpp:3299-3387: for each segment the
   basis functions with support on it, in ascending basis order. */
void mo_coefficients(const mo_structure* S, const double* x_, double* abc, double* cur) {
  const int64_t n = S->n;
  const cx* x = (const cx*)x_;
  double *air = abc, *aii = abc + n, *bir = abc + 2 * n, *bii = abc + 3 * n, *cir = abc + 4 * n,
         *cii = abc + 5 * n;
  memset(abc, 0, sizeof(double) * 6 * n);
  /* walk basis i ascending; add into the segments it covers */
  int64_t nt = S->trio_ptr[n];
  int64_t* order = (int64_t*)malloc(sizeof(int64_t) * (nt > 0 ? nt : 1));
  int64_t* seg_of = (int64_t*)malloc(sizeof(int64_t) * (nt > 0 ? nt : 1));
  for (int64_t j = 0; j < n; j++)
    for (int32_t k = S->trio_ptr[j]; k < S->trio_ptr[j + 1]; k++) seg_of[k] = j;
  /* counting sort of entries by basis index (stable) */
  int64_t* cnt = (int64_t*)calloc(n + 1, sizeof(int64_t));
  for (int64_t k = 0; k < nt; k++) cnt[S->trio_basis[k] + 1]++;
  for (int64_t i = 0; i < n; i++) cnt[i + 1] += cnt[i];
  for (int64_t k = 0; k < nt; k++) order[cnt[S->trio_basis[k]]++] = k;
  for (int64_t q = 0; q < nt; q++) {
    int64_t k = order[q];
    int64_t i = S->trio_basis[k], j = seg_of[k];
    double ar = creal(x[i]), ai = cimag(x[i]);
    air[j] += S->trio_a[k] * ar;
    aii[j] += S->trio_a[k] * ai;
    bir[j] += S->trio_b[k] * ar;
    bii[j] += S->trio_b[k] * ai;
    cir[j] += S->trio_c[k] * ar;
    cii[j] += S->trio_c[k] * ai;
  }
  for (int64_t j = 0; j < n; j++) {
    cur[2 * j] = air[j] + cir[j];
    cur[2 * j + 1] = aii[j] + cii[j];
  }
  free(order);
  free(seg_of);
  free(cnt);
}

/* ffld, 6639-6888 (wires; free space or infinite-ground image) */
void mo_ffld(const mo_structure* S, const double* abc, double thet, double phi, double* eth_,
             double* eph_) {
  const int64_t n = S->n;
  const double *air = abc, *aii = abc + n, *bir = abc + 2 * n, *bii = abc + 3 * n, *cir = abc + 4 * n,
               *cii = abc + 5 * n;
  const cx CONST3 = CMPLX(0.0, -S->eta / (4.0 * PI));
  const cx zrati = CMPLX(S->zrati_re, S->zrati_im);
  double phx = -sin(phi), phy = cos(phi), roz = cos(thet);
  double thx = roz * phy, thy = -roz * phx, thz = -sin(thet);
  double rox = -thz * phy, roy = thz * phx;
  int ksymp = S->ground ? 2 : 1;
  cx cix = 0, ciy = 0, ciz = 0, ccx = 0, ccy = 0, ccz = 0, rrv = 0, rrh = 0;
  for (int k = 0; k < ksymp; k++) {
    if (k != 0) {
      if (S->ground == 1) {
        rrv = -1.;
        rrh = -1.;
      } else {
        cx zrsin = csqrt(1. - zrati * zrati * thz * thz);
        rrv = -(roz - zrati * zrsin) / (roz + zrati * zrsin);
        rrh = (zrati * roz - zrsin) / (zrati * roz + zrsin);
      }
      roz = -roz;
      ccx = cix;
      ccy = ciy;
      ccz = ciz;
    }
    cix = 0;
    ciy = 0;
    ciz = 0;
    for (int64_t i = 0; i < n; i++) {
      double omega = -(rox * S->cab[i] + roy * S->sab[i] + roz * S->salp[i]);
      double el = PI * S->s[i];
      double sill = omega * el, top = el + sill, bot = el - sill, a, too, boo;
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
      double b = el * (boo - too), c = el * (boo + too);
      double rr = a * air[i] + b * bii[i] + c * cir[i];
      double ri = a * aii[i] - b * bir[i] + c * cii[i];
      double arg = TWO_PI * (S->x[i] * rox + S->y[i] * roy + S->z[i] * roz);
      cx exa = CMPLX(cos(arg), sin(arg)) * CMPLX(rr, ri);
      cix = cix + rmul(S->cab[i], exa);
      ciy = ciy + rmul(S->sab[i], exa);
      ciz = ciz + rmul(S->salp[i], exa);
    }
    if (k == 0) continue;
    cx cdp = (rmul(phx, cix) + rmul(phy, ciy)) * (rrh - rrv);
    cix = ccx + cix * rrv + rmul(phx, cdp);
    ciy = ccy + ciy * rrv + rmul(phy, cdp);
    ciz = ccz - ciz * rrv;
  }
  cx eth = (rmul(thx, cix) + rmul(thy, ciy) + rmul(thz, ciz)) * CONST3;
  cx eph = (rmul(phx, cix) + rmul(phy, ciy)) * CONST3;
  eth_[0] = creal(eth);
  eth_[1] = cimag(eth);
  eph_[0] = creal(eph);
  eph_[1] = cimag(eph);
}

/* ---- near fields (nefld 4304-4490, nhfld 5189-5265) ---- */

static src_t source_of(const mo_structure* S, int64_t i) {
  src_t J = {S->x[i], S->y[i], S->z[i], S->s[i], S->b[i], S->cab[i], S->sab[i], S->salp[i],
             S->ind1 ? S->ind1[i] : 0, S->ind2 ? S->ind2[i] : 0};
  return J;
}

/* radius of the segment whose volume holds the point, else 0 (4316-4334) */
static double point_radius(const mo_structure* S, double xob, double yob, double zob) {
  for (int64_t i = 0; i < S->n; i++) {
    double xj = xob - S->x[i], yj = yob - S->y[i], zj = zob - S->z[i];
    double zp = S->cab[i] * xj + S->sab[i] * yj + S->salp[i] * zj;
    if (fabs(zp) > 0.5001 * S->s[i]) continue;
    zp = xj * xj + yj * yj + zj * zj - zp * zp;
    xj = S->b[i];
    if (zp > 0.9 * xj * xj) continue;
    return xj;
  }
  return 0.0;
}

static cx seg_coef(const double* abc, int64_t n, int64_t i, int k) {
  return CMPLX(abc[2 * k * n + i], abc[(2 * k + 1) * n + i]);
}

void mo_nefld(const mo_structure* S, const double* abc, double xob, double yob, double zob, double* out) {
  const int64_t n = S->n;
  cx f[3] = {0, 0, 0};
  const double ax = point_radius(S, xob, yob, zob);
  int st = 0;
  for (int64_t i = 0; i < n; i++) {
    src_t J = source_of(S, i);
    cx e[9];
    efld_point(S, &J, xob, yob, zob, ax, 1, e, &st);
    cx acx = seg_coef(abc, n, i, 0), bcx = seg_coef(abc, n, i, 1), ccx = seg_coef(abc, n, i, 2);
    f[0] += e[0] * acx + e[3] * bcx + e[6] * ccx;
    f[1] += e[1] * acx + e[4] * bcx + e[7] * ccx;
    f[2] += e[2] * acx + e[5] * bcx + e[8] * ccx;
  }
  for (int k = 0; k < 3; k++) {
    out[2 * k] = creal(f[k]);
    out[2 * k + 1] = cimag(f[k]);
  }
}

typedef struct {
  double zpka, rhks;
} ghstate;

/* gh, 3582-3600 */
static void gh(const ghstate* g, double zk, double* hr, double* hi) {
  double rs = zk - g->zpka;
  rs = g->rhks + rs * rs;
  double r = sqrt(rs), ckr = cos(r), skr = sin(r), rr2 = 1. / rs, rr3 = rr2 / r;
  *hr = skr * rr2 + ckr * rr3;
  *hi = ckr * rr2 - skr * rr3;
}

/* hfk, 3681-3822: H field of a uniform filament by Romberg integration */
static void hfk(double el1, double el2, double rhk, double zpkx, double* sgr, double* sgi) {
  const int nx = 1, nma = 65536, nts = 4;
  const double rx = 1.0e-4;
  ghstate G = {zpkx, rhk * rhk};
  double z = el1, ze = el2, s = ze - z, ep = s / (10. * nma), zend = ze - ep, dz = 0., dzot = 0., zp;
  double g1r, g1i, g2r, g2i, g3r, g3i, g4r, g4i, g5r, g5i, te1r, te1i, te2r, te2i;
  *sgr = 0.0;
  *sgi = 0.0;
  int ns = nx, nt = 0, flag = 1;
  gh(&G, z, &g1r, &g1i);
  for (;;) {
    if (flag) {
      dz = s / ns;
      zp = z + dz;
      if (zp > ze) {
        dz = ze - z;
        if (fabs(dz) <= ep) {
          *sgr = *sgr * rhk * .5;
          *sgi = *sgi * rhk * .5;
          return;
        }
      }
      dzot = dz * .5;
      zp = z + dzot;
      gh(&G, zp, &g3r, &g3i);
      zp = z + dz;
      gh(&G, zp, &g5r, &g5i);
    }
    double t00r = (g1r + g5r) * dzot, t00i = (g1i + g5i) * dzot;
    double t01r = (t00r + dz * g3r) * 0.5, t01i = (t00i + dz * g3i) * 0.5;
    double t10r = (4.0 * t01r - t00r) / 3.0, t10i = (4.0 * t01i - t00i) / 3.0;
    test2(t01r, t10r, &te1r, t01i, t10i, &te1i);
    if ((te1i <= rx) && (te1r <= rx)) {
      *sgr = *sgr + t10r;
      *sgi = *sgi + t10i;
      nt += 2;
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
      flag = 1;
      continue;
    }
    zp = z + dz * 0.25;
    gh(&G, zp, &g2r, &g2i);
    zp = z + dz * 0.75;
    gh(&G, zp, &g4r, &g4i);
    double t02r = (t01r + dzot * (g2r + g4r)) * 0.5, t02i = (t01i + dzot * (g2i + g4i)) * 0.5;
    double t11r = (4.0 * t02r - t01r) / 3.0, t11i = (4.0 * t02i - t01i) / 3.0;
    double t20r = (16.0 * t11r - t10r) / 15.0, t20i = (16.0 * t11i - t10i) / 15.0;
    test2(t11r, t20r, &te2r, t11i, t20i, &te2i);
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
        flag = 0;
        continue;
      }
    }
    *sgr = *sgr + t20r;
    *sgi = *sgi + t20i;
    nt++;
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
    flag = 1;
  }
}

/* hsflx, 4059-4133: H of the constant, sine and cosine currents of a segment */
static void hsflx(double s, double rh, double zpx, cx* hpk, cx* hps, cx* hpc) {
  const double pi8 = PI * 8.0;
  const cx fjk = -CMPLX(0.0, TWO_PI);
  if (rh >= 1.0e-10) {
    double zp, hss;
    if (zpx >= 0.0) {
      zp = zpx;
      hss = 1.;
    } else {
      zp = -zpx;
      hss = -1.;
    }
    double dh = 0.5 * s, z1 = zp + dh, z2a = zp - dh, rhz;
    if (z2a >= 1.0e-7)
      rhz = rh / z2a;
    else
      rhz = 1.;
    double dk = TWO_PI * dh, cdk = cos(dk), sdk = sin(dk), hkr, hki;
    hfk(-dk, dk, rh * TWO_PI, zp * TWO_PI, &hkr, &hki);
    *hpk = CMPLX(hkr, hki);
    if (rhz >= 1.0e-3) {
      double rh2 = rh * rh, r1 = sqrt(rh2 + z1 * z1), r2 = sqrt(rh2 + z2a * z2a);
      cx ekr1 = cexp(fjk * r1), ekr2 = cexp(fjk * r2);
      cx t1 = z1 * ekr1 / r1, t2 = z2a * ekr2 / r2;
      *hps = (cdk * (ekr2 - ekr1) - I * sdk * (t2 + t1)) * hss;
      *hpc = -sdk * (ekr2 + ekr1) - I * cdk * (t2 - t1);
      cx cons = -I / (2.0 * TWO_PI * rh);
      *hps = cons * *hps;
      *hpc = cons * *hpc;
      return;
    }
    cx ekr1 = CMPLX(cdk, sdk) / (z2a * z2a), ekr2 = CMPLX(cdk, -sdk) / (z1 * z1);
    double t1 = TWO_PI * (1.0 / z1 - 1.0 / z2a);
    cx t2 = cexp(fjk * zp) * rh / pi8;
    *hps = t2 * (t1 + (ekr1 + ekr2) * sdk) * hss;
    *hpc = t2 * (-I * t1 + (ekr1 - ekr2) * cdk);
    return;
  }
  *hps = 0;
  *hpc = 0;
  *hpk = 0;
}

/* hsfld, 3927-4056: H of segment J at (xi, yi, zi) with its image */
static void hsfld(const mo_structure* S, const src_t* J, double xi, double yi, double zi, double ai, cx h[9]) {
  const double xij = xi - J->x, yij = yi - J->y;
  const int ksymp = (S->ground != 0) ? 2 : 1;
  double rfl = -1.;
  for (int k = 0; k < 9; k++) h[k] = 0;
  for (int gl = 0; gl < ksymp; gl++) {
    rfl = -rfl;
    double salpr = J->salp * rfl, zij = zi - rfl * J->z;
    double zp = xij * J->cab + yij * J->sab + zij * salpr;
    double rhox = xij - J->cab * zp, rhoy = yij - J->sab * zp, rhoz = zij - salpr * zp;
    double rh = sqrt(rhox * rhox + rhoy * rhoy + rhoz * rhoz + ai * ai);
    if (rh <= 1.0e-10) {
      for (int k = 0; k < 9; k++) h[k] = 0;
      continue;
    }
    rhox = rhox / rh;
    rhoy = rhoy / rh;
    rhoz = rhoz / rh;
    double phx = J->sab * rhoz - salpr * rhoy, phy = salpr * rhox - J->cab * rhoz, phz = J->cab * rhoy - J->sab * rhox;
    cx hp[3];
    hsflx(J->s, rh, zp, &hp[0], &hp[1], &hp[2]);
    if (gl == 1) {
      if (S->ground != 1) {
        cx zratx = CMPLX(S->zrati_re, S->zrati_im), rrv, rrh;
        double rmag = sqrt(zp * zp + rh * rh), xymag = sqrt(xij * xij + yij * yij), px, py, cth;
        if (xymag <= 1.0e-6) {
          px = 0.;
          py = 0.;
          cth = 1.;
          rrv = 1.0;
        } else {
          px = -yij / xymag;
          py = xij / xymag;
          cth = zij / rmag;
          rrv = csqrt(1. - zratx * zratx * (1. - cth * cth));
        }
        rrh = zratx * cth;
        rrh = -(rrh - rrv) / (rrh + rrv);
        rrv = zratx * rrv;
        rrv = (cth - rrv) / (cth + rrv);
        cx qy = (phx * px + phy * py) * (rrv - rrh);
        cx qx = qy * px + phx * rrh;
        qy = qy * py + phy * rrh;
        cx qz = phz * rrh;
        for (int k = 0; k < 3; k++) {
          h[3 * k] = h[3 * k] - hp[k] * qx;
          h[3 * k + 1] = h[3 * k + 1] - hp[k] * qy;
          h[3 * k + 2] = h[3 * k + 2] - hp[k] * qz;
        }
        continue;
      }
      for (int k = 0; k < 3; k++) {
        h[3 * k] = h[3 * k] - hp[k] * phx;
        h[3 * k + 1] = h[3 * k + 1] - hp[k] * phy;
        h[3 * k + 2] = h[3 * k + 2] - hp[k] * phz;
      }
      continue;
    }
    for (int k = 0; k < 3; k++) {
      h[3 * k] = hp[k] * phx;
      h[3 * k + 1] = hp[k] * phy;
      h[3 * k + 2] = hp[k] * phz;
    }
  }
}

void mo_nhfld(const mo_structure* S, const double* abc, double xob, double yob, double zob, double* out) {
  const int64_t n = S->n;
  cx f[3] = {0, 0, 0};
  const double ax = point_radius(S, xob, yob, zob);
  for (int64_t i = 0; i < n; i++) {
    src_t J = source_of(S, i);
    cx h[9];
    hsfld(S, &J, xob, yob, zob, ax, h);
    cx acx = seg_coef(abc, n, i, 0), bcx = seg_coef(abc, n, i, 1), ccx = seg_coef(abc, n, i, 2);
    f[0] += h[0] * acx + h[3] * bcx + h[6] * ccx;
    f[1] += h[1] * acx + h[4] * bcx + h[7] * ccx;
    f[2] += h[2] * acx + h[5] * bcx + h[8] * ccx;
  }
  for (int k = 0; k < 3; k++) {
    out[2 * k] = creal(f[k]);
    out[2 * k + 1] = cimag(f[k]);
  }
}
