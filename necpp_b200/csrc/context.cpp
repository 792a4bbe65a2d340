// Card state machine, excitation, network-free solve and far-field epilogue.
// Follows nec_context (src/nec_context.cpp, line ranges per function); the
// fill, factor, solve and far-field sum run on the GPU via necgpu.h.
#include "context.h"
#include "host_parallel.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>

#include "../../include/necgpu.h"
#include "nec_constants.h"
#include "nec_error.h"

namespace necb {

Medium& medium() {
  static Medium m;
  return m;
}

namespace {
void check(necgpu_engine* e, int st) {
  if (st != NECGPU_OK) fail("GPU: ", necgpu_last_error(e));
}
}  // namespace

Context::Context() {}
Context::~Context() {
  if (eng_) necgpu_release(eng_);
}

necgpu_engine* Context::engine() {
  if (!eng_) {
    int dev = 0;
    if (const char* s = std::getenv("NECPP_B200_DEVICE")) dev = std::atoi(s);
    necgpu_engine* e = nullptr;
    int st = necgpu_acquire(&e, dev);
    if (st != NECGPU_OK) {
      std::string msg = e ? necgpu_last_error(e) : "no CUDA device";
      if (e) necgpu_destroy(e);
      fail("GPU: ", msg);
    }
    eng_ = e;
  }
  return eng_;
}

// calc_prepare, src/nec_context.cpp:123-165
void Context::calc_prepare() {
  iflow = 1;
  state_ = MEM;
  rkh = 1.;
  use_exk = false;
  ex_type = 0;
  m_near = -1;
  ifar = -1;
  freq_mhz = speed_of_light() / 1.0e6;
  zrati = cd(1.0, 0.0);
  ksymp = 1;
  nradl = 0;
  iperf = 0;
  epsr = 0;
  sig = 0;
  nfrq = 1;
  iptflg = -2;
  iptflq = -1;
  iped = 0;
}

void Context::reset_to_structure_loading() {
  if (state_ != MEM) state_ = STRUCT;
}
void Context::reset_to_excitation_setup() {
  if (state_ != MEM && state_ != STRUCT) state_ = EXSETUP;
}

void Context::geometry_complete(int gpflag) {
  geo_.complete(gpflag);
  calc_prepare();
}

// fr_card, src/nec_context.cpp:406-420
void Context::fr_card(int in_ifrq, int in_nfrq, double in_freq, double in_del) {
  ifrq = in_ifrq;
  nfrq = in_nfrq == 0 ? 1 : in_nfrq;
  freq_mhz = in_freq;
  delfrq = in_del;
  if (iped == 1) zpnorm = 0.0;
  state_ = MEM;
  iflow = 1;
}

// gn_card / nec_ground::parse_gn, src/nec_context.cpp:486-499,
// src/nec_ground.cpp:75-120
// ld_card, src/nec_context.cpp:424-473: consecutive LD cards accumulate;
// the first after other cards (or type -1) clears the previous loads.
void Context::ld_card(int type, int tag, int tag_from, int tag_to, double zr, double zi, double zc) {
  if (iflow != 3) {
    iflow = 3;
    ldtyp.clear();
    ldtag.clear();
    ldtagf.clear();
    ldtagt.clear();
    zlr.clear();
    zli.clear();
    zlc.clear();
    zarray.clear();
    reset_to_structure_loading();
    if (type == -1) return;
  }
  if (tag_to == 0) tag_to = tag_from;
  ldtyp.push_back(type);
  ldtag.push_back(tag);
  ldtagf.push_back(tag_from);
  ldtagt.push_back(tag_to);
  // a faulty card stays in the list with zero impedance, as in the reference
  zlr.push_back(0.0);
  zli.push_back(0.0);
  zlc.push_back(0.0);
  if (tag_to < tag_from)
    fail("DATA FAULT ON LOADING CARD No: ", (int)ldtyp.size(), ": ITAG STEP1: ", tag_from,
         " IS GREATER THAN ITAG STEP2: ", tag_to);
  zlr.back() = zr;
  zli.back() = zi;
  zlc.back() = zc;
}

// nt_card / tl_card, src/nec_context.cpp:630-707: the first NT or TL card
// after other cards clears the networks (seg1 == -1 cancels them all).
void Context::network_card(int type, int tag1, int seg1, int tag2, int seg2, const double* x) {
  if (iflow != 6) {
    ntyp.clear();
    iseg1.clear();
    iseg2.clear();
    x11r.clear();
    x11i.clear();
    x12r.clear();
    x12i.clear();
    x22r.clear();
    x22i.clear();
    ntsol = 0;
    iflow = 6;
    reset_to_excitation_setup();
    if (seg1 == -1) return;
  }
  if (!geo_.completed) fail("NT/TL card before geometry_complete");
  const int64_t s1 = geo_.segment_number(tag1, seg1);
  const int64_t s2 = geo_.segment_number(tag2, seg2);
  if (s1 < 1 || s1 > geo_.n || s2 < 1 || s2 > geo_.n)
    fail("NETWORK DATA ERROR: SEGMENT NUMBER OUT OF RANGE (", s1, ", ", s2, ")");
  ntyp.push_back(type);
  iseg1.push_back(s1);
  iseg2.push_back(s2);
  x11r.push_back(x[0]);
  x11i.push_back(x[1]);
  x12r.push_back(x[2]);
  x12i.push_back(x[3]);
  x22r.push_back(x[4]);
  x22i.push_back(x[5]);
  if (type == 2 && x[0] <= 0.0) {  // a negative characteristic impedance is a crossed line
    ntyp.back() = 3;
    x11r.back() = -x[0];
  }
}

void Context::nt_card(int tag1, int seg1, int tag2, int seg2, double y11r, double y11i, double y12r,
                      double y12i, double y22r, double y22i) {
  const double x[6] = {y11r, y11i, y12r, y12i, y22r, y22i};
  network_card(1, tag1, seg1, tag2, seg2, x);
}

void Context::tl_card(int tag1, int seg1, int tag2, int seg2, double z0, double length, double y1r,
                      double y1i, double y2r, double y2i) {
  const double x[6] = {z0, length, y1r, y1i, y2r, y2i};
  network_card(2, tag1, seg1, tag2, seg2, x);
}

// ne_nh_card, src/nec_context.cpp:928-961: a near-field request (electric
// for nfeh 0, magnetic for 1) over nx x ny x nz points, rectangular
// (near = 0: x, y, z from (x0, y0, z0) in steps (dx, dy, dz), metres) or
// spherical (near = 1: r, phi, theta, degrees); blank counts mean 1.  With
// one frequency the request runs at once.
void Context::ne_nh_card(int in_nfeh, int near, int nx, int ny, int nz, double x0, double y0, double z0,
                         double dx, double dy, double dz) {
  nfeh = in_nfeh;
  m_near = near;
  nrx = nx == 0 ? 1 : nx;
  nry = ny == 0 ? 1 : ny;
  nrz = nz == 0 ? 1 : nz;
  xnr = x0;
  ynr = y0;
  znr = z0;
  dxnr = dx;
  dynr = dy;
  dznr = dz;
  iflow = 8;
  if (nfrq == 1) simulate(false);
}

// nfpat, src/nec_context.cpp:5068-5186: the points in the reference's order
// (z outer, then y, then x), their fields from one device call.
void Context::nfpat() {
  NearFieldPattern p;
  p.freq_hz = freq_mhz * 1.0e6;
  p.nfeh = nfeh;
  std::vector<double> pts;
  double znrt = znr - dznr, cth = 0., sth = 0., cph = 0., sph = 0.;
  for (int i = 0; i < nrz; i++) {
    znrt += dznr;
    if (m_near != 0) {
      cth = std::cos(degrees_to_rad(znrt));
      sth = std::sin(degrees_to_rad(znrt));
    }
    double ynrt = ynr - dynr;
    for (int j = 0; j < nry; j++) {
      ynrt += dynr;
      if (m_near != 0) {
        cph = std::cos(degrees_to_rad(ynrt));
        sph = std::sin(degrees_to_rad(ynrt));
      }
      double xnrt = xnr - dxnr;
      for (int k = 0; k < nrx; k++) {
        xnrt += dxnr;
        double xob, yob, zob;
        if (m_near != 0) {
          xob = xnrt * sth * cph;
          yob = xnrt * sth * sph;
          zob = xnrt * cth;
        } else {
          xob = xnrt;
          yob = ynrt;
          zob = znrt;
        }
        p.x.push_back(xob);
        p.y.push_back(yob);
        p.z.push_back(zob);
        pts.push_back(xob / wavelength_);
        pts.push_back(yob / wavelength_);
        pts.push_back(zob / wavelength_);
      }
    }
  }
  const int np = (int)p.x.size();
  std::vector<cd> f(3 * (size_t)np);
  necgpu_engine* e = engine();
  check(e, necgpu_near_field(e, nfeh == 1 ? 1 : 0, np, pts.data(), reinterpret_cast<double*>(f.data())));
  for (int i = 0; i < np; i++) {
    p.fx.push_back(f[3 * i]);
    p.fy.push_back(f[3 * i + 1]);
    p.fz.push_back(f[3 * i + 2]);
  }
  p.seq = next_seq();
  near_fields.push_back(std::move(p));
}

// calculate_network_data, src/nec_context.cpp:1210-1243: a transmission line
// given with length <= 0 takes the straight distance between its two port
// segments (metres, kept for later frequencies).  Done once per excitation
// sweep, before the first incidence angle.
void Context::network_lengths() {
  if (ntyp.empty() || inc > 1) return;
  for (size_t j = 0; j < ntyp.size(); j++) {
    if (ntyp[j] < 2 || x11i[j] > 0.0) continue;
    const int64_t a = iseg1[j] - 1, b = iseg2[j] - 1;
    const double dx = geo_.x[b] - geo_.x[a], dy = geo_.y[b] - geo_.y[a], dz = geo_.z[b] - geo_.z[a];
    x11i[j] = wavelength_ * std::sqrt(dx * dx + dy * dy + dz * dz);
  }
}

namespace {
// Internal impedance of a round wire of conductivity sigl (S/m, times the
// wavelength) and radius rolam (wavelengths): the reference's zint
// (src/nec_context.cpp:6321-6400), i.e. the NEC-2 ratio of Kelvin functions
// from polynomial approximations for x <= 8, asymptotic series up to 110 and
// the skin-effect limit beyond.
cd wire_internal_impedance(double sigl, double rolam) {
  const cd j1(0.0, 1.0);
  const double tpcmu = 2.368705e+3, cmotp = 60.00;
  const double x = std::sqrt(tpcmu * sigl) * rolam;
  if (x > 110.0) {
    const cd br1(0.70710678, -0.70710678);
    return j1 * std::sqrt(cmotp / sigl) * br1 / rolam;
  }
  if (x > 8.0) {
    const cd c1(6.0e-7, 1.9e-6), c2(-3.4e-6, 5.1e-6), c3(-2.52e-5, 0.0), c4(-9.06e-5, -9.01e-5),
        c5(0., -9.765e-4), c6(.0110486, -.0110485), c7(0., -.3926991), c8(1.6e-6, -3.2e-6), c9(1.17e-5, -2.4e-6),
        c10(3.46e-5, 3.38e-5), c11(5.0e-7, 2.452e-4), c12(-1.3813e-3, 1.3811e-3), c13(-6.25001e-2, -1.0e-7),
        c14(.7071068, .7071068);
    auto th = [&](double d) { return (((((c1 * d + c2) * d + c3) * d + c4) * d + c5) * d + c6) * d + c7; };
    auto ph = [&](double d) { return (((((c8 * d + c9) * d + c10) * d + c11) * d + c12) * d + c13) * d + c14; };
    const cd f = std::sqrt(kPi * 0.5 / x) * std::exp(-c14 * x + th(-8. / x));
    const cd g = std::exp(c14 * x + th(8. / x)) / std::sqrt(kTwoPi * x);
    cd br2 = j1 * f / kPi;
    cd br1 = g + br2;
    br2 = g * ph(8.0 / x) - br2 * ph(-8.0 / x);
    br1 = br1 / br2;
    return j1 * std::sqrt(cmotp / sigl) * br1 / rolam;
  }
  const double x8 = x / 8.0, y = x8 * x8, s = y * y;
  double ber = ((((((-9.01e-6 * s + 1.22552e-3) * s - .08349609) * s + 2.6419140) * s - 32.363456) * s + 113.77778) * s -
                64.) * s + 1.;
  double bei = ((((((1.1346e-4 * s - .01103667) * s + .52185615) * s - 10.567658) * s + 72.817777) * s - 113.77778) * s +
                16.) * y;
  cd br1(ber, bei);
  ber = (((((((-3.94e-6 * s + 4.5957e-4) * s - 0.02609253) * s + 0.66047849) * s - 6.0681481) * s + 14.222222) * s -
          4.0) * y) * x;
  bei = ((((((4.609e-5 * s - 3.79386e-3) * s + .14677204) * s - 2.3116751) * s + 11.377778) * s - 10.666667) * s + .5) *
        x;
  const cd br2(ber, bei);
  br1 = br1 / br2;
  return j1 * std::sqrt(cmotp / sigl) * br1 / rolam;
}
}  // namespace

// load, src/nec_context.cpp:1861-2072: lambda x impedance per unit length of
// every loaded segment at the current scaling (lengths in wavelengths).
void Context::load() {
  const int64_t n = geo_.n;
  zarray.assign(n, cd(0, 0));
  if (ldtyp.empty()) {
    zarray.clear();
    return;
  }
  const cd tpcj(0.0, 1.883698955e+9);
  const double lam = wavelength_;
  for (size_t k = 0; k < ldtyp.size(); k++) {
    if (ldtyp[k] > 5 || ldtyp[k] < 0) fail("IMPROPER LOAD TYPE CHOSEN, REQUESTED TYPE IS ", ldtyp[k]);
    const int tags = ldtag[k];
    int64_t l1 = 1, l2 = n;
    int ichk = 0;
    if (tags == 0 && (ldtagf[k] != 0 || ldtagt[k] != 0)) {
      l1 = ldtagf[k];
      l2 = ldtagt[k];
    }
    for (int64_t i = l1 - 1; i < l2 && i < n; i++) {
      if (i < 0) continue;
      if (tags != 0) {
        if (tags != geo_.tags[i]) continue;
        if (ldtagf[k] != 0) {
          ichk++;
          if (ichk < ldtagf[k] || ichk > ldtagt[k]) continue;
        } else {
          ichk = 1;
        }
      } else {
        ichk = 1;
      }
      const double sl = geo_.length[i];
      cd zt;
      switch (ldtyp[k]) {
        case 0:  // series RLC
          zt = zlr[k] / sl + tpcj * zli[k] / (sl * lam);
          if (std::fabs(zlc[k]) > 1.0e-20) zt += lam / (tpcj * sl * zlc[k]);
          break;
        case 1:  // parallel RLC
          zt = tpcj * sl * zlc[k] / lam;
          if (std::fabs(zli[k]) > 1.0e-20) zt += sl * lam / (tpcj * zli[k]);
          if (std::fabs(zlr[k]) > 1.0e-20) zt += sl / zlr[k];
          zt = 1. / zt;
          break;
        case 2:  // series RLC per metre
          zt = zlr[k] * lam + tpcj * zli[k];
          if (std::fabs(zlc[k]) > 1.0e-20) zt += 1. / (tpcj * sl * sl * zlc[k]);
          break;
        case 3:  // parallel RLC per metre
          zt = tpcj * sl * sl * zlc[k];
          if (std::fabs(zli[k]) > 1.0e-20) zt += 1. / (tpcj * zli[k]);
          if (std::fabs(zlr[k]) > 1.0e-20) zt += 1. / (zlr[k] * lam);
          zt = 1. / zt;
          break;
        case 4:  // fixed impedance
          zt = cd(zlr[k], zli[k]) / sl;
          break;
        default:  // wire conductivity
          zt = wire_internal_impedance(zlr[k] * lam, geo_.radius[i]);
      }
      zarray[i] += zt;
    }
    if (ichk == 0) fail("LOADING DATA CARD ERROR, NO SEGMENT HAS AN ITAG = ", tags);
  }
}

// compute_structure_power_loss, src/nec_context.cpp:1423-1441
double Context::compute_structure_power_loss() const {
  double loss = 0.0;
  for (size_t i = 0; i < zarray.size(); i++)
    if (std::fabs(zarray[i].real()) >= 1.e-20) {
      const double cmag = std::abs(solution[i] * wavelength_);
      loss += 0.5 * cmag * cmag * zarray[i].real() * geo_.length[i];
    }
  return loss;
}

void Context::gn_card(int itmp1, int itmp2, double t1, double t2, double t3,
                      double t4, double t5, double t6) {
  (void)t3;
  (void)t4;
  (void)t5;
  (void)t6;
  if (itmp1 == -1) {
    ksymp = 1;
    nradl = 0;
    iperf = 0;
  } else {
    if (itmp1 < 0 || itmp1 > 2) fail("GN: unknown ground type ", itmp1);
    iperf = itmp1;
    nradl = itmp2;
    ksymp = 2;
    epsr = t1;
    sig = t2;
    if (nradl != 0) {
      if (iperf == 2)
        fail("RADIAL WIRE G.S. APPROXIMATION MAY NOT BE USED WITH SOMMERFELD GROUND OPTION");
      fail("GN: radial-wire ground screen is not part of the B200 hot path");
    }
    if (iperf == 0) {
      if (epsr == 0.0) fail("GROUND DIELECTRIC CONSTANT IS ZERO");
      if (sig == 0.0) fail("GROUND CONDUCTIVITY IS ZERO");
    }
  }
  iflow = 4;
  reset_to_structure_loading();
}

// ex_card, src/nec_context.cpp:521-608
void Context::ex_card(int type, int i2, int i3, int i4, double f1, double f2,
                      double f3, double f4, double f5, double f6) {
  if (!geo_.completed) fail("EX card before geometry_complete");
  if (type < 0 || type > 5) fail("EX: unknown excitation type ", type);
  if (type == 5) fail("EX 5 (voltage discontinuity source) is not part of the B200 hot path");
  if (iflow != 5) {
    src_seg.clear();
    src_volt.clear();
    iped = 0;
    iflow = 5;
    reset_to_excitation_setup();
  }
  masym = i4 / 10;
  ex_type = type;
  if (type == 0) {
    ntsol = 0;
    int64_t seg = geo_.segment_number(i2, i3);
    if (seg > geo_.n)
      fail("CHECK DATA, PARAMETER SPECIFYING EXCITATION SOURCE SEGMENT [", seg, "] IS TOO LARGE");
    cd v(f1, f2);
    if (std::abs(v) < 1.e-20) v = cd(1.0, 0.0);
    src_seg.push_back(seg);
    src_volt.push_back(v);
    iped = i4 - masym * 10;
    zpnorm = f3;
    if (iped == 1 && zpnorm > 0.0) iped = 2;
    return;
  }
  nthi = i2;
  nphi = i3;
  xpr1 = f1;
  xpr2 = f2;
  xpr3 = f3;
  xpr4 = f4;
  xpr5 = f5;
  xpr6 = f6;
  src_seg.clear();
  src_volt.clear();
  thetis = xpr1;
  phiss = xpr2;
}

// xq_card, src/nec_context.cpp:709-743
void Context::xq_card(int mode) {
  if ((iflow == 10 && mode == 0) || (nfrq == 1 && mode == 0 && iflow > 7)) return;
  if (mode == 0) {
    iflow = (iflow > 7) ? 11 : 7;
  } else {
    ifar = 0;
    rfld = 0.;
    ipd = 0;
    iavp = 0;
    rp_norm = 0;
    rp_fmt = 0;
    nth = 91;
    nph = 1;
    thets = 0.0;
    phis = 0.0;
    dth = 1.0;
    dph = 0.0;
    if (mode == 2) phis = 90.0;
    if (mode == 3) {
      nph = 2;
      dph = 90.0;
    }
  }
  simulate(true);
}

// rp_card, src/nec_context.cpp:828-869
void Context::rp_card(int mode, int n_theta, int n_phi, int fmt, int norm, int d,
                      int a, double th0, double ph0, double in_dth, double in_dph,
                      double radial, double gain_norm) {
  if (mode != 0) fail("RP mode ", mode, " (ground-wave / cliff patterns) is not part of the B200 hot path");
  ifar = mode;
  nth = n_theta == 0 ? 1 : n_theta;
  nph = n_phi == 0 ? 1 : n_phi;
  rp_fmt = fmt != 0 ? 1 : 0;
  rp_norm = norm;
  ipd = d != 0 ? 1 : 0;
  iavp = a;
  if (nth < 2 || nph < 2 || ifar == 1) iavp = 0;
  thets = th0;
  phis = ph0;
  dth = in_dth;
  dph = in_dph;
  rfld = radial;
  gnor = gain_norm;
  iflow = 10;
  simulate(true);
}

void Context::kh_card(double r) {
  rkh = r;
  reset_to_structure_loading();
  iflow = 1;
}

void Context::ek_card(int flag) {
  use_exk = (-1 != flag);
  reset_to_structure_loading();
  iflow = 1;
}

void Context::pt_card(int a, int b, int c, int d) {
  iptflg = a;
  iptag = b;
  iptagf = c;
  iptagt = d;
  if (c == 0 && iptflg != -1) iptflg = -2;
  if (d == 0) iptagt = iptagf;
}

void Context::pq_card(int a, int b, int c, int d) {
  iptflq = a;
  iptaq = b;
  iptaqf = c;
  iptaqt = d;
  if (c == 0 && iptflq != -1) iptflq = -2;
  if (d == 0) iptaqt = iptaqf;
}

void Context::medium_parameters(double permittivity, double permeability) {
  medium().permittivity = permittivity;
  medium().permeability = permeability;
}

// simulate, src/nec_context.cpp:1031-1160.  The processing state the call
// starts from decides how much is recomputed; for every frequency of an FR
// sweep the structure is rescaled, refilled and refactored.
void Context::simulate(bool far_field_flag) {
  if (!geo_.completed) fail("simulation requested before geometry_complete");
  const int igox = (far_field_flag && state_ == NEAR) ? FAR : state_;
  int mhz = 1;
  bool in_freq_loop = false;
  do {
    if (igox <= MEM) {
      if (!in_freq_loop) {
        mhz = 1;
        in_freq_loop = true;
      }
      if (mhz != 1) {
        if (ifrq == 1)
          freq_mhz *= delfrq;
        else
          freq_mhz += delfrq;
      }
      wavelength_ = wavelength_of(1.0e6 * freq_mhz);
      geo_.frequency_scale(freq_mhz);
      state_ = STRUCT;
    }
    if (igox <= STRUCT) {
      structure_loading();
      state_ = EXSETUP;
    }
    if (igox <= EXSETUP) {
      nthic = 1;
      nphic = 1;
      inc = 1;
    }
    int ret = excitation_loop(igox, mhz);
    if (ret == FREQ_CONT) continue;
    if (ret == CARD_CONT) return;
    nphic = 1;
    xpr2 = phiss;
    if (mhz == nfrq) ifar = -1;
    if (nfrq == 1) return;
    nfrq = 1;
    mhz = 1;
  } while (++mhz <= nfrq);
}

// excitation_loop, src/nec_context.cpp:1793-1857
int Context::excitation_loop(int state_in, int mhz) {
  while (true) {
    if (state_in < EXLOOP) {
      int ret = excitation_inner(mhz);
      if (ret == INNER_CONT) continue;
      if (ret != PHASE_DONE) return ret;
    }
    if (state_in < NEAR) state_ = NEAR;
    // near fields, excitation_compute_near_field (1741-1758)
    if (state_in != FAR && m_near != -1) {
      if (nrx * nry * nrz != 0) nfpat();
      if (mhz == nfrq) m_near = -1;
      if (nfrq == 1) return CARD_CONT;
    }
    far_field();
    if (ex_type == 0 || ex_type == 4 || ex_type == 5) {
      if (mhz == nfrq) ifar = -1;
      if (nfrq != 1) return FREQ_CONT;
      return CARD_CONT;
    }
    nthic++;
    inc++;
    xpr1 += xpr4;
    if (nthic <= nthi) continue;
    nthic = 1;
    xpr1 = thetis;
    xpr2 += xpr5;
    nphic++;
    if (nphic > nphi) {
      if (nfrq != 1) return FREQ_CONT;
      return PRINT_NORM;
    }
  }
}

// excitation_process_inner, src/nec_context.cpp:1622-1738 (no coupling).
int Context::excitation_inner(int mhz) {
  (void)mhz;
  network_lengths();
  network_solve();
  ntsol = 1;
  if (iptflg < -2 || iptflg > 3) iptflg = -1;
  if (iptflq < -2 || iptflq > 0) iptflq = -1;
  if (ex_type != 1 && ex_type != 2 && ex_type != 3 && (iptflg == 2 || iptflg == 3)) iptflg = -1;
  structure_power_loss = compute_structure_power_loss();
  if (ex_type == 0 || ex_type == 5) {
    PowerBudget b;
    b.seq = next_seq();
    b.freq_hz = freq_mhz * 1.0e6;
    b.input = input_power;
    b.structure_loss = structure_power_loss;
    b.network_loss = network_power_loss;
    b.radiated = input_power - network_power_loss - structure_power_loss;
    b.efficiency = 100.0 * b.radiated / input_power;
    budgets.push_back(b);
  }
  if (iptflg != -1 || iptflq != -1) {
    if ((iptflg < 1 || iptflg == 3 || ((iptflg == 1 || iptflg == 2) && inc <= 1)) ||
        (iptflg == -1 && iptflq != -1)) {
      if (iptflg != 3) {
        StructureCurrents sc;
        sc.freq_hz = freq_mhz * 1.0e6;
        sc.current.resize(geo_.n);
        for (int64_t i = 0; i < geo_.n; i++) sc.current[i] = solution[i] * wavelength_;
        currents.push_back(std::move(sc));
      }
    }
  }
  state_ = EXLOOP;
  if (iflow == 7) {
    if (ex_type >= 1 && ex_type <= 3) {
      nthic++;
      inc++;
      xpr1 += xpr4;
      if (nthic <= nthi) return INNER_CONT;
      nthic = 1;
      xpr1 = thetis;
      xpr2 = xpr2 + xpr5;
      nphic++;
      if (nphic <= nphi) return INNER_CONT;
      return PRINT_NORM;
    }
    if (nfrq != 1) return FREQ_CONT;
    return CARD_CONT;
  }
  return PHASE_DONE;
}

// nec_ground::calculate_antenna_environment, src/nec_ground.cpp:177-219
void Context::antenna_environment() {
  if (ksymp != 2) return;
  frati = cd(1.0, 0.0);
  if (iperf == 1) return;
  double lambda = wavelength_of(freq_mhz * 1.0e6);
  if (sig < 0.) sig = -sig / (impedance_over_2pi() * lambda);
  epsc = cd(epsr, -sig * lambda * impedance_over_2pi());
  zrati = 1.0 / std::sqrt(epsc);
  if (iperf == 2) frati = (epsc - 1.0) / (epsc + 1.0);
}

void Context::prepare_structure(double freq) {
  if (!geo_.completed) fail("geometry not complete");
  freq_mhz = freq;
  wavelength_ = wavelength_of(1.0e6 * freq_mhz);
  geo_.frequency_scale(freq_mhz);
  build_tables();
  load();
}

// Ground environment, basis tables (trio per source segment) and the
// extended-kernel end flags at the current scaling.
void Context::build_tables() {
  antenna_environment();
  const int64_t n = geo_.n;
  geo_.prepare_basis();

  std::vector<int32_t>& tptr = tables.tptr;
  std::vector<int32_t>& tbasis = tables.tbasis;
  std::vector<double>&ta = tables.ta, &tb = tables.tb, &tc = tables.tc;
  tptr.assign(n + 1, 0);
  tbasis.clear();
  ta.clear();
  tb.clear();
  tc.clear();
  tbasis.reserve(3 * n);
  ta.reserve(3 * n);
  tb.reserve(3 * n);
  tc.reserve(3 * n);
  std::vector<BasisEntry> entries;
  tptr[0] = 0;
  for (int64_t j = 0; j < n; j++) {
    geo_.trio((int)(j + 1), entries);
    for (auto& e : entries) {
      tbasis.push_back(e.basis - 1);
      ta.push_back(e.a);
      tb.push_back(e.b);
      tc.push_back(e.c);
    }
    tptr[j + 1] = (int32_t)tbasis.size();
  }

  // extended thin-wire kernel end flags, cmww src/nec_context.cpp:2533-2594
  std::vector<int32_t>& ind1 = tables.ind1;
  std::vector<int32_t>& ind2 = tables.ind2;
  ind1.assign(n, 0);
  ind2.assign(n, 0);
  if (use_exk) {
    for (int64_t jj = 0; jj < n; jj++) {
      const int jx = (int)jj + 1;
      const double cabj = geo_.cab[jj], sabj = geo_.sab[jj];
      int ipr = geo_.icon1[jj];
      int i1 = 2;
      int iprx = std::abs(ipr) - 1;
      if (ipr > kPatchConnection)
        i1 = 0;
      else if (ipr == 0)
        i1 = 1;
      else if (ipr == jx && cabj * cabj + sabj * sabj <= 1.e-8)
        i1 = 0;
      else if (ipr > 0 && geo_.icon2[iprx] == jx)
        i1 = geo_.test_ek_approximation((int)jj, ipr - 1);
      else if (ipr < 0 && geo_.icon1[iprx] == -jx)
        i1 = geo_.test_ek_approximation((int)jj, -ipr - 1);
      ind1[jj] = i1;

      ipr = geo_.icon2[jj];
      int i2;
      if (ipr > kPatchConnection)
        i2 = 2;
      else if (ipr == 0)
        i2 = 1;
      else if (ipr < 0) {
        int ix = -ipr - 1;
        i2 = (-geo_.icon2[ix] != jx) ? 2 : geo_.test_ek_approximation((int)jj, ix);
      } else if (ipr != jx) {
        int ix = ipr - 1;
        i2 = (geo_.icon1[ix] != jx) ? 2 : geo_.test_ek_approximation((int)jj, ix);
      } else {
        i2 = (cabj * cabj + sabj * sabj > 1.e-8) ? 2 : 0;
      }
      ind2[jj] = i2;
    }
  }
  if (ksymp != 2)
    tables.ground = NECGPU_GROUND_NONE;
  else if (iperf == 1)
    tables.ground = NECGPU_GROUND_PERFECT;
  else if (iperf == 0)
    tables.ground = NECGPU_GROUND_REFLECTION;
  else
    tables.ground = NECGPU_GROUND_SOMMERFELD;
  tables.zr_re = zrati.real();
  tables.zr_im = zrati.imag();
  tables.fr_re = frati.real();
  tables.fr_im = frati.imag();
  tables.eta = impedance();
  const bool finite = ksymp == 2 && iperf != 1;
  tables.eps_re = finite ? epsc.real() : 0.0;
  tables.eps_im = finite ? epsc.imag() : 0.0;
  tables.rkh = rkh;
  tables.use_exk = use_exk ? 1 : 0;
}

// structure_segment_loading, src/nec_context.cpp:1523-1558: ground
// environment and tables, then fill and factor on the GPU.
necgpu_structure Context::structure_view() const {
  const int64_t n = geo_.n;
  necgpu_structure s{};
  s.n = n;
  s.x = geo_.x.data();
  s.y = geo_.y.data();
  s.z = geo_.z.data();
  s.length = geo_.length.data();
  s.radius = geo_.radius.data();
  s.cab = geo_.cab.data();
  s.sab = geo_.sab.data();
  s.salp = geo_.salp.data();
  s.trio_ptr = tables.tptr.data();
  s.trio_basis = tables.tbasis.data();
  s.trio_a = tables.ta.data();
  s.trio_b = tables.tb.data();
  s.trio_c = tables.tc.data();
  s.ek_ind1 = tables.ind1.data();
  s.ek_ind2 = tables.ind2.data();
  s.rkh = tables.rkh;
  s.use_exk = tables.use_exk;
  s.ground = tables.ground;
  s.zrati_re = tables.zr_re;
  s.zrati_im = tables.zr_im;
  s.frati_re = tables.fr_re;
  s.frati_im = tables.fr_im;
  s.eta = tables.eta;
  return s;
}

void Context::structure_loading() {
  ntsol = 0;
  build_tables();
  load();
  const necgpu_structure s = structure_view();
  necgpu_engine* e = engine();
  check(e, necgpu_set_structure(e, &s));
  check(e, necgpu_set_loads(e, zarray.empty() ? nullptr : reinterpret_cast<const double*>(zarray.data())));
  // Sommerfeld tables of this frequency (calculate_antenna_environment,
  // src/nec_ground.cpp:204-209)
  if (tables.ground == NECGPU_GROUND_SOMMERFELD) check(e, necgpu_set_sommerfeld(e, tables.eps_re, tables.eps_im));
  check(e, necgpu_set_fill_precision(e, precision_));
  check(e, necgpu_fill(e));
  check(e, necgpu_factor(e, precision_));
  have_factor_ = true;
}

// etmns and its helpers, src/nec_context.cpp:3193-3550 (wires only).
void Context::build_rhs(std::vector<cd>& e) {
  const int64_t n = geo_.n;
  e.assign(n, cd(0, 0));
  double p1 = 0, p2 = 0, p3 = 0, p4 = 0, p5 = 0, p6 = 0;
  if (ex_type != 0 && ex_type != 5) {
    p5 = degrees_to_rad(xpr5);
    p4 = degrees_to_rad(xpr4);
    if (ex_type == 4) {
      p1 = xpr1 / wavelength_;
      p2 = xpr2 / wavelength_;
      p3 = xpr3 / wavelength_;
      p6 = xpr6 / (wavelength_ * wavelength_);
    } else {
      p1 = degrees_to_rad(xpr1);
      p2 = degrees_to_rad(xpr2);
      p3 = degrees_to_rad(xpr3);
      p6 = xpr6;
    }
  }
  const double amp = (xpr7 != 0.0) ? xpr7 : 1.0;
  const auto& g = geo_;

  if (ex_type == 0) {
    for (size_t k = 0; k < src_seg.size(); k++) {
      int64_t s = src_seg[k] - 1;
      e[s] = -src_volt[k] / (g.length[s] * wavelength_);
    }
    return;
  }
  if (ex_type == 4) {  // elementary current source, 3387-3486
    double cosp4 = std::cos(p4);
    double wx = cosp4 * std::cos(p5), wy = cosp4 * std::sin(p5), wz = std::sin(p4);
    double ds = p6 * impedance_over_2pi();
    for (int64_t i = 0; i < n; i++) {
      double pxl = g.x[i] - p1, pyl = g.y[i] - p2, pzl = g.z[i] - p3;
      double rs = pxl * pxl + pyl * pyl + pzl * pzl;
      if (rs < 1.0e-30) continue;
      double r = std::sqrt(rs);
      pxl = pxl / r;
      pyl = pyl / r;
      pzl = pzl / r;
      double cth = pxl * wx + pyl * wy + pzl * wz;
      double sth = std::sqrt(1.0 - cth * cth);
      double qx = pxl - wx * cth, qy = pyl - wy * cth, qz = pzl - wz * cth;
      double arg = std::sqrt(qx * qx + qy * qy + qz * qz);
      if (arg >= 1.e-30) {
        qx = qx / arg;
        qy = qy / arg;
        qz = qz / arg;
      } else {
        qx = 1.0;
        qy = 0.0;
        qz = 0.0;
      }
      arg = kTwoPi * r;
      cd tt1(std::cos(arg), -std::sin(arg));
      cd tt2 = cd(1.0, -1.0 / arg) / rs;
      cd er = ds * tt1 * tt2 * cth;
      cd et = 0.5 * ds * tt1 * (cd(0.0, 1.0) * kTwoPi / r + tt2) * sth;
      cd ezh = er * cth - et * sth;
      cd erh = er * sth + et * cth;
      cd cx = ezh * wx + erh * qx, cy = ezh * wy + erh * qy, cz = ezh * wz + erh * qz;
      e[i] = -(cx * g.cab[i] + cy * g.sab[i] + cz * g.salp[i]);
    }
    return;
  }
  // plane waves, 3505-3550
  double cth = std::cos(p1), sth = std::sin(p1);
  double cph = std::cos(p2), sph = std::sin(p2);
  double cet = std::cos(p3), set = std::sin(p3);
  double pxl = cth * cph * cet - sph * set;
  double pyl = cth * sph * cet + cph * set;
  double pzl = -sth * cet;
  double wx = -sth * cph, wy = -sth * sph, wz = -cth;
  double qx = wy * pzl - wz * pyl;
  double qy = wz * pxl - wx * pzl;
  double qz = wx * pyl - wy * pxl;
  cd rrv, rrh;
  if (ksymp == 2) {
    if (iperf == 1) {
      rrv = -cd(1.0, 0.0);
      rrh = -cd(1.0, 0.0);
    } else {
      rrv = std::sqrt(1.0 - zrati * zrati * sth * sth);
      rrh = zrati * cth;
      rrh = (rrh - rrv) / (rrh + rrv);
      rrv = zrati * rrv;
      rrv = -(cth - rrv) / (cth + rrv);
    }
  }
  if (ex_type == 1) {  // 3213-3291
    for (int64_t i = 0; i < n; i++) {
      double arg = -kTwoPi * (wx * g.x[i] + wy * g.y[i] + wz * g.z[i]);
      cd ea(std::cos(arg), std::sin(arg));
      e[i] = -(pxl * g.cab[i] + pyl * g.sab[i] + pzl * g.salp[i]) * ea * amp;
    }
    if (ksymp == 2) {
      cd tt1 = (pyl * cph - pxl * sph) * (rrh - rrv);
      cd cx = rrv * pxl - tt1 * sph;
      cd cy = rrv * pyl + tt1 * cph;
      cd cz = -rrv * pzl;
      for (int64_t i = 0; i < n; i++) {
        double arg = -kTwoPi * (wx * g.x[i] + wy * g.y[i] - wz * g.z[i]);
        cd ea(std::cos(arg), std::sin(arg));
        e[i] -= (cx * g.cab[i] + cy * g.sab[i] + cz * g.salp[i]) * ea * amp;
      }
    }
    return;
  }
  // elliptic, 3294-3385
  cd tt1 = -(cd(0.0, 1.0)) * p6;
  if (ex_type == 3) tt1 = -tt1;
  cd cx = pxl + tt1 * qx, cy = pyl + tt1 * qy, cz = pzl + tt1 * qz;
  for (int64_t i = 0; i < n; i++) {
    double arg = -kTwoPi * (wx * g.x[i] + wy * g.y[i] + wz * g.z[i]);
    cd ea(std::cos(arg), std::sin(arg));
    e[i] = -(cx * g.cab[i] + cy * g.sab[i] + cz * g.salp[i]) * ea * amp;
  }
  if (ksymp == 2) {
    cd tt2 = (cy * cph - cx * sph) * (rrh - rrv);
    cd ccx = rrv * cx - tt2 * sph;
    cd ccy = rrv * cy + tt2 * cph;
    cd ccz = -rrv * cz;
    for (int64_t i = 0; i < n; i++) {
      double arg = -kTwoPi * (wx * g.x[i] + wy * g.y[i] - wz * g.z[i]);
      cd ea(std::cos(arg), std::sin(arg));
      e[i] -= (ccx * g.cab[i] + ccy * g.sab[i] + ccz * g.salp[i]) * ea * amp;
    }
  }
}

// netwk without networks (src/nec_context.cpp:4494-5065): solve, currents,
// antenna input parameters of the voltage sources.
// One structure solve on the held factors: segment-centre currents into
// `solution`, current coefficients into `abc` (the reference's solves +
// get_current_coefficients).  A mixed solve whose refinement fails
// refactors the intact FP64 matrix and solves again.
void Context::solve_structure(const std::vector<cd>& rhs) {
  const int64_t n = geo_.n;
  solution.assign(n, cd(0, 0));
  abc.assign(6 * n, 0.0);
  necgpu_engine* e = engine();
  int rc = necgpu_solve(e, reinterpret_cast<const double*>(rhs.data()), reinterpret_cast<double*>(solution.data()),
                        abc.data());
  if (rc == NECGPU_ERR_REFINE && precision_ == NECGPU_MIXED) {
    check(e, necgpu_factor(e, NECGPU_FP64));
    rc = necgpu_solve(e, reinterpret_cast<const double*>(rhs.data()), reinterpret_cast<double*>(solution.data()),
                      abc.data());
  }
  check(e, rc);
  necgpu_stats st{};
  necgpu_get_stats(e, &st);
  last_refine_residual = st.refine_residual;
  last_refine_iters = st.refine_iters;
}

namespace {
// Dense LU with partial pivoting of the small network matrix (row-major,
// n x n) and the solve on it; stands in for lu_decompose / solve
// (src/matrix_algebra.cpp:217-307) on the network equations.
void small_lu(int n, std::vector<cd>& a, std::vector<int>& piv) {
  piv.resize(n);
  for (int k = 0; k < n; k++) {
    int p = k;
    for (int i = k + 1; i < n; i++)
      if (std::abs(a[i * n + k]) > std::abs(a[p * n + k])) p = i;
    piv[k] = p;
    if (p != k)
      for (int j = 0; j < n; j++) std::swap(a[k * n + j], a[p * n + j]);
    const cd d = a[k * n + k];
    if (d == cd(0, 0)) fail("NETWORK EQUATIONS ARE SINGULAR");
    for (int i = k + 1; i < n; i++) {
      const cd l = a[i * n + k] / d;
      a[i * n + k] = l;
      for (int j = k + 1; j < n; j++) a[i * n + j] -= l * a[k * n + j];
    }
  }
}

void small_solve(int n, const std::vector<cd>& a, const std::vector<int>& piv, cd* b) {
  for (int k = 0; k < n; k++) std::swap(b[k], b[piv[k]]);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < i; j++) b[i] -= a[i * n + j] * b[j];
  for (int i = n - 1; i >= 0; i--) {
    for (int j = i + 1; j < n; j++) b[i] -= a[i * n + j] * b[j];
    b[i] /= a[i * n + i];
  }
}

double port_power(cd v, cd i) { return 0.5 * std::real(v * std::conj(i)); }
}  // namespace

// netwk, src/nec_context.cpp:4496-5066.  Without networks: one solve and
// the inputs of the voltage sources.  With networks: every network port
// that is not a source gets a unit-field solve on the held factors; its
// port currents plus the networks' short-circuit admittances form the
// network equations, which give the port voltages; those voltages are added
// to the applied field and the structure is solved once more.  As in the
// reference, the network equations exist only in the excitation pass that
// builds them (ntsol == 0); later passes on the same factors see none.
void Context::network_solve() {
  input_power = 0.0;
  network_power_loss = 0.0;
  std::vector<cd> einc;
  build_rhs(einc);
  const int nsrc = (int)src_seg.size();
  const int nnet = (ntsol == 0) ? (int)ntyp.size() : 0;
  const int ndimn = 2 * (int)ntyp.size() + nsrc;
  std::vector<cd> cmn, rhnx, rhnt, vsrc;
  std::vector<int64_t> nteqa, ntsca;
  int nteq = 0, ntsc = 0;
  if (ntyp.empty()) {
    solve_structure(einc);
  } else {
    cmn.assign((size_t)ndimn * ndimn, cd(0, 0));
    rhnx.assign(ndimn, cd(0, 0));
    rhnt.assign(ndimn, cd(0, 0));
    vsrc.assign(ndimn, cd(0, 0));
    nteqa.assign(ndimn, 0);
    ntsca.assign(ndimn, 0);
    // equation row of a port segment: sources count from the end
    auto port_row = [&](int64_t seg, int& isc) {
      isc = -1;
      for (int i = 0; i < nsrc; i++)
        if (src_seg[i] == seg) {
          isc = i;
          break;
        }
      if (isc < 0) {
        for (int i = 0; i < nteq; i++)
          if (nteqa[i] == seg) return i;
        nteqa[nteq] = seg;
        return nteq++;
      }
      for (int i = 0; i < ntsc; i++)
        if (ntsca[i] == seg) return ndimn - (i + 1);
      ntsca[ntsc] = seg;
      vsrc[ntsc] = src_volt[isc];
      ntsc++;
      return ndimn - ntsc;
    };
    // cmn[c + r * ndimn] is row r, column c of the network matrix
    for (int j = 0; j < nnet; j++) {
      cd y11, y12, y22;
      if (ntyp[j] <= 1) {
        y11 = cd(x11r[j], x11i[j]);
        y12 = cd(x12r[j], x12i[j]);
        y22 = cd(x22r[j], x22i[j]);
      } else {
        // lossless line of impedance x11r and length x11i (m) plus the shunt
        // admittances at its two ends; a crossed line flips y12
        const double bl = kTwoPi * x11i[j] / wavelength_;
        const double b12 = 1.0 / (x11r[j] * std::sin(bl));
        const double b11 = -b12 * std::cos(bl);
        y12 = cd(0.0, ntyp[j] == 2 ? b12 : -b12);
        y11 = cd(x12r[j], b11 + x12i[j]);
        y22 = cd(x22r[j], b11 + x22i[j]);
      }
      int isc1, isc2;
      const int irow1 = port_row(iseg1[j], isc1);
      const int irow2 = port_row(iseg2[j], isc2);
      if (isc1 == -1) {
        const double len = geo_.length[iseg1[j] - 1];
        cmn[irow1 + (size_t)irow1 * ndimn] -= y11 * len;
        cmn[irow1 + (size_t)irow2 * ndimn] -= y12 * len;
      } else {
        rhnx[irow1] += y11 * src_volt[isc1] / wavelength_;
        rhnx[irow2] += y12 * src_volt[isc1] / wavelength_;
      }
      if (isc2 == -1) {
        const double len = geo_.length[iseg2[j] - 1];
        cmn[irow2 + (size_t)irow2 * ndimn] -= y22 * len;
        cmn[irow2 + (size_t)irow1 * ndimn] -= y12 * len;
      } else {
        rhnx[irow1] += y12 * src_volt[isc2] / wavelength_;
        rhnx[irow2] += y22 * src_volt[isc2] / wavelength_;
      }
    }
    // structure admittance at the ports: one unit-field solve per port
    std::vector<cd> unit(geo_.n, cd(0, 0));
    for (int i = 0; i < nteq; i++) {
      unit[nteqa[i] - 1] = cd(1, 0);
      solve_structure(unit);
      unit[nteqa[i] - 1] = cd(0, 0);
      for (int j = 0; j < nteq; j++) cmn[i + (size_t)j * ndimn] += solution[nteqa[j] - 1];
    }
    std::vector<cd> a((size_t)nteq * nteq);
    for (int r = 0; r < nteq; r++)
      for (int c = 0; c < nteq; c++) a[(size_t)r * nteq + c] = cmn[c + (size_t)r * ndimn];
    std::vector<int> piv;
    small_lu(nteq, a, piv);
    // port voltages from the currents the applied field drives
    solve_structure(einc);
    for (int i = 0; i < nteq; i++) rhnt[i] = rhnx[i] + solution[nteqa[i] - 1];
    small_solve(nteq, a, piv, rhnt.data());
    for (int i = 0; i < nteq; i++) einc[nteqa[i] - 1] -= rhnt[i];
    if (nteq > 0) solve_structure(einc);
    for (int i = 0; i < nteq; i++) {
      const int64_t sidx = nteqa[i] - 1;
      network_power_loss -= port_power(rhnt[i] * geo_.length[sidx] * wavelength_, solution[sidx] * wavelength_);
    }
    for (int i = 0; i < ntsc; i++)
      network_power_loss -= port_power(vsrc[i], solution[ntsca[i] - 1] * wavelength_);
  }
  structure_power_loss = compute_structure_power_loss();

  if (src_seg.empty()) return;
  AntennaInput ai;
  ai.freq_hz = freq_mhz * 1.0e6;
  for (int k = 0; k < nsrc; k++) {
    int64_t s = src_seg[k] - 1;
    cd voltage = src_volt[k];
    cd current = solution[s] * wavelength_;
    bool network_loss = false;
    if (ntsc != 0) {
      // a source that is also a network port: add the current its networks draw
      int j = 0;
      while (j < ntsc && ntsca[j] != s + 1) j++;
      if (j == ntsc) fail("NETWORK DATA ERROR: SOURCE SEGMENT [", s + 1, "] NOT FOUND IN NETWORK TABLE");
      const int row = ndimn - (j + 1);
      cd temp = rhnx[row];
      for (int m = 0; m < nteq; m++) temp -= cmn[m + (size_t)row * ndimn] * rhnt[m];
      current = (solution[s] + temp) * wavelength_;
      network_loss = true;
    }
    cd admittance = current / voltage;
    cd imp = voltage / current;
    double power = port_power(voltage, current);
    if (network_loss) network_power_loss += power;
    input_power += power;
    ai.tag.push_back(geo_.tags[s]);
    ai.seg.push_back((int)(s + 1));
    ai.voltage.push_back(voltage);
    ai.current.push_back(current);
    ai.impedance.push_back(imp);
    ai.admittance.push_back(admittance);
    ai.power.push_back(power);
  }
  ai.seq = next_seq();
  inputs.push_back(std::move(ai));
}

// excitation_compute_far_field + nec_radiation_pattern::analyze,
// src/nec_context.cpp:1761-1790, src/nec_radiation_pattern.cpp:209-450.
// The direction grid is stepped exactly as the reference steps it; the field
// sum runs on the GPU; gains and polarisation are evaluated here.
void Context::far_field() {
  if (ifar == -1) return;
  const bool ground = (ksymp == 2);
  RadiationPattern rp;
  rp.freq_hz = freq_mhz * 1.0e6;
  rp.nth = nth;
  rp.nph = nph;
  rp.th0 = thets;
  rp.ph0 = phis;
  rp.dth = dth;
  rp.dph = dph;
  rp.ground = ground;
  rp.fmt = rp_fmt;
  rp.ipd = ipd;
  rp.range = rfld;
  rp.wavelength = wavelength_;
  const size_t cells = (size_t)nth * nph;
  rp.gain.assign(cells, 0.0);
  rp.gain_vert.assign(cells, 0.0);
  rp.gain_horiz.assign(cells, 0.0);
  rp.gain_tot.assign(cells, 0.0);
  rp.gain_rhcp.assign(cells, 0.0);
  rp.gain_lhcp.assign(cells, 0.0);
  rp.axial_ratio.assign(cells, 0.0);
  rp.tilt.assign(cells, 0.0);
  rp.avg_scale.assign(cells, 0.0);
  rp.sense.assign(cells, 0);
  rp.e_theta.assign(cells, cd(0, 0));
  rp.e_phi.assign(cells, cd(0, 0));

  double gcon, gcop;
  const double pinr_in = input_power, pnlr = network_power_loss;
  double pinr = pinr_in;
  if (ex_type == 0 || ex_type == 5) {
    gcop = wavelength_ * wavelength_ * 2.0 * kPi / (impedance() * pinr);
    double prad = pinr - structure_power_loss - pnlr;
    gcon = gcop;
    if (ipd != 0) gcon = gcon * pinr / prad;
  } else if (ex_type == 4) {
    pinr = 394.51 * xpr6 * xpr6 * wavelength_ * wavelength_;
    gcop = wavelength_ * wavelength_ * 2. * kPi / (impedance() * pinr);
    double prad = pinr - structure_power_loss - pnlr;
    gcon = gcop;
    if (ipd != 0) gcon = gcon * pinr / prad;
  } else {
    gcon = 4. * kPi / (1.0 + xpr6 * xpr6);
    gcop = gcon;
  }
  double exrm = 0., exra = 0.;
  if (rfld >= 1.0e-20) {
    exrm = 1. / rfld;
    exra = rfld / wavelength_;
    exra = -360. * (exra - std::floor(exra));
  }

  // direction list, stepped as in analyze (accumulated degrees)
  std::vector<double> tha_list, pha_list;
  std::vector<int> cell_list;
  {
    double phi = phis - dph;
    for (int kph = 0; kph < nph; kph++) {
      phi += dph;
      double pha = degrees_to_rad(phi);
      double thet = thets - dth;
      for (int kth = 0; kth < nth; kth++) {
        thet += dth;
        if (ground && thet > 90.01) continue;
        tha_list.push_back(degrees_to_rad(thet));
        pha_list.push_back(pha);
        cell_list.push_back(kth + kph * nth);
      }
    }
  }
  const int ndir = (int)tha_list.size();
  std::vector<cd> eth(ndir), eph(ndir);
  if (ndir > 0) {
    necgpu_engine* e = engine();
    check(e, necgpu_pattern(e, ndir, tha_list.data(), pha_list.data(),
                            reinterpret_cast<double*>(eth.data()),
                            reinterpret_cast<double*>(eph.data())));
  }

  if (ndir > 0 && (rp_norm < 0 || rp_norm > 5)) fail("Unknown Gain Normalization Encountered.");
  const double delta_phi_rad = degrees_to_rad(dph);
  const double tmp2 = 0.5 * degrees_to_rad(dth);
  // per-direction gains and polarisation over worker threads; the averaging
  // integral's terms are kept per direction and summed in direction order
  std::vector<double> pint_d(iavp != 0 ? ndir : 0);
  auto analyze = [&](int, int64_t d0, int64_t d1) {
    for (int64_t d = d0; d < d1; d++) {
      const int cell = cell_list[d];
      const int kth = cell % nth, kph = cell / nth;
      const double tha = tha_list[d];
      double ethm2 = std::norm(eth[d]);
      double ethm = std::sqrt(ethm2);
      double etha = rad_to_degrees(std::arg(eth[d]));
      double ephm2 = std::norm(eph[d]);
      double ephm = std::sqrt(ephm2);
      double epha = rad_to_degrees(std::arg(eph[d]));
      double tilta, emajr2, eminr2, axrat;
      int sense;
      if (ethm2 <= 1.0e-20 && ephm2 <= 1.0e-20) {
        tilta = 0.;
        emajr2 = 0.;
        eminr2 = 0.;
        axrat = 0.;
        sense = 3;
      } else {
        double dfaz = epha - etha;
        double dfaz2 = (epha >= 0.) ? dfaz - 360. : dfaz + 360.;
        if (std::fabs(dfaz) > std::fabs(dfaz2)) dfaz = dfaz2;
        double cdfaz = std::cos(degrees_to_rad(dfaz));
        double tstor1 = ethm2 - ephm2;
        double tstor2 = 2. * ephm * ethm * cdfaz;
        tilta = .5 * std::atan2(tstor2, tstor1);
        double stilta = std::sin(tilta);
        tstor1 = tstor1 * stilta * stilta;
        tstor2 = tstor2 * stilta * std::cos(tilta);
        emajr2 = -tstor1 + tstor2 + ethm2;
        eminr2 = tstor1 - tstor2 + ephm2;
        if (eminr2 < 0.) eminr2 = 0.;
        axrat = std::sqrt(eminr2 / emajr2);
        tilta = rad_to_degrees(tilta);
        if (axrat <= 1.0e-5)
          sense = 0;  // linear
        else if (dfaz <= 0.)
          sense = 1;  // right
        else
          sense = 2;  // left
      }
      double gnmj = db10(gcon * emajr2);
      double gnmn = db10(gcon * eminr2);
      double gnv = db10(gcon * ethm2);
      double gnh = db10(gcon * ephm2);
      double gtot = db10(gcon * (ethm2 + ephm2));
      double g;
      switch (rp_norm) {
        case 0: g = gtot; break;
        case 1: g = gnmj; break;
        case 2: g = gnmn; break;
        case 3: g = gnv; break;
        case 4: g = gnh; break;
        default: g = gtot; break;  // 5
      }
      rp.gain[cell] = g;
      if (iavp != 0) {
        double tstor1 = gcop * (ethm2 + ephm2);
        double tmp3 = tha - tmp2, tmp4 = tha + tmp2;
        if (kth == 0)
          tmp3 = tha;
        else if (kth == nth - 1)
          tmp4 = tha;
        double da = std::fabs(delta_phi_rad * (std::cos(tmp3) - std::cos(tmp4)));
        if (kph == 0 || kph == nph - 1) da *= .5;
        pint_d[d] = tstor1 * da;
        if (iavp == 2) continue;
      }
      if (rp_fmt != 1) {
        rp.gain_vert[cell] = gnmj;
        rp.gain_horiz[cell] = gnmn;
      } else {
        rp.gain_vert[cell] = gnv;
        rp.gain_horiz[cell] = gnh;
      }
      ethm *= wavelength_;
      ephm *= wavelength_;
      if (rfld >= 1.0e-20) {
        ethm = ethm * exrm;
        etha = etha + exra;
        ephm = ephm * exrm;
        epha = epha + exra;
      }
      rp.e_theta[cell] = std::polar(ethm, degrees_to_rad(etha));
      rp.e_phi[cell] = std::polar(ephm, degrees_to_rad(epha));
      rp.gain_tot[cell] = gtot;
      {
        double a = axrat;
        if (sense == 1) a = -a;
        double gain = from_db10(gtot);
        double lhcp_f = (1 + 2 * a + a * a) / (2 * (1 + a * a));
        double rhcp_f = (1 - 2 * a + a * a) / (2 * (1 + a * a));
        rp.gain_rhcp[cell] = db10(gain * rhcp_f);
        rp.gain_lhcp[cell] = db10(gain * lhcp_f);
      }
      rp.axial_ratio[cell] = axrat;
      rp.tilt[cell] = tilta;
      rp.sense[cell] = sense;
      rp.avg_scale[cell] = (std::sin(tha) * (nth - 1) / nth) + 1.0 / nth;
    }
  };
  parallel_chunks(ndir, host_workers(ndir, 512), analyze);
  double pint = 0.0;
  for (double v : pint_d) pint += v;
  if (iavp != 0) {
    double th0r = degrees_to_rad(thets);
    double th_range = degrees_to_rad(dth) * static_cast<double>(nth - 1);
    double ph_range = degrees_to_rad(dph) * static_cast<double>(nph - 1);
    double total = th0r + th_range;
    double solid = std::fabs(ph_range * (std::cos(th0r) - std::cos(total)));
    rp.average_power_gain = pint / solid;
    rp.average_power_solid_angle = solid / kPi;
  }
  rp.max_gain = *std::max_element(rp.gain.begin(), rp.gain.end());
  rp.seq = next_seq();
  patterns.push_back(std::move(rp));
}

// statistics of nec_radiation_pattern.h:246-320; matrices are walked row
// (theta) outer, column (phi) inner as the reference's loops do.
double RadiationPattern::stat_max(const std::vector<double>& v) const {
  return *std::max_element(v.begin(), v.end());
}
double RadiationPattern::stat_min(const std::vector<double>& v) const {
  return *std::min_element(v.begin(), v.end());
}
double RadiationPattern::stat_mean(const std::vector<double>& v) const {
  double sum = 0.0;
  for (int i = 0; i < nth; i++)
    for (int j = 0; j < nph; j++) sum += v[i + j * nth] * avg_scale[i + j * nth];
  int64_t len = (int64_t)nth * nph;
  return sum / (double(len * 2) / kPi);
}
double RadiationPattern::stat_sd(const std::vector<double>& v) const {
  double mean = stat_mean(v);
  double sum = 0.0;
  for (int i = 0; i < nth; i++)
    for (int j = 0; j < nph; j++) {
      double diff = v[i + j * nth] - mean;
      sum += diff * diff * avg_scale[i + j * nth];
    }
  int64_t len = (int64_t)nth * nph;
  return std::sqrt(sum / (double(len * 2) / kPi));
}

// Adjoint gradients.  Each output is built from three complex-linear
// functionals of the basis amplitudes x (Z x = e):
//   J = cur_f (feed current / wavelength), E_theta, E_phi = phi^T x,
// whose total derivative is
//   dPhi/dp = (d phi/dp)^T x + w^T (de/dp - (dZ/dp) x),   Z^T w = phi.
// The adjoint vectors w come from one transposed solve each on the held
// factors; w^T (dZ/dp) x from fills of the perturbed structures contracted
// on the fly; the explicit terms from the perturbed tables, right-hand side
// and far-field geometry.  Central differences of width 2 h_k resolve the
// parameter dependence of those explicit and contracted terms.
void Context::gradient(int nparam, Context* const* plus, Context* const* minus, const double* h,
                       double theta_deg, double phi_deg, double* value, double* grad) {
  if (nparam < 1 || !plus || !minus || !h || !value || !grad) fail("gradient: bad arguments");
  if (!have_factor_ || !eng_ || inputs.empty()) fail("gradient: run the forward solve (an XQ or RP card) first");
  if (src_seg.size() != 1) fail("gradient: exactly one voltage source is supported");
  if (precision_ != 1) fail("gradient: needs the mixed-precision path (nec_set_precision(ctx, 1))");
  if (!zarray.empty()) fail("gradient: loaded structures (LD cards) are not supported");
  if (!ntyp.empty()) fail("gradient: networks and transmission lines (NT/TL cards) are not supported");
  necgpu_engine* e = eng_;
  const int64_t n = geo_.n;
  const int64_t f = src_seg[0] - 1;
  const cd V = src_volt[0];
  const double lam = wavelength_;
  // forward quantities
  std::vector<cd> x(n);
  check(e, necgpu_copy_solution(e, reinterpret_cast<double*>(x.data())));
  const double th = degrees_to_rad(theta_deg), ph = degrees_to_rad(phi_deg);
  cd Et, Ep;
  check(e, necgpu_pattern(e, 1, &th, &ph, reinterpret_cast<double*>(&Et), reinterpret_cast<double*>(&Ep)));
  auto feed_current = [&](const Tables& t) {  // J = sum (a + c) x over the feed segment's bases
    cd J(0, 0);
    for (int32_t k = t.tptr[f]; k < t.tptr[f + 1]; k++) J += (t.ta[k] + t.tc[k]) * x[t.tbasis[k]];
    return J;
  };
  const cd J = solution[f];
  // adjoint right-hand sides: phi_J, phi_theta, phi_phi
  std::vector<cd> phis(3 * n, cd(0, 0)), w(3 * n);
  for (int32_t k = tables.tptr[f]; k < tables.tptr[f + 1]; k++) phis[tables.tbasis[k]] += tables.ta[k] + tables.tc[k];
  check(e, necgpu_pattern_weights(e, th, ph, reinterpret_cast<double*>(phis.data() + n),
                                  reinterpret_cast<double*>(phis.data() + 2 * n)));
  check(e, necgpu_adjoint_solve(e, 3, reinterpret_cast<const double*>(phis.data()), reinterpret_cast<double*>(w.data())));
  // perturbed structures at this frequency: tables, right-hand sides
  std::vector<necgpu_structure> structs;
  std::vector<std::vector<cd>> rhss;
  std::vector<cd> Jp;
  structs.reserve(2 * nparam);
  for (int k = 0; k < nparam; k++)
    for (int side = 0; side < 2; side++) {
      Context* c = side == 0 ? plus[k] : minus[k];
      if (!c) fail("gradient: missing perturbed context");
      c->prepare_structure(freq_mhz);
      if (c->geo_.n != n) fail("gradient: a perturbed structure has a different segment count");
      if (c->src_seg.size() != 1 || c->src_seg[0] != src_seg[0] || c->src_volt[0] != V)
        fail("gradient: a perturbed structure has a different excitation");
      structs.push_back(c->structure_view());
      rhss.emplace_back();
      c->rhs(rhss.back());
      Jp.push_back(feed_current(c->tables));
    }
  std::vector<cd> zx(2 * nparam * 3), efar(2 * nparam * 2);
  check(e, necgpu_perturbed_terms(e, 2 * nparam, structs.data(), 3, reinterpret_cast<const double*>(w.data()), th, ph,
                                  reinterpret_cast<double*>(zx.data()), reinterpret_cast<double*>(efar.data())));
  // outputs and their derivatives
  const cd zin = V / (J * lam);
  const double e2 = std::norm(Et) + std::norm(Ep);
  const double P = 0.5 * std::real(V * std::conj(J * lam));
  const double gcop = lam * lam * 2.0 * kPi / (impedance() * P);
  value[0] = zin.real();
  value[1] = zin.imag();
  value[2] = db10(gcop * e2);
  for (int k = 0; k < nparam; k++) {
    const int qp = 2 * k, qm = 2 * k + 1;
    const double inv2h = 1.0 / (2.0 * h[k]);
    cd wde[3] = {cd(0, 0), cd(0, 0), cd(0, 0)};
    for (int64_t i = 0; i < n; i++) {
      const cd de = rhss[qp][i] - rhss[qm][i];
      for (int a = 0; a < 3; a++) wde[a] += w[a * n + i] * de;
    }
    const cd explicit_[3] = {Jp[qp] - Jp[qm], efar[2 * qp] - efar[2 * qm], efar[2 * qp + 1] - efar[2 * qm + 1]};
    cd d[3];
    for (int a = 0; a < 3; a++) d[a] = (explicit_[a] + wde[a] - (zx[3 * qp + a] - zx[3 * qm + a])) * inv2h;
    const cd dzin = -zin * d[0] / J;
    const double dP = 0.5 * std::real(V * std::conj(d[0] * lam));
    const double dlng = 2.0 * std::real(std::conj(Et) * d[1] + std::conj(Ep) * d[2]) / e2 - dP / P;
    grad[3 * k] = dzin.real();
    grad[3 * k + 1] = dzin.imag();
    grad[3 * k + 2] = 10.0 / std::log(10.0) * dlng;
  }
}

}  // namespace necb
