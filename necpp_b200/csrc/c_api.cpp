// The NEC2++ C API (src/libnecpp.h, src/libNEC.cpp:27-282) over the B200
// context.  Errors are caught, their message kept in a process-global string
// and 1 returned, as NEC_ERROR_HANDLE does (src/libNEC.cpp:27-30).
#include <cstring>
#include <string>

#include "../../include/libnecpp.h"
#include "context.h"
#include "nec_constants.h"
#include "nec_error.h"

using necb::Context;

static std::string g_err;

#define NEC_TRY(body)                                        \
  do {                                                       \
    try {                                                    \
      body;                                                  \
    } catch (const std::exception& ex) {                     \
      g_err = ex.what();                                     \
      return 1;                                              \
    }                                                        \
    return 0;                                                \
  } while (0)

#define NEC_UNSUPPORTED(what) \
  NEC_TRY(necb::fail(what, " is not part of the B200 thin-wire hot path"))

extern "C" {

nec_context* nec_create(void) { return new Context(); }

long nec_delete(nec_context* c) { NEC_TRY(delete c); }

long nec_benchmark(void) {
  g_err = "nec_benchmark: the reference's benchmark decks fail its own overlap check";
  return 0;
}

const char* nec_error_message(void) { return g_err.c_str(); }

long nec_wire(nec_context* c, int tag, int nseg, double xw1, double yw1, double zw1,
              double xw2, double yw2, double zw2, double rad, double rdel, double rrad) {
  NEC_TRY(c->geometry().wire(tag, nseg, xw1, yw1, zw1, xw2, yw2, zw2, rad, rdel, rrad));
}

long nec_helix(nec_context* c, int tag, int nseg, double s, double hl, double a1, double b1,
               double a2, double b2, double rad) {
  NEC_TRY(c->geometry().helix(tag, nseg, s, hl, a1, b1, a2, b2, rad));
}

long nec_sp_card(nec_context*, int, double, double, double, double, double, double) {
  NEC_UNSUPPORTED("SP (surface patch)");
}
long nec_sc_card(nec_context*, int, double, double, double, double, double, double) {
  NEC_UNSUPPORTED("SC (surface patch)");
}

long nec_gm_card(nec_context* c, int itsi, int nrpt, double rox, double roy, double roz,
                 double xs, double ys, double zs, int its) {
  double roxd = necb::degrees_to_rad(rox);
  double royd = necb::degrees_to_rad(roy);
  double rozd = necb::degrees_to_rad(roz);
  NEC_TRY(c->geometry().move(roxd, royd, rozd, xs, ys, zs, its, nrpt, itsi));
}

long nec_gx_card(nec_context*, int, int) { NEC_UNSUPPORTED("GX (symmetry)"); }

long nec_geometry_complete(nec_context* c, int gpflag) { NEC_TRY(c->geometry_complete(gpflag)); }

long nec_medium_parameters(nec_context* c, double permittivity, double permeability) {
  NEC_TRY(c->medium_parameters(permittivity, permeability));
}

long nec_gn_card(nec_context* c, int iperf, int nradl, double epse, double sig, double t3,
                 double t4, double t5, double t6) {
  NEC_TRY(c->gn_card(iperf, nradl, epse, sig, t3, t4, t5, t6));
}

long nec_fr_card(nec_context* c, int ifrq, int nfrq, double f, double df) {
  NEC_TRY(c->fr_card(ifrq, nfrq, f, df));
}

long nec_ek_card(nec_context* c, int itmp1) { NEC_TRY(c->ek_card(itmp1)); }

long nec_ld_card(nec_context* c, int ldtyp, int ldtag, int ldtagf, int ldtagt, double tmp1, double tmp2,
                 double tmp3) {
  NEC_TRY(c->ld_card(ldtyp, ldtag, ldtagf, ldtagt, tmp1, tmp2, tmp3));
}

long nec_network_count(nec_context* c) { return c ? c->network_count() : -1; }

long nec_get_loads(nec_context* c, double* out) {
  if (!c || !out) return 1;
  const auto& z = c->loads();
  const int64_t n = c->geometry().n;
  for (int64_t i = 0; i < n; i++) {
    out[2 * i] = z.empty() ? 0.0 : z[i].real();
    out[2 * i + 1] = z.empty() ? 0.0 : z[i].imag();
  }
  return 0;
}

long nec_ex_card(nec_context* c, int extype, int i2, int i3, int i4, double t1, double t2,
                 double t3, double t4, double t5, double t6) {
  NEC_TRY(c->ex_card(extype, i2, i3, i4, t1, t2, t3, t4, t5, t6));
}

long nec_excitation_voltage(nec_context* c, int tag, int segment, double vr, double vi) {
  NEC_TRY(c->ex_card(0, tag, segment, 0, vr, vi, 0.0, 0.0, 0.0, 0.0));
}

long nec_excitation_current(nec_context* c, double x, double y, double z, double a,
                            double beta, double moment) {
  NEC_TRY(c->ex_card(4, 0, 0, 0, x, y, z, a, beta, moment));
}

long nec_excitation_planewave(nec_context* c, int n_theta, int n_phi, double theta,
                              double phi, double eta, double dtheta, double dphi,
                              double pol_ratio) {
  NEC_TRY(c->ex_card(1, n_theta, n_phi, 0, theta, phi, eta, dtheta, dphi, pol_ratio));
}

long nec_tl_card(nec_context* c, int itmp1, int itmp2, int itmp3, int itmp4, double tmp1, double tmp2,
                 double tmp3, double tmp4, double tmp5, double tmp6) {
  NEC_TRY(c->tl_card(itmp1, itmp2, itmp3, itmp4, tmp1, tmp2, tmp3, tmp4, tmp5, tmp6));
}
long nec_nt_card(nec_context* c, int itmp1, int itmp2, int itmp3, int itmp4, double tmp1, double tmp2,
                 double tmp3, double tmp4, double tmp5, double tmp6) {
  NEC_TRY(c->nt_card(itmp1, itmp2, itmp3, itmp4, tmp1, tmp2, tmp3, tmp4, tmp5, tmp6));
}

long nec_xq_card(nec_context* c, int itmp1) { NEC_TRY(c->xq_card(itmp1)); }

long nec_gd_card(nec_context*, double, double, double, double) {
  NEC_UNSUPPORTED("GD (cliff ground)");
}

long nec_rp_card(nec_context* c, int mode, int nth, int nph, int fmt, int norm, int d, int a,
                 double th0, double ph0, double dth, double dph, double rfld, double gnor) {
  NEC_TRY(c->rp_card(mode, nth, nph, fmt, norm, d, a, th0, ph0, dth, dph, rfld, gnor));
}

long nec_pt_card(nec_context* c, int a, int b, int cc, int d) { NEC_TRY(c->pt_card(a, b, cc, d)); }
long nec_pq_card(nec_context* c, int a, int b, int cc, int d) { NEC_TRY(c->pq_card(a, b, cc, d)); }

long nec_kh_card(nec_context* c, double r) { NEC_TRY(c->kh_card(r)); }

long nec_ne_card(nec_context* c, int itmp1, int itmp2, int itmp3, int itmp4, double tmp1, double tmp2,
                 double tmp3, double tmp4, double tmp5, double tmp6) {
  NEC_TRY(c->ne_nh_card(0, itmp1, itmp2, itmp3, itmp4, tmp1, tmp2, tmp3, tmp4, tmp5, tmp6));
}
long nec_nh_card(nec_context* c, int itmp1, int itmp2, int itmp3, int itmp4, double tmp1, double tmp2,
                 double tmp3, double tmp4, double tmp5, double tmp6) {
  NEC_TRY(c->ne_nh_card(1, itmp1, itmp2, itmp3, itmp4, tmp1, tmp2, tmp3, tmp4, tmp5, tmp6));
}

long nec_near_field(nec_context* c, int index, int* nfeh, double* xyz, double* fields) {
  if (!c || index < 0 || index >= (int)c->near_fields.size()) return -1;
  const necb::NearFieldPattern& p = c->near_fields[index];
  if (nfeh) *nfeh = p.nfeh;
  const size_t np = p.x.size();
  for (size_t i = 0; xyz && i < np; i++) {
    xyz[3 * i] = p.x[i];
    xyz[3 * i + 1] = p.y[i];
    xyz[3 * i + 2] = p.z[i];
  }
  for (size_t i = 0; fields && i < np; i++) {
    const necb::cd v[3] = {p.fx[i], p.fy[i], p.fz[i]};
    for (int k = 0; k < 3; k++) {
      fields[6 * i + 2 * k] = v[k].real();
      fields[6 * i + 2 * k + 1] = v[k].imag();
    }
  }
  return (long)np;
}
long nec_cp_card(nec_context*, int, int, int, int) { NEC_UNSUPPORTED("CP (coupling)"); }
long nec_pl_card(nec_context*, char*, int, int, int, int) { NEC_UNSUPPORTED("PL (plot file)"); }

// ---- accessors (src/nec_context.h:130-260) ----
static const necb::RadiationPattern* pattern_at(nec_context* c, int f) {
  if (!c || f < 0 || f >= (int)c->patterns.size()) return nullptr;
  return &c->patterns[f];
}

double nec_gain(nec_context* c, int f, int th, int ph) {
  auto* p = pattern_at(c, f);
  if (!p) return -999.0;
  if (th < 0 || th >= p->nth || ph < 0 || ph >= p->nph) return -999.0;
  return p->gain[th + ph * p->nth];
}

#define GAIN_STAT(name, field, stat)                 \
  double name(nec_context* c, int f) {               \
    auto* p = pattern_at(c, f);                      \
    if (!p) return -999.0;                           \
    return p->stat(p->field);                        \
  }
GAIN_STAT(nec_gain_max, gain_tot, stat_max)
GAIN_STAT(nec_gain_min, gain_tot, stat_min)
GAIN_STAT(nec_gain_mean, gain_tot, stat_mean)
GAIN_STAT(nec_gain_sd, gain_tot, stat_sd)
GAIN_STAT(nec_gain_rhcp_max, gain_rhcp, stat_max)
GAIN_STAT(nec_gain_rhcp_min, gain_rhcp, stat_min)
GAIN_STAT(nec_gain_rhcp_mean, gain_rhcp, stat_mean)
GAIN_STAT(nec_gain_rhcp_sd, gain_rhcp, stat_sd)
GAIN_STAT(nec_gain_lhcp_max, gain_lhcp, stat_max)
GAIN_STAT(nec_gain_lhcp_min, gain_lhcp, stat_min)
GAIN_STAT(nec_gain_lhcp_mean, gain_lhcp, stat_mean)
GAIN_STAT(nec_gain_lhcp_sd, gain_lhcp, stat_sd)

double nec_impedance_real_indexed(nec_context* c, int f, int feed) {
  if (!c || f < 0 || f >= (int)c->inputs.size()) return -999.0;
  auto& imp = c->inputs[f].impedance;
  if (feed < 0 || feed >= (int)imp.size()) return -999.0;
  return imp[feed].real();
}
double nec_impedance_imag_indexed(nec_context* c, int f, int feed) {
  if (!c || f < 0 || f >= (int)c->inputs.size()) return -999.0;
  auto& imp = c->inputs[f].impedance;
  if (feed < 0 || feed >= (int)imp.size()) return -999.0;
  return imp[feed].imag();
}
double nec_impedance_real(nec_context* c, int f) { return nec_impedance_real_indexed(c, f, 0); }
double nec_impedance_imag(nec_context* c, int f) { return nec_impedance_imag_indexed(c, f, 0); }

// ---- extensions ----
long nec_set_precision(nec_context* c, int p) {
  NEC_TRY(if (p != 0 && p != 1) necb::fail("precision must be 0 (FP64) or 1 (mixed)");
          c->set_precision(p));
}

long nec_set_intersection_check(nec_context* c, int enable, int fatal) {
  NEC_TRY(c->geometry().set_intersection_check(enable != 0);
          c->geometry().set_intersection_fatal(fatal != 0));
}

long nec_segment_count(nec_context* c) { return c ? (long)c->geometry().n : -1; }

long nec_frequency_scale(nec_context* c, double freq_mhz) {
  NEC_TRY(if (!c->geometry().completed) necb::fail("geometry not complete");
          c->geometry().frequency_scale(freq_mhz));
}

long nec_get_currents(nec_context* c, int index, double* out, long cap) {
  if (!c || index < 0 || index >= (int)c->currents.size()) return -1;
  auto& cur = c->currents[index].current;
  long n = (long)cur.size();
  if (cap < n) return -1;
  std::memcpy(out, cur.data(), sizeof(double) * 2 * n);
  return n;
}

long nec_get_segments(nec_context* c, double* x, double* y, double* z, double* si, double* bi,
                      double* cab, double* sab, double* salp, int* tags, int* icon1,
                      int* icon2) {
  if (!c || !c->geometry().completed) return -1;
  auto& g = c->geometry();
  for (int64_t i = 0; i < g.n; i++) {
    x[i] = g.x[i];
    y[i] = g.y[i];
    z[i] = g.z[i];
    si[i] = g.length[i];
    bi[i] = g.radius[i];
    cab[i] = g.cab[i];
    sab[i] = g.sab[i];
    salp[i] = g.salp[i];
    tags[i] = g.tags[i];
    icon1[i] = g.icon1[i];
    icon2[i] = g.icon2[i];
  }
  return (long)g.n;
}

long nec_get_trio(nec_context* c, int j, int* jco, double* ax, double* bx, double* cx, long cap) {
  if (!c || !c->geometry().completed) return -1;
  try {
    auto& g = c->geometry();
    g.prepare_basis();
    std::vector<necb::BasisEntry> e;
    g.trio(j, e);
    long k = 0;
    for (; k < (long)e.size() && k < cap; k++) {
      jco[k] = e[k].basis;
      ax[k] = e[k].a;
      bx[k] = e[k].b;
      cx[k] = e[k].c;
    }
    return (long)e.size();
  } catch (const std::exception& ex) {
    g_err = ex.what();
    return -1;
  }
}

long nec_prepare_structure(nec_context* c, double freq_mhz) { NEC_TRY(c->prepare_structure(freq_mhz)); }

long nec_get_structure(nec_context* c, double* seg, int* tptr, int* tbasis, double* tabc, int* ind,
                       double* params) {
  if (!c || c->tables.tptr.empty()) return -1;
  auto& g = c->geometry();
  auto& t = c->tables;
  const int64_t n = g.n, nt = (int64_t)t.tbasis.size();
  if (seg)
    for (int64_t i = 0; i < n; i++) {
      seg[i] = g.x[i];
      seg[n + i] = g.y[i];
      seg[2 * n + i] = g.z[i];
      seg[3 * n + i] = g.length[i];
      seg[4 * n + i] = g.radius[i];
      seg[5 * n + i] = g.cab[i];
      seg[6 * n + i] = g.sab[i];
      seg[7 * n + i] = g.salp[i];
    }
  if (tptr) std::memcpy(tptr, t.tptr.data(), sizeof(int) * (n + 1));
  if (tbasis) std::memcpy(tbasis, t.tbasis.data(), sizeof(int) * nt);
  if (tabc) {
    std::memcpy(tabc, t.ta.data(), sizeof(double) * nt);
    std::memcpy(tabc + nt, t.tb.data(), sizeof(double) * nt);
    std::memcpy(tabc + 2 * nt, t.tc.data(), sizeof(double) * nt);
  }
  if (ind) {
    std::memcpy(ind, t.ind1.data(), sizeof(int) * n);
    std::memcpy(ind + n, t.ind2.data(), sizeof(int) * n);
  }
  if (params) {
    params[0] = t.rkh;
    params[1] = t.use_exk;
    params[2] = t.ground;
    params[3] = t.zr_re;
    params[4] = t.zr_im;
    params[5] = t.fr_re;
    params[6] = t.fr_im;
    params[7] = t.eta;
    params[8] = t.eps_re;
    params[9] = t.eps_im;
  }
  return (long)nt;
}

long nec_get_rhs(nec_context* c, double* out) {
  NEC_TRY(if (c->tables.tptr.empty()) necb::fail("structure not prepared");
          std::vector<necb::cd> e; c->rhs(e);
          std::memcpy(out, e.data(), sizeof(double) * 2 * e.size()));
}

void* nec_gpu_engine(nec_context* c) {
  if (!c) return nullptr;
  try {
    return (void*)c->engine();
  } catch (const std::exception& ex) {
    g_err = ex.what();
    return nullptr;
  }
}

long nec_gradient(nec_context* base, int nparam, nec_context** plus, nec_context** minus, const double* h,
                  double theta_deg, double phi_deg, double* value, double* grad) {
  if (!base) return 1;
  NEC_TRY(base->gradient(nparam, plus, minus, h, theta_deg, phi_deg, value, grad));
}

long nec_last_refinement(nec_context* c, int* iters, double* residual) {
  if (!c) return 1;
  *iters = c->last_refine_iters;
  *residual = c->last_refine_residual;
  return 0;
}

long nec_get_pattern_fields(nec_context* c, int index, double* eth, double* eph, long cap) {
  auto* p = pattern_at(c, index);
  if (!p) return -1;
  long n = (long)p->e_theta.size();
  if (cap < n) return -1;
  std::memcpy(eth, p->e_theta.data(), sizeof(double) * 2 * n);
  std::memcpy(eph, p->e_phi.data(), sizeof(double) * 2 * n);
  return n;
}

}  // extern "C"
