// Host-side card state machine and result objects of the B200 hot path.
//
// Mirrors the observable behaviour of nec_context (src/nec_context.h:82-786,
// src/nec_context.cpp:406-1857) for the wire-only cards of the hot path:
// GW/GH/GM geometry, GE, FR, GN (free space, perfect, reflection coefficient,
// Sommerfeld/Norton), EK, KH, EX 0-4, XQ and RP (modes 0), plus the result
// accessors of the C API.  The fill, factor, solve and pattern run on the GPU
// through include/necgpu.h; there is no CPU fallback.
#pragma once
#include <complex>
#include <memory>
#include <string>
#include <vector>

#include "../../include/necgpu.h"
#include "geometry.h"


namespace necb {

using cd = std::complex<double>;

// Results carry `seq`, the order in which the context produced them (the
// order of the reference's printed output).
struct AntennaInput {
  int seq = 0;
  double freq_hz = 0;
  std::vector<int> tag, seg;
  std::vector<cd> voltage, current, impedance, admittance;
  std::vector<double> power;
};

struct StructureCurrents {
  double freq_hz = 0;
  std::vector<cd> current;  // amperes (current_vector * wavelength)
};

// nec_near_field_pattern (src/nec_results.h:564-655): points in metres,
// fields in V/m (electric) or A/m (magnetic)
struct NearFieldPattern {
  int seq = 0;
  double freq_hz = 0;
  int nfeh = 0;  // 0 electric, 1 magnetic
  std::vector<double> x, y, z;
  std::vector<cd> fx, fy, fz;
};

// print_power_budget, src/nec_context.cpp:1443-1466 (voltage excitation)
struct PowerBudget {
  int seq = 0;
  double freq_hz = 0;
  double input = 0, radiated = 0, structure_loss = 0, network_loss = 0, efficiency = 0;
};

struct RadiationPattern {
  int seq = 0;
  double freq_hz = 0;
  int nth = 0, nph = 0;
  double th0 = 0, ph0 = 0, dth = 0, dph = 0;
  bool ground = false;  // directions below the horizon are not evaluated
  int fmt = 0, ipd = 0;  // RP card's X (axis labels) and D (directive gain)
  double range = 0, wavelength = 0;
  // (kth, kph) stored at kth + kph * nth
  std::vector<double> gain, gain_vert, gain_horiz, gain_tot, gain_rhcp, gain_lhcp;
  std::vector<double> axial_ratio, tilt, avg_scale;
  std::vector<int> sense;
  std::vector<cd> e_theta, e_phi;
  double max_gain = -999.0;
  double average_power_gain = 0, average_power_solid_angle = 0;
  double stat_max(const std::vector<double>& v) const;
  double stat_min(const std::vector<double>& v) const;
  double stat_mean(const std::vector<double>& v) const;
  double stat_sd(const std::vector<double>& v) const;
};

class Context {
 public:
  Context();
  ~Context();

  Geometry& geometry() { return geo_; }

  // cards (src/nec_context.cpp line ranges in context.cpp)
  void geometry_complete(int gpflag);
  void fr_card(int ifrq, int nfrq, double freq_mhz, double del_freq);
  void gn_card(int ground_type, int nradl, double t1, double t2, double t3,
               double t4, double t5, double t6);
  void ex_card(int type, int i2, int i3, int i4, double f1, double f2, double f3,
               double f4, double f5, double f6);
  void xq_card(int mode);
  void rp_card(int mode, int nth, int nph, int xnda_x, int xnda_n, int xnda_d,
               int xnda_a, double th0, double ph0, double dth, double dph,
               double rfld, double gnor);
  void kh_card(double rkh);
  void ld_card(int type, int tag, int tag_from, int tag_to, double zr, double zi, double zc);
  void nt_card(int tag1, int seg1, int tag2, int seg2, double y11r, double y11i, double y12r, double y12i,
               double y22r, double y22i);
  void ne_nh_card(int nfeh, int near, int nx, int ny, int nz, double x0, double y0, double z0, double dx,
                  double dy, double dz);
  void tl_card(int tag1, int seg1, int tag2, int seg2, double z0, double length, double y1r, double y1i,
               double y2r, double y2i);
  int network_count() const { return (int)ntyp.size(); }
  void ek_card(int flag);
  void pt_card(int a, int b, int c, int d);
  void pq_card(int a, int b, int c, int d);
  void medium_parameters(double permittivity, double permeability);

  // build options (extensions)
  void set_precision(int p) { precision_ = p; }
  int precision() const { return precision_; }

  // results
  std::vector<AntennaInput> inputs;
  std::vector<RadiationPattern> patterns;
  std::vector<NearFieldPattern> near_fields;
  std::vector<PowerBudget> budgets;
  int next_seq() { return ++result_seq_; }
  std::vector<StructureCurrents> currents;
  double last_refine_residual = 0;
  int last_refine_iters = 0;

  necgpu_engine* engine();

  // Structure tables handed to the GPU at the current frequency (host only):
  // scale to freq_mhz, ground environment, basis tables, EK flags.
  void prepare_structure(double freq_mhz);
  // Applied-field vector of the current excitation at the prepared
  // frequency (etmns), host only.
  void rhs(std::vector<cd>& e) { build_rhs(e); }
  // Gradient of (Re Zin, Im Zin, gain in dB at (theta, phi)) of the last
  // solve with respect to nparam geometry parameters, by the adjoint method
  // on the held factors.  plus[k] / minus[k] hold the same cards with
  // parameter k moved by +h[k] / -h[k] (geometry complete, excitation set,
  // no solve).  One voltage source; mixed-precision factors.  value: 3,
  // grad: 3 * nparam (row k: d/dp_k of the three outputs).
  void gradient(int nparam, Context* const* plus, Context* const* minus, const double* h, double theta_deg,
                double phi_deg, double* value, double* grad);
  // the current structure as the GPU receives it (views of this context's arrays)
  necgpu_structure structure_view() const;
  // impedance loading of every segment at the prepared frequency (lambda x
  // impedance per unit length, as the reference's zarray), empty if unloaded
  const std::vector<cd>& loads() const { return zarray; }
  struct Tables {
    std::vector<int32_t> tptr, tbasis, ind1, ind2;
    std::vector<double> ta, tb, tc;
    int ground = 0;
    double zr_re = 1, zr_im = 0, fr_re = 1, fr_im = 0, eta = 0, rkh = 1;
    double eps_re = 0, eps_im = 0;  // complex permittivity of a finite ground
    int use_exk = 0;
  } tables;

 private:
  void build_tables();
  void load();
  double compute_structure_power_loss() const;
  // LD cards (names follow the reference's members) and their zarray
  std::vector<int> ldtyp, ldtag, ldtagf, ldtagt;
  std::vector<double> zlr, zli, zlc;
  std::vector<cd> zarray;
  // NT/TL cards (names follow the reference's members): type 1 network,
  // 2 transmission line, 3 crossed line; ports as 1-based segment numbers
  std::vector<int> ntyp;
  std::vector<int64_t> iseg1, iseg2;
  std::vector<double> x11r, x11i, x12r, x12i, x22r, x22i;
  int ntsol = 0;  // network equations solved for the current structure
  void network_card(int type, int tag1, int seg1, int tag2, int seg2, const double* x);
  void network_lengths();
  void solve_structure(const std::vector<cd>& rhs);
  enum State { MEM = 1, STRUCT = 2, EXSETUP = 3, EXLOOP = 4, NEAR = 5, FAR = 6 };
  enum Ret { PRINT_NORM = 0, FREQ_CONT = 1, CARD_CONT = 2, INNER_CONT = 3, PHASE_DONE = 4 };

  void calc_prepare();
  void reset_to_structure_loading();
  void reset_to_excitation_setup();
  void simulate(bool far_field_flag);
  int excitation_loop(int state_in, int mhz);
  int excitation_inner(int mhz);
  void far_field();
  void structure_loading();
  void antenna_environment();
  void build_rhs(std::vector<cd>& e);
  void network_solve();

  Geometry geo_;
  necgpu_engine* eng_ = nullptr;
  int precision_ = 1;  // NECGPU_MIXED; NECGPU_FP64 if its refinement fails

  // card state (names follow the reference's members)
  int iflow = 1, state_ = MEM;
  int ifrq = 0, nfrq = 1;
  double freq_mhz = 0, delfrq = 0, wavelength_ = 0;
  double rkh = 1.0;
  bool use_exk = false;
  int ex_type = 0;
  std::vector<int64_t> src_seg;
  std::vector<cd> src_volt;
  int nthi = 0, nphi = 0, nthic = 1, nphic = 1, inc = 1;
  double xpr1 = 0, xpr2 = 0, xpr3 = 0, xpr4 = 0, xpr5 = 0, xpr6 = 0, xpr7 = 0;
  double thetis = 0, phiss = 0;
  int iped = 0, masym = 0;
  double zpnorm = 0;
  int ifar = -1, nth = 0, nph = 0, rp_fmt = 0, rp_norm = 0, ipd = 0, iavp = 0;
  double thets = 0, phis = 0, dth = 0, dph = 0, rfld = 0, gnor = 0;
  int iptflg = -2, iptag = 0, iptagf = 0, iptagt = 0;
  int iptflq = -1, iptaq = 0, iptaqf = 0, iptaqt = 0;
  int result_seq_ = 0;
  int m_near = -1;
  int nfeh = 0, nrx = 0, nry = 0, nrz = 0;
  double xnr = 0, ynr = 0, znr = 0, dxnr = 0, dynr = 0, dznr = 0;
  void nfpat();
  double input_power = 0, network_power_loss = 0, structure_power_loss = 0;

  // ground
  int ksymp = 1, iperf = 0, nradl = 0;
  double epsr = 0, sig = 0;
  cd zrati{1.0, 0.0}, frati{1.0, 0.0}, epsc{0, 0};

  // per-frequency device structure state
  std::vector<cd> solution;  // segment-centre currents (current_vector)
  std::vector<double> abc;   // air aii bir bii cir cii
  bool have_factor_ = false;
};

}  // namespace necb
