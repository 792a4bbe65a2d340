// Thin-wire structure geometry for the B200 hot path (host side).
//
// Replaces c_geometry (src/c_geometry.h:63-305) for the wire-only subset the
// hot path covers: straight and tapered wires (c_geometry.cpp:614-696),
// helices and flat spirals (698-826), GM moves/copies (830-980), segment
// connection search and junction averaging (1337-2075), the segment-overlap
// rule (1405-1703), frequency scaling (3389-3418) and the basis-function
// tables trio/sbf/tbf (2763-3297).
//
// The integer connection tables icon1/icon2 and the junction-averaged end
// points must be bit-identical to the reference's, so every floating-point
// expression that feeds them keeps the reference's operation order.  The
// host library is compiled with -ffp-contract=off for the same reason.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace necb {

struct BasisEntry {
  int basis;  // 1-based segment index of the basis function (jco)
  double a, b, c;
};

class Geometry {
 public:
  // --- construction (metres) ---
  void wire(int tag, int nseg, double xw1, double yw1, double zw1, double xw2,
            double yw2, double zw2, double rad, double rdel, double rrad);
  void helix(int tag, int nseg, double s, double hl, double a1, double b1,
             double a2, double b2, double rad);
  void arc(int tag, int nseg, double rada, double ang1, double ang2, double rad);
  void move(double rox, double roy, double roz, double xs, double ys, double zs,
            int its, int nrpt, int itgi);
  void scale(double factor);
  void complete(int gpflag);
  void set_intersection_check(bool on) { check_overlaps_ = on; }
  void set_intersection_fatal(bool fatal) { overlap_fatal_ = fatal; }

  // --- per frequency ---
  void frequency_scale(double freq_mhz);
  int64_t segment_number(int tag, int m) const;

  // Basis tables at the current scaling (wavelengths).  sbf(i, is) is the
  // coefficient of the basis function centred on segment i, evaluated on
  // segment is; trio(j) lists every basis function that has support on
  // source segment j; tbf(i, icap) lists segment i's basis function on every
  // segment it covers.  All indices are 1-based as in the reference.
  void prepare_basis();
  void sbf(int i, int is, double* aa, double* bb, double* cc) const;
  void trio(int j, std::vector<BasisEntry>& out) const;
  void tbf(int i, int icap, std::vector<BasisEntry>& out) const;
  int test_ek_approximation(int seg1, int seg2) const;

  int64_t n = 0;   // segment count
  int64_t np = 0;  // segments in a symmetric cell (no symmetry: np == n)
  int ipsym = 0;
  bool completed = false;

  std::vector<int> tags;
  // before complete(): end points; after: x,y,z are centres, x2.. end 2
  std::vector<double> x, y, z, x2, y2, z2, radius;
  std::vector<double> length, cab, sab, salp;
  std::vector<int> icon1, icon2;

 private:
  void grow(int64_t new_n);
  void build_connections(int ignd);
  void resolve_junctions();
  void check_overlaps();

  std::vector<double> x_m_, y_m_, z_m_, si_m_, bi_m_;  // unscaled copies
  bool check_overlaps_ = true;
  bool overlap_fatal_ = true;

  // Per-segment terms of the basis functions at the current scaling.
  struct SegTerms {
    double sdh, cdh, sd, omc_link, omc_self, cd, aj, xxi;
  };
  std::vector<SegTerms> terms_;
};

}  // namespace necb
