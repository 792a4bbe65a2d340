// Physical and numerical constants of the NEC2++ thin-wire hot path.
//
// Every value here must be bit-identical to the reference's, because the
// reference derives all of its geometry scaling and kernel constants from
// them:
//   pi()            = 3.1415926536 (truncated)        math_util.h:72-74
//   two_pi/four_pi  = 2*pi(), 4*pi()                  math_util.h:76-82
//   rad<->deg       = multiply by 360/(2 pi), (2 pi)/360  math_util.h:97-105
//   eps0            = 8.854e-12                       electromag.cpp:22
//   mu0             = 4 pi() 1e-7                     electromag.cpp:23
//   c, eta          = 1/sqrt(mu eps), sqrt(mu/eps)    electromag.cpp:25-35
// The medium parameters are process-global and mutable in the reference
// (nec_medium_parameters, libnecpp.h:240); they are mirrored the same way.
#pragma once
#include <cmath>

namespace necb {

constexpr double kPi = 3.1415926536;
constexpr double kTwoPi = 2.0 * kPi;
constexpr double kFourPi = 4.0 * kPi;
constexpr double kPiTwo = kPi / 2.0;

// Constant of the thin-wire kernels: j*4.771341189 (nec_context.cpp:3055).
constexpr double kConst1Im = 4.771341189;

inline double rad_to_degrees(double r) {
  static const double k = 360.0 / (2 * kPi);
  return r * k;
}
inline double degrees_to_rad(double d) {
  static const double k = (2 * kPi) / 360.0;
  return d * k;
}

struct Medium {
  double permittivity = 8.854e-12;
  double permeability = kFourPi * 1.0e-7;
};
Medium& medium();  // process-global, like em::constants

inline double speed_of_light() {
  return 1.0 / std::sqrt(medium().permeability * medium().permittivity);
}
inline double impedance() {
  return std::sqrt(medium().permeability / medium().permittivity);
}
inline double impedance_over_2pi() { return impedance() / kTwoPi; }
inline double inverse_impedance() { return 1.0 / impedance(); }
inline double wavelength_of(double freq_hz) { return speed_of_light() / freq_hz; }

inline double db10(double x) { return x < 1.0e-20 ? -999.99 : 10.0 * std::log10(x); }
inline double from_db10(double x) { return x < -99.9 ? 0.0 : std::pow(10, x / 10.0); }

// Connection code marking a segment end joined to a surface patch
// (c_geometry.h:26).  Patches are not part of this build; the code is kept so
// the connection tables keep the reference's meaning.
constexpr int kPatchConnection = 100000;
// Relative contact distance of two segment ends (common.h:57).
constexpr double kSmin = 1.0e-3;

}  // namespace necb
