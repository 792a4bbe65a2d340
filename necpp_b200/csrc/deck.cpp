// Deck-file front end: runs a NEC input deck (the card images nec2++ reads,
// src/nec2cpp.cpp:134-445 and src/c_geometry.cpp:115-440) through the B200
// context and writes the result sections of nec2++'s text output that the
// reference's regression comparison reads (nec2diff, src/necDiff.cpp:41-93):
// antenna input parameters, power budget and radiation patterns, plus the
// near-field tables.  Section titles, column order and number formats follow
// nec2++ (nec_results.h output_helper: %W.PE / %W.Pf fields separated by a
// blank) so that a deck's output can be compared with the reference's.
//
// Cards: comments CM/CE; geometry GW (with GC taper), GA, GH, GM, GS, GE;
// program control FR, LD, GN, EX, NT, TL, EK, KH, PT, PQ, NE, NH, RP, XQ,
// MP, NX, EN, XT.  Cards outside this build (GR, GX, SP, SM, SC, GF, GD, CP,
// PL, WG) stop the run with a message, as any card error does.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/libnecpp.h"
#include "context.h"
#include "nec_constants.h"
#include "nec_error.h"

namespace necb {
namespace {

// One card image: the mnemonic and its numeric fields in free format
// (separated by blanks or commas), missing fields zero.
struct Card {
  std::string id;
  int i[4] = {0, 0, 0, 0};
  double f[7] = {0, 0, 0, 0, 0, 0, 0};
};

bool is_sep(char c) { return c == ' ' || c == '\t' || c == ',' || c == '\r' || c == '\n'; }

// nint integer fields then nflt real fields (2 + 7 for geometry cards,
// 4 + 6 for program-control cards).
Card parse_card(const std::string& line, int nint, int nflt) {
  Card c;
  if (line.size() < 2) fail("DATA CARD ERROR: CARD'S MNEMONIC CODE TOO SHORT OR MISSING");
  c.id = line.substr(0, 2);
  for (char& ch : c.id) ch = (char)std::toupper((unsigned char)ch);
  std::vector<std::string> tok;
  std::string cur;
  for (size_t k = 2; k < line.size(); k++) {
    if (is_sep(line[k])) {
      if (!cur.empty()) tok.push_back(cur);
      cur.clear();
    } else {
      cur.push_back(line[k]);
    }
  }
  if (!cur.empty()) tok.push_back(cur);
  for (int k = 0; k < nint && k < (int)tok.size(); k++) {
    const std::string& t = tok[k];
    size_t p = (t[0] == '+' || t[0] == '-') ? 1 : 0;
    if (p == t.size()) fail("DATA CARD \"", c.id, "\" ERROR: NON-NUMERICAL INTEGER FIELD '", t, "'");
    for (size_t q = p; q < t.size(); q++)
      if (!std::isdigit((unsigned char)t[q]))
        fail("DATA CARD \"", c.id, "\" ERROR: NON-NUMERICAL CHARACTER '", t[q], "' IN INTEGER FIELD");
    c.i[k] = std::atoi(t.c_str());
  }
  for (int k = 0; k < nflt && nint + k < (int)tok.size(); k++) {
    const std::string& t = tok[nint + k];
    char* end = nullptr;
    c.f[k] = std::strtod(t.c_str(), &end);
    if (end == t.c_str()) fail("DATA CARD \"", c.id, "\" ERROR: NON-NUMERICAL REAL FIELD '", t, "'");
  }
  return c;
}

// printf into a std::string
template <typename... A>
std::string fmt(const char* f, A... a) {
  char buf[512];
  std::snprintf(buf, sizeof(buf), f, a...);
  return buf;
}

void section(std::ostream& os, const std::string& title) {
  // output_helper::section_start / center_text (nec_results.h)
  os << "\n\n\n";
  const size_t len = title.size() + 2 * (5 + 1);
  os << std::string(40 - len / 2, ' ') << "----- " << title << " -----\n";
}

double arg_deg(cd z) { return std::atan2(z.imag(), z.real()) * (180.0 / kPi); }

void write_inputs(std::ostream& os, const AntennaInput& ai) {
  if (ai.tag.empty()) return;
  section(os, "ANTENNA INPUT PARAMETERS");
  os << "  TAG   SEG       VOLTAGE (VOLTS)         CURRENT (AMPS)         IMPEDANCE (OHMS)        "
        "ADMITTANCE (MHOS)     POWER\n";
  os << "  NO.   NO.     REAL      IMAGINARY     REAL      IMAGINARY     REAL      IMAGINARY    REAL       "
        "IMAGINARY   (WATTS)\n";
  for (size_t k = 0; k < ai.tag.size(); k++)
    os << fmt("%4d %5d %11.4E %11.4E %11.4E %11.4E %11.4E %11.4E %11.4E %11.4E %11.4E\n", ai.tag[k], ai.seg[k],
              ai.voltage[k].real(), ai.voltage[k].imag(), ai.current[k].real(), ai.current[k].imag(),
              ai.impedance[k].real(), ai.impedance[k].imag(), ai.admittance[k].real(),
              ai.admittance[k].imag(), ai.power[k]);
}

void write_budget(std::ostream& os, const PowerBudget& b) {
  const std::string pad(31, ' ');
  os << "\n\n\n" << pad << "---------- POWER BUDGET ---------\n";
  os << pad << fmt("INPUT POWER   = %11.4E Watts\n", b.input);
  os << pad << fmt("RADIATED POWER= %11.4E Watts\n", b.radiated);
  os << pad << fmt("STRUCTURE LOSS= %11.4E Watts\n", b.structure_loss);
  os << pad << fmt("NETWORK LOSS  = %11.4E Watts\n", b.network_loss);
  os << pad << fmt("EFFICIENCY    = %7.2f Percent\n", b.efficiency);
}

void write_pattern(std::ostream& os, const RadiationPattern& rp) {
  static const char* hpol[4] = {"LINEAR", "RIGHT ", "LEFT  ", " "};
  static const char* gain_type[2] = {"----- POWER GAINS ----- ", "--- DIRECTIVE GAINS ---"};
  static const char* igax[4] = {" MAJOR", " MINOR", " VERTC", " HORIZ"};
  section(os, "RADIATION PATTERNS");
  if (rp.range >= 1.0e-20) {
    double exra = rp.range / rp.wavelength;
    exra = -360.0 * (exra - std::floor(exra));
    os << "                             RANGE: " << fmt("%13.6E", rp.range) << " METERS\n";
    os << "                             EXP(-JKR)/R: " << fmt("%12.5E", 1.0 / rp.range)
       << " AT PHASE: " << fmt("%7.2f", exra) << " DEGREES\n";
  }
  const int a = 2 * rp.fmt, b = a + 1;
  os << " ---- ANGLES -----     " << fmt("%23s", gain_type[rp.ipd ? 1 : 0])
     << "      ---- POLARIZATION ----   ---- E(THETA) ----    ----- E(PHI) ------\n";
  os << "  THETA      PHI      " << fmt("%6s", igax[a]) << "  " << fmt("%6s", igax[b])
     << "   TOTAL       AXIAL      TILT  SENSE   MAGNITUDE    PHASE    MAGNITUDE     PHASE\n";
  os << " DEGREES   DEGREES        DB       DB       DB       RATIO   DEGREES            VOLTS/M   DEGREES"
        "     VOLTS/M   DEGREES\n";
  double phi = rp.ph0 - rp.dph;
  for (int kph = 0; kph < rp.nph; kph++) {
    phi += rp.dph;
    double thet = rp.th0 - rp.dth;
    for (int kth = 0; kth < rp.nth; kth++) {
      thet += rp.dth;
      if (rp.ground && thet > 90.01) continue;
      const size_t c = (size_t)kth + (size_t)kph * rp.nth;
      const int si = rp.sense[c] >= 0 && rp.sense[c] < 4 ? rp.sense[c] : 3;
      os << fmt(" %7.2f %9.2f  %8.2f %8.2f %8.2f %11.4f %9.2f %6s %11.4E %9.2f %11.4E %9.2f\n", thet, phi,
                rp.gain_vert[c], rp.gain_horiz[c], rp.gain_tot[c], rp.axial_ratio[c], rp.tilt[c], hpol[si],
                std::abs(rp.e_theta[c]), arg_deg(rp.e_theta[c]), std::abs(rp.e_phi[c]), arg_deg(rp.e_phi[c]));
    }
  }
  os << "\n";
}

void write_near(std::ostream& os, const NearFieldPattern& p) {
  if (p.x.empty()) return;
  if (p.nfeh != 1) {
    section(os, "NEAR ELECTRIC FIELDS");
    os << "     ------- LOCATION -------     ------- EX ------    ------- EY ------    ------- EZ ------\n";
    os << "      X         Y         Z       MAGNITUDE   PHASE    MAGNITUDE   PHASE    MAGNITUDE   PHASE\n";
    os << "    METERS    METERS    METERS     VOLTS/M  DEGREES    VOLTS/M   DEGREES     VOLTS/M  DEGREES\n";
  } else {
    section(os, "NEAR MAGNETIC FIELDS");
    os << "     ------- LOCATION -------     ------- HX ------    ------- HY ------    ------- HZ ------\n";
    os << "      X         Y         Z       MAGNITUDE   PHASE    MAGNITUDE   PHASE    MAGNITUDE   PHASE\n";
    os << "    METERS    METERS    METERS      AMPS/M  DEGREES      AMPS/M  DEGREES      AMPS/M  DEGREES\n";
  }
  for (size_t k = 0; k < p.x.size(); k++)
    os << fmt("  %9.4f %9.4f %9.4f  %11.4E %7.2f  %11.4E %7.2f  %11.4E %7.2f\n", p.x[k], p.y[k], p.z[k],
              std::abs(p.fx[k]), arg_deg(p.fx[k]), std::abs(p.fy[k]), arg_deg(p.fy[k]), std::abs(p.fz[k]),
              arg_deg(p.fz[k]));
}

// Everything the context produced since the last call, in its order.
void write_new_results(std::ostream& os, const Context& c, int& printed) {
  for (int seq = printed + 1;; seq++) {
    bool found = false;
    for (const auto& a : c.inputs)
      if (a.seq == seq) write_inputs(os, a), found = true;
    for (const auto& b : c.budgets)
      if (b.seq == seq) write_budget(os, b), found = true;
    for (const auto& p : c.near_fields)
      if (p.seq == seq) write_near(os, p), found = true;
    for (const auto& r : c.patterns)
      if (r.seq == seq) write_pattern(os, r), found = true;
    if (!found) break;
    printed = seq;
  }
}

bool read_line(std::istream& in, std::string& line) {
  if (!std::getline(in, line)) return false;
  while (!line.empty() && (line.back() == '\r' || line.back() == '\n')) line.pop_back();
  return true;
}

void banner(std::ostream& os) {
  const std::string pad(31, ' ');
  os << "\n\n" << pad << " __________________________________________\n"
     << pad << "|                                          |\n"
     << pad << "| NUMERICAL ELECTROMAGNETICS CODE (B200)   |\n"
     << pad << "|__________________________________________|\n";
}

// The geometry section up to GE (c_geometry::parse_geometry); `first`, if
// not empty, is its first card, already read.
void read_geometry(std::istream& in, std::ostream& os, Context& c, std::string first) {
  std::string line;
  for (;;) {
    if (!first.empty()) {
      line = first;
      first.clear();
    } else if (!read_line(in, line)) {
      fail("Error reading input file (no GE card).");
    }
    if (line.empty()) continue;
    Card g = parse_card(line, 2, 7);
    Geometry& geo = c.geometry();
    if (g.id == "GW") {
      double rdel = 1.0, rrad = 1.0, rad = g.f[6];
      if (rad == 0.0) {
        // tapered wire: GC continuation card (segment ratio, end radii)
        if (!read_line(in, line)) fail("GEOMETRY DATA CARD ERROR");
        Card gc = parse_card(line, 2, 7);
        if (gc.id != "GC") fail("GEOMETRY DATA CARD ERROR");
        if (gc.f[1] == 0 || gc.f[2] == 0) fail("GEOMETRY DATA CARD ERROR");
        rdel = gc.f[0];
        rad = gc.f[1];
        rrad = std::pow(gc.f[2] / gc.f[1], 1. / (g.i[1] - 1.));
      }
      geo.wire(g.i[0], g.i[1], g.f[0], g.f[1], g.f[2], g.f[3], g.f[4], g.f[5], rad, rdel, rrad);
    } else if (g.id == "GA") {
      geo.arc(g.i[0], g.i[1], g.f[0], g.f[1], g.f[2], g.f[3]);
    } else if (g.id == "GH") {
      geo.helix(g.i[0], g.i[1], g.f[0], g.f[1], g.f[2], g.f[3], g.f[4], g.f[5], g.f[6]);
    } else if (g.id == "GM") {
      geo.move(degrees_to_rad(g.f[0]), degrees_to_rad(g.f[1]), degrees_to_rad(g.f[2]), g.f[3], g.f[4], g.f[5],
               (int)(g.f[6] + .5), g.i[1], g.i[0]);
    } else if (g.id == "GS") {
      geo.scale(g.f[0]);
    } else if (g.id == "GE") {
      c.geometry_complete(g.i[0]);
      os << "\n\n     TOTAL SEGMENTS USED: " << geo.n << "     NO. SEG. IN A SYMMETRIC CELL: " << geo.np
         << "     SYMMETRY FLAG: " << geo.ipsym << "\n";
      return;
    } else if (g.id == "GR" || g.id == "GX" || g.id == "SP" || g.id == "SM" || g.id == "SC" || g.id == "GF") {
      fail(g.id, " is not part of the B200 thin-wire hot path");
    } else {
      fail("GEOMETRY DATA CARD ERROR: UNKNOWN CARD \"", g.id, "\"");
    }
  }
}

}  // namespace

// Runs every job of the deck; returns 0 at EN (or end of input after a
// complete job), 1 on an error (message in *err).
int run_deck(std::istream& in, std::ostream& os, std::string* err) {
  try {
    std::string line;
    for (;;) {
      banner(os);
      // comments
      if (!read_line(in, line)) fail("Error reading input file.");
      std::string id = line.substr(0, std::min<size_t>(2, line.size()));
      for (char& ch : id) ch = (char)std::toupper((unsigned char)ch);
      if (id == "XT") return 0;
      std::unique_ptr<Context> ctx(new Context());
      std::string first;
      if (id == "CM" || id == "CE") {
        os << "\n\n" << std::string(31, ' ') << "---------------- COMMENTS ----------------\n";
        os << (line.size() > 2 ? line.substr(2) : "") << "\n";
        while (id == "CM") {
          if (!read_line(in, line)) fail("Error reading input file (comments not terminated?)");
          id = line.substr(0, std::min<size_t>(2, line.size()));
          for (char& ch : id) ch = (char)std::toupper((unsigned char)ch);
          os << (line.size() > 2 ? line.substr(2) : "") << "\n";
        }
        if (id != "CE") fail("ERROR: INCORRECT LABEL FOR A COMMENT CARD");
      } else {
        first = line;  // the first geometry card
      }
      read_geometry(in, os, *ctx, first);
      // program control cards
      int printed = 0, ncard = 0;
      bool next_job = false;
      while (!next_job) {
        if (!read_line(in, line)) {
          write_new_results(os, *ctx, printed);
          return 0;
        }
        if (line.empty()) continue;
        Card c = parse_card(line, 4, 6);
        ncard++;
        os << fmt("\n*****  DATA CARD N0. %3d %s %3d %5d %5d %5d %12.5E %12.5E %12.5E %12.5E %12.5E %12.5E", ncard,
                  c.id.c_str(), c.i[0], c.i[1], c.i[2], c.i[3], c.f[0], c.f[1], c.f[2], c.f[3], c.f[4], c.f[5]);
        const std::string& m = c.id;
        if (m == "XT") return 0;
        if (m == "NX") {
          write_new_results(os, *ctx, printed);
          next_job = true;
        } else if (m == "EN") {
          write_new_results(os, *ctx, printed);
          os << "\n";
          return 0;
        } else if (m == "FR") {
          ctx->fr_card(c.i[0], c.i[1], c.f[0], c.f[1]);
        } else if (m == "LD") {
          ctx->ld_card(c.i[0], c.i[1], c.i[2], c.i[3], c.f[0], c.f[1], c.f[2]);
        } else if (m == "GN") {
          ctx->gn_card(c.i[0], c.i[1], c.f[0], c.f[1], c.f[2], c.f[3], c.f[4], c.f[5]);
        } else if (m == "EX") {
          ctx->ex_card(c.i[0], c.i[1], c.i[2], c.i[3], c.f[0], c.f[1], c.f[2], c.f[3], c.f[4], c.f[5]);
        } else if (m == "NT") {
          ctx->nt_card(c.i[0], c.i[1], c.i[2], c.i[3], c.f[0], c.f[1], c.f[2], c.f[3], c.f[4], c.f[5]);
        } else if (m == "TL") {
          ctx->tl_card(c.i[0], c.i[1], c.i[2], c.i[3], c.f[0], c.f[1], c.f[2], c.f[3], c.f[4], c.f[5]);
        } else if (m == "EK") {
          ctx->ek_card(c.i[0]);
        } else if (m == "KH") {
          ctx->kh_card(c.f[0]);
        } else if (m == "PT") {
          ctx->pt_card(c.i[0], c.i[1], c.i[2], c.i[3]);
        } else if (m == "PQ") {
          ctx->pq_card(c.i[0], c.i[1], c.i[2], c.i[3]);
        } else if (m == "MP") {
          ctx->medium_parameters(c.f[0], c.f[1]);
        } else if (m == "NE" || m == "NH") {
          ctx->ne_nh_card(m == "NH" ? 1 : 0, c.i[0], c.i[1], c.i[2], c.i[3], c.f[0], c.f[1], c.f[2], c.f[3],
                          c.f[4], c.f[5]);
          write_new_results(os, *ctx, printed);
        } else if (m == "RP") {
          const int x = c.i[3];
          ctx->rp_card(c.i[0], c.i[1], c.i[2], x / 1000, (x / 100) % 10, (x / 10) % 10, x % 10, c.f[0], c.f[1],
                       c.f[2], c.f[3], c.f[4], c.f[5]);
          write_new_results(os, *ctx, printed);
        } else if (m == "XQ") {
          ctx->xq_card(c.i[0]);
          write_new_results(os, *ctx, printed);
        } else if (m == "GD" || m == "CP" || m == "PL" || m == "WG") {
          fail(m, " is not part of the B200 thin-wire hot path");
        } else {
          fail("FAULTY DATA CARD LABEL AFTER GEOMETRY SECTION.");
        }
      }
    }
  } catch (const std::exception& ex) {
    if (err) *err = ex.what();
    os << "\n\nERROR: " << ex.what() << "\n";
    return 1;
  }
}

}  // namespace necb

static std::string g_deck_err;

extern "C" long nec_run_deck(const char* input_path, const char* output_path) {
  if (!input_path) return 1;
  std::ifstream in(input_path);
  if (!in) {
    g_deck_err = std::string("cannot open input file ") + input_path;
    return 1;
  }
  std::ofstream fout;
  std::ostream* os = &std::cout;
  if (output_path && *output_path) {
    fout.open(output_path);
    if (!fout) {
      g_deck_err = std::string("cannot open output file ") + output_path;
      return 1;
    }
    os = &fout;
  }
  return necb::run_deck(in, *os, &g_deck_err);
}

extern "C" const char* nec_deck_error(void) { return g_deck_err.c_str(); }
