// Thin-wire geometry, connection tables and basis-function tables.
// Algorithms follow NEC2++ src/c_geometry.cpp (line ranges cited per
// function); the code is organised around per-segment precomputed terms
// instead of the reference's recomputation inside every sbf/tbf call.
#include "geometry.h"
#include "host_parallel.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <numeric>
#include <tuple>
#include <thread>
#include <unordered_map>
#include <cstdint>
#include <climits>

#include "nec_constants.h"
#include "nec_error.h"

namespace necb {

namespace {

struct V3 {
  double x, y, z;
};
inline V3 sub(const V3& a, const V3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
// Euclidean norm, summed x, y, z in order then sqrt (the order of a
// fixed-size 3-vector reduction).
inline double norm3(const V3& v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
inline double norm_l1(const V3& v) { return std::fabs(v.x) + std::fabs(v.y) + std::fabs(v.z); }

}  // namespace

void Geometry::grow(int64_t new_n) {
  tags.resize(new_n);
  x.resize(new_n);
  y.resize(new_n);
  z.resize(new_n);
  x2.resize(new_n);
  y2.resize(new_n);
  z2.resize(new_n);
  radius.resize(new_n);
}

// Straight or tapered wire: c_geometry.cpp:614-696.
void Geometry::wire(int tag, int nseg, double xw1, double yw1, double zw1,
                    double xw2, double yw2, double zw2, double rad, double rdel,
                    double rrad) {
  if (completed) fail("GEOMETRY ALREADY COMPLETE");
  int64_t istart = n;
  n += nseg;
  np = n;
  ipsym = 0;
  if (nseg < 1) return;
  grow(n);

  double dx = xw2 - xw1, dy = yw2 - yw1, dz = zw2 - zw1;
  double delz, rd;
  if (std::fabs(rdel - 1.0) >= 1.0e-6) {
    delz = norm3({dx, dy, dz});
    dx /= delz;
    dy /= delz;
    dz /= delz;
    delz = delz * (1. - rdel) / (1. - std::pow(rdel, nseg));
    rd = rdel;
  } else {
    double fns = nseg;
    dx /= fns;
    dy /= fns;
    dz /= fns;
    delz = 1.0;
    rd = 1.0;
  }
  double radz = rad;
  double sx = xw1, sy = yw1, sz = zw1;
  for (int64_t i = istart; i < n; i++) {
    tags[i] = tag;
    double ex = sx + dx * delz, ey = sy + dy * delz, ez = sz + dz * delz;
    x[i] = sx;
    y[i] = sy;
    z[i] = sz;
    x2[i] = ex;
    y2[i] = ey;
    z2[i] = ez;
    radius[i] = radz;
    delz = delz * rd;
    radz = radz * rrad;
    sx = ex;
    sy = ey;
    sz = ez;
  }
  x2[n - 1] = xw2;
  y2[n - 1] = yw2;
  z2[n - 1] = zw2;
}

// Arc of radius rada in the x-z plane from ang1 to ang2 degrees (GA card),
// c_geometry.cpp:2077-2127: nseg chords of equal angle.
void Geometry::arc(int tag, int nseg, double rada, double ang1, double ang2, double rad) {
  if (completed) fail("GEOMETRY ALREADY COMPLETE");
  const int64_t istart = n;
  n += nseg;
  np = n;
  ipsym = 0;
  if (nseg < 1) return;
  if (std::fabs(ang2 - ang1) > 360.0) fail("ERROR -- ARC ANGLE EXCEEDS 360 DEGREES");
  grow(n);
  double ang = degrees_to_rad(ang1);
  const double dang = degrees_to_rad(ang2 - ang1) / nseg;
  double xs1 = rada * std::cos(ang), zs1 = rada * std::sin(ang);
  for (int64_t i = istart; i < n; i++) {
    ang += dang;
    const double xs2 = rada * std::cos(ang), zs2 = rada * std::sin(ang);
    x[i] = xs1;
    y[i] = 0.;
    z[i] = zs1;
    x2[i] = xs2;
    y2[i] = 0.;
    z2[i] = zs2;
    xs1 = xs2;
    zs1 = zs2;
    radius[i] = rad;
    tags[i] = tag;
  }
}

// Helix / spiral: c_geometry.cpp:698-826 (the printout is not reproduced).
void Geometry::helix(int tag, int nseg, double s, double hl, double a1,
                     double b1, double a2, double b2, double rad) {
  if (completed) fail("GEOMETRY ALREADY COMPLETE");
  if (nseg < 1) fail("HELIX: segment count must be >= 1");
  int64_t ist = n;
  n += nseg;
  np = n;
  ipsym = 0;
  double zinc = std::fabs(hl / nseg);
  grow(n);

  if (hl == 0.) {  // flat spiral
    double phi = 0.;
    double dphi = 2. * kPi / s;
    double da = (a1 - a2) / nseg;
    double db = (b1 - b2) / nseg;
    for (int64_t i = ist; i < n; i++) {
      radius[i] = rad;
      tags[i] = tag;
      z[i] = 0.;
      z2[i] = 0.;
      x[i] = a1 * std::cos(phi);
      y[i] = b1 * std::sin(phi);
      a1 -= da;
      b1 -= db;
      phi += dphi;
      x2[i] = a1 * std::cos(phi);
      y2[i] = b1 * std::sin(phi);
    }
    return;
  }

  z[ist] = 0.;
  for (int64_t i = ist; i < n; i++) {
    radius[i] = rad;
    tags[i] = tag;
    if (i != ist) z[i] = z[i - 1] + zinc;
    z2[i] = z[i] + zinc;
    if (a2 == a1) {
      if (b1 == 0.) b1 = a1;
      x[i] = a1 * std::cos(2. * kPi * z[i] / s);
      y[i] = b1 * std::sin(2. * kPi * z[i] / s);
      x2[i] = a1 * std::cos(2. * kPi * z2[i] / s);
      y2[i] = b1 * std::sin(2. * kPi * z2[i] / s);
    } else {
      if (b2 == 0.) b2 = a2;
      x[i] = (a1 + (a2 - a1) * z[i] / std::fabs(hl)) * std::cos(2. * kPi * z[i] / s);
      y[i] = (b1 + (b2 - b1) * z[i] / std::fabs(hl)) * std::sin(2. * kPi * z[i] / s);
      x2[i] = (a1 + (a2 - a1) * z2[i] / std::fabs(hl)) * std::cos(2. * kPi * z2[i] / s);
      y2[i] = (b1 + (b2 - b1) * z2[i] / std::fabs(hl)) * std::sin(2. * kPi * z2[i] / s);
    }
    if (hl < 0.) {  // left-handed
      y[i] = -y[i];
      y2[i] = -y2[i];
    }
  }
}

int64_t Geometry::segment_number(int tag, int m) const {
  if (m <= 0)
    fail("CHECK DATA, PARAMETER SPECIFYING SEGMENT POSITION IN A GROUP OF "
         "EQUAL TAGS MUST NOT BE ZERO");
  if (tag == 0) return m;
  int64_t count = 0;
  for (int64_t i = 0; i < n; i++)
    if (tags[i] == tag && ++count == m) return i + 1;
  fail("NO SEGMENT HAS AN ITAG OF ", tag);
}

// GM card: rotate by (rox, roy, roz) radians then shift; nrpt copies with
// tag increment itgi, starting at the first segment of tag its
// (c_geometry.cpp:830-980; patches are not part of this build).
void Geometry::move(double rox, double roy, double roz, double xs, double ys,
                    double zs, int its, int nrpt, int itgi) {
  if (completed) fail("GEOMETRY ALREADY COMPLETE");
  if (std::fabs(rox) + std::fabs(roy) > 1.0e-10) ipsym = ipsym * 3;
  double sps = std::sin(rox), cps = std::cos(rox);
  double sth = std::sin(roy), cth = std::cos(roy);
  double sph = std::sin(roz), cph = std::cos(roz);
  double xx = cph * cth;
  double xy = cph * sth * sps - sph * cps;
  double xz = cph * sth * cps + sph * sps;
  double yx = sph * cth;
  double yy = sph * sth * sps + cph * cps;
  double yz = sph * sth * cps - cph * sps;
  double zx = -sth;
  double zy = cth * sps;
  double zz = cth * cps;
  int64_t nrp = (nrpt == 0) ? 1 : nrpt;
  int64_t ix = 1;
  if (n > 0) {
    int64_t i1 = segment_number(its, 1);
    if (i1 < 1) i1 = 1;
    ix = i1;
    int64_t k;
    if (nrpt == 0) {
      k = i1 - 1;
    } else {
      k = n;
      grow(n + (n + 1 - i1) * nrpt);
    }
    for (int64_t ir = 0; ir < nrp; ir++) {
      for (int64_t i = i1 - 1; i < n; i++) {
        double xi = x[i], yi = y[i], zi = z[i];
        x[k] = xi * xx + yi * xy + zi * xz + xs;
        y[k] = xi * yx + yi * yy + zi * yz + ys;
        z[k] = xi * zx + yi * zy + zi * zz + zs;
        xi = x2[i];
        yi = y2[i];
        zi = z2[i];
        x2[k] = xi * xx + yi * xy + zi * xz + xs;
        y2[k] = xi * yx + yi * yy + zi * yz + ys;
        z2[k] = xi * zx + yi * zy + zi * zz + zs;
        radius[k] = radius[i];
        tags[k] = tags[i];
        if (tags[i] != 0) tags[k] = tags[i] + itgi;
        k++;
      }
      i1 = n + 1;
      n = k;
    }
  }
  if (nrpt == 0 && ix == 1) return;
  np = n;
  ipsym = 0;
}

void Geometry::scale(double f) {
  if (completed) fail("GEOMETRY ALREADY COMPLETE");
  for (int64_t i = 0; i < n; i++) {
    x[i] *= f;
    y[i] *= f;
    z[i] *= f;
    x2[i] *= f;
    y2[i] *= f;
    z2[i] *= f;
    radius[i] *= f;
  }
}

// Connection search, c_geometry.cpp:1705-1916 (wire part).  For every end of
// every segment, the other segments are scanned starting after the segment
// itself, wrapping round; the first end within SMIN * length (L1 distance)
// wins.  The sign of the stored index says whether the touching end is of
// the same kind (negative) or the opposite kind (positive).
namespace {
// Endpoints of all segments bucketed on a cubic grid of edge 2 * max(slen):
// every end within L1 distance slen of a point lies in the 27 cells around
// the point's cell.  The search below returns what the reference's cyclic
// scan returns (the first segment after i, wrapping, whose start and then
// end satisfies the same test), looking only at those cells.
struct EndGrid {
  double cell = 0;
  std::unordered_map<uint64_t, std::vector<int64_t>> cells;  // value: 2 * segment + (0 start, 1 end)
  static int64_t idx(double v, double cell) { return (int64_t)std::floor(v / cell); }
  static uint64_t key(int64_t a, int64_t b, int64_t c) {
    return ((uint64_t)(a & 0x1FFFFF) << 42) | ((uint64_t)(b & 0x1FFFFF) << 21) | (uint64_t)(c & 0x1FFFFF);
  }
};

// Points bucketed on a cubic grid without per-cell allocations: the items
// sorted by cell, and an open-addressing table from a cell's key to its
// range in that order.
struct FlatGrid {
  double cell = 1;
  std::vector<int64_t> order;                  // item ids sorted by cell key
  std::vector<uint64_t> slot_key;              // table: key + 1 (0 = empty)
  std::vector<std::pair<int64_t, int64_t>> slot_range;
  std::vector<uint32_t> slot_of, used;  // build scratch: each item's slot, the occupied slots
  uint64_t mask = 0;
  static uint64_t hash(uint64_t k) {  // splitmix64 finaliser
    k ^= k >> 30;
    k *= 0xbf58476d1ce4e5b9ULL;
    k ^= k >> 27;
    k *= 0x94d049bb133111ebULL;
    k ^= k >> 31;
    return k;
  }
  template <typename Pos>
  void build(size_t count, double c, Pos pos) {
    cell = c;
    // counting sort by cell: the table gives each distinct key a slot, the
    // slots' counts become ranges, and the items are scattered in item
    // order, so each cell lists its items in ascending order
    size_t cap = 16;
    while (cap < 2 * count) cap *= 2;
    mask = cap - 1;
    slot_key.assign(cap, 0);
    slot_range.assign(cap, {0, 0});
    slot_of.resize(count);
    used.clear();
    for (size_t i = 0; i < count; i++) {
      const V3 v = pos(i);
      const uint64_t k = EndGrid::key(EndGrid::idx(v.x, c), EndGrid::idx(v.y, c), EndGrid::idx(v.z, c));
      uint64_t h = hash(k) & mask;
      while (slot_key[h] && slot_key[h] != k + 1) h = (h + 1) & mask;
      if (!slot_key[h]) used.push_back((uint32_t)h);
      slot_key[h] = k + 1;
      slot_range[h].second++;
      slot_of[i] = (uint32_t)h;
    }
    int64_t at = 0;
    for (const uint32_t h : used) {
      const int64_t cnt = slot_range[h].second;
      slot_range[h] = {at, at};
      at += cnt;
    }
    order.resize(count);
    for (size_t i = 0; i < count; i++) order[slot_range[slot_of[i]].second++] = (int64_t)i;
  }
  // the range in `order` of the cell with key k (empty if none)
  std::pair<int64_t, int64_t> find(uint64_t k) const {
    for (uint64_t h = hash(k) & mask;; h = (h + 1) & mask) {
      if (!slot_key[h]) return {0, 0};
      if (slot_key[h] == k + 1) return slot_range[h];
    }
  }
};
}  // namespace

void Geometry::build_connections(int ignd) {
  if (ignd != 0) {
    if (ipsym == 2) np = 2 * np;
    if (std::abs(ipsym) > 2) np = n;
    if (np > n) fail("ERROR: NP > N IN c_geometry::build_connections()");
    if (np == n) ipsym = 0;
  }
  icon1.assign(n, 0);
  icon2.assign(n, 0);
  // Without a ground plane the coordinates do not change during the search,
  // so it can use the endpoint grid (the O(N^2) scan dominates card
  // processing of large structures otherwise).
  double max_slen = 0.0;
  for (int64_t i = 0; i < n; i++)
    max_slen = std::max(max_slen, norm3(sub(V3{x2[i], y2[i], z2[i]}, V3{x[i], y[i], z[i]})) * kSmin);
  const bool use_grid = ignd == 0 && n > 256 && std::isfinite(max_slen) && max_slen > 0.0;
  // kept per thread between calls: a new structure reuses the mapped buffers.
  // Worker threads reach it through the reference (naming the thread_local
  // inside their lambdas would give them their own, empty, instances).
  static thread_local FlatGrid tl_grid;
  FlatGrid& grid = tl_grid;
  // cells of four times the search distance: a query box then meets one
  // or two cells per axis (3.4 on average, against 8 with cells of twice
  // the distance), and the sparse end points add few candidates per cell
  if (use_grid)
    grid.build((size_t)(2 * n), 4.0 * max_slen, [&](size_t code) {
      const int64_t i = (int64_t)(code >> 1);
      return (code & 1) ? V3{x2[i], y2[i], z2[i]} : V3{x[i], y[i], z[i]};
    });
  // first match in the cyclic order i+1, i+2, ..., i-1 (start before end of
  // the same segment): returns 2 * segment + end, or -1
  auto grid_first = [&](int64_t i, const V3& v, double slen) -> int64_t {
    // ends within L1 distance slen lie in the cubes the box v +- slen meets
    const double cell = grid.cell;
    const int64_t x0 = EndGrid::idx(v.x - slen, cell), x1 = EndGrid::idx(v.x + slen, cell);
    const int64_t y0 = EndGrid::idx(v.y - slen, cell), y1 = EndGrid::idx(v.y + slen, cell);
    const int64_t z0 = EndGrid::idx(v.z - slen, cell), z1 = EndGrid::idx(v.z + slen, cell);
    int64_t best = -1, best_rank = INT64_MAX;
    for (int64_t a = x0; a <= x1; a++)
      for (int64_t b = y0; b <= y1; b++)
        for (int64_t c = z0; c <= z1; c++) {
          const auto rg = grid.find(EndGrid::key(a, b, c));
          for (int64_t q = rg.first; q < rg.second; q++) {
            const int64_t code = grid.order[q];
            const int64_t ic = code >> 1;
            if (ic == i) continue;
            const int end = (int)(code & 1);
            const V3 p = end == 0 ? V3{x[ic], y[ic], z[ic]} : V3{x2[ic], y2[ic], z2[ic]};
            if (!(norm_l1(sub(v, p)) <= slen)) continue;
            const int64_t rank = ((ic - i - 1 + n) % n) * 2 + end;
            if (rank < best_rank) {
              best_rank = rank;
              best = code;
            }
          }
        }
    return best;
  };
  if (use_grid) {
    // no ground: the searches only read the coordinates, so the segments
    // are split over worker threads
    auto search = [&](int, int64_t i0, int64_t i1) {
      for (int64_t i = i0; i < i1; i++) {
        const V3 v1{x[i], y[i], z[i]}, v2{x2[i], y2[i], z2[i]};
        const double slen = norm3(sub(v2, v1)) * kSmin;
        int64_t m = grid_first(i, v1, slen);
        icon1[i] = m < 0 ? 0 : ((m & 1) == 0 ? -(int)((m >> 1) + 1) : (int)((m >> 1) + 1));
        m = grid_first(i, v2, slen);
        icon2[i] = m < 0 ? 0 : ((m & 1) == 0 ? (int)((m >> 1) + 1) : -(int)((m >> 1) + 1));
      }
    };
    parallel_chunks(n, host_workers(n, 512), search);
  }
  for (int64_t i = 0; i < n && !use_grid; i++) {
    int64_t iz = i + 1;
    double zi1 = z[i], zi2 = z2[i];
    V3 v1{x[i], y[i], z[i]}, v2{x2[i], y2[i], z2[i]};
    double slen = norm3(sub(v2, v1)) * kSmin;

    bool on_ground = false;
    if (ignd > 0) {
      if (zi1 <= -slen) fail("GEOMETRY DATA ERROR--SEGMENT ", iz, "EXTENDS BELOW GROUND");
      if (zi1 <= slen) {
        icon1[i] = (int)iz;
        z[i] = 0.;
        on_ground = true;
      }
    }
    if (!on_ground) {
      int64_t ic = i;
      bool found = false;
      for (int64_t j = 1; j < n; j++) {
        if (++ic >= n) ic = 0;
        if (norm_l1(sub(v1, V3{x[ic], y[ic], z[ic]})) <= slen) {
          icon1[i] = -(int)(ic + 1);
          found = true;
          break;
        }
        if (norm_l1(sub(v1, V3{x2[ic], y2[ic], z2[ic]})) <= slen) {
          icon1[i] = (int)(ic + 1);
          found = true;
          break;
        }
      }
      if (!found) icon1[i] = 0;
    }

    if (ignd > 0 || on_ground) {
      if (zi2 <= -slen) fail("GEOMETRY DATA ERROR--SEGMENT ", iz, "EXTENDS BELOW GROUND");
      if (zi2 <= slen) {
        if (icon1[i] == iz) fail("GEOMETRY DATA ERROR--SEGMENT ", iz, "LIES IN GROUND PLANE");
        icon2[i] = (int)iz;
        z2[i] = 0.;
        continue;
      }
    }
    v1 = V3{x[i], y[i], z[i]};
    v2 = V3{x2[i], y2[i], z2[i]};
    int64_t ic = i;
    bool found = false;
    for (int64_t j = 1; j < n; j++) {
      if (++ic >= n) ic = 0;
      if (norm_l1(sub(v2, V3{x[ic], y[ic], z[ic]})) <= slen) {
        icon2[i] = (int)(ic + 1);
        found = true;
        break;
      }
      if (norm_l1(sub(v2, V3{x2[ic], y2[ic], z2[ic]})) <= slen) {
        icon2[i] = -(int)(ic + 1);
        found = true;
        break;
      }
    }
    if (!found) icon2[i] = 0;
  }
  if (np == 0) fail("connect_segments Geometry has zero wires and zero patches.");
  if (n / np != 1 && ipsym == 0) fail("ERROR: IPSYM=0 IN build_connections()");
}

// Junction averaging, c_geometry.cpp:1918-2075.  Starting from each end of
// each segment, the ring of ends joined there is walked through icon1/icon2;
// the walk is abandoned when it meets a lower-numbered segment (that segment
// already averaged the junction).  Otherwise all ends on the ring are moved
// to the mean of their positions, summed in walk order.
void Geometry::resolve_junctions() {
  std::vector<int64_t> ring(8);
  for (int64_t j = 0; j < n; j++) {
    const int64_t jx = j + 1;
    int iend = -1, jend = -1;
    int64_t ix = icon1[j];
    int64_t ic = 1;
    ring[0] = -jx;
    double xa = x[j], ya = y[j], za = z[j];
    while (true) {
      if (ix != 0 && ix != jx && ix <= n) {
        bool jump = false;
        do {
          if (ix == 0) fail("CONNECT - SEGMENT CONNECTION ERROR FOR SEGMENT: ", ix);
          if (ix < 0)
            ix = -ix;
          else
            jend = -jend;
          jump = false;
          if (ix == jx) break;
          if (ix < jx) {
            jump = true;
            break;
          }
          ic++;
          if ((int64_t)ring.size() < ic) ring.resize(ic * 2);
          ring[ic - 1] = ix * jend;
          int64_t ixx = ix - 1;
          if (ixx < 0 || ixx >= n) fail("CONNECT - SEGMENT CONNECTION ERROR (bad index): ", ix);
          if (jend != 1) {
            xa = xa + x[ixx];
            ya = ya + y[ixx];
            za = za + z[ixx];
            ix = icon1[ixx];
          } else {
            xa = xa + x2[ixx];
            ya = ya + y2[ixx];
            za = za + z2[ixx];
            ix = icon2[ixx];
          }
        } while (ix != 0);

        if (jump && iend == 1) break;
        if (jump) {
          iend = 1;
          jend = 1;
          ix = icon2[j];
          ic = 1;
          ring[0] = jx;
          xa = x2[j];
          ya = y2[j];
          za = z2[j];
          continue;
        }
        double sep = static_cast<double>(ic);
        xa = xa / sep;
        ya = ya / sep;
        za = za / sep;
        for (int64_t i = 0; i < ic; i++) {
          int64_t e = ring[i];
          if (e <= 0) {
            int64_t ixx = -e - 1;
            if (ixx < 0 || ixx >= n) fail("CONNECT - JUNCTION INDEX ERROR: ", -e);
            x[ixx] = xa;
            y[ixx] = ya;
            z[ixx] = za;
          } else {
            int64_t ixx = e - 1;
            if (ixx < 0 || ixx >= n) fail("CONNECT - JUNCTION INDEX ERROR: ", e);
            x2[ixx] = xa;
            y2[ixx] = ya;
            z2[ixx] = za;
          }
        }
      }
      if (iend == 1) break;
      iend = 1;
      jend = 1;
      ix = icon2[j];
      ic = 1;
      ring[0] = jx;
      xa = x2[j];
      ya = y2[j];
      za = z2[j];
    }
  }
}

// Segment-overlap rule, c_geometry.cpp:1405-1703: a segment centre lying
// inside the volume of a segment it does not share exactly one node with is
// an error (fatal by default).  Nodes are the classes of segment ends in
// contact (L1 distance within the larger of the two ends' thresholds).
void Geometry::check_overlaps() {
  if (!check_overlaps_ || n < 2) return;
  struct End {
    V3 p;
    int64_t idx;
    double thr;
  };
  struct View {
    int64_t idx;
    V3 a, b, c;  // end one, end two, centre
    double r;
    int tag;
  };
  // per-thread scratch kept between structures (the pages stay mapped);
  // worker threads reach it through these references
  static thread_local std::vector<End> tl_ends;
  static thread_local std::vector<View> tl_views;
  static thread_local std::vector<int64_t> tl_parent;
  static thread_local std::vector<std::pair<int64_t, int64_t>> tl_nodes;
  std::vector<End>& ends = tl_ends;
  std::vector<View>& views = tl_views;
  // a structure much smaller than the largest one seen returns the memory
  // (one large structure would otherwise stay mapped in this thread)
  const size_t nseg = (size_t)n;
  auto trim = [nseg](auto& v, size_t per) {
    if (v.capacity() > 4096 && v.capacity() > 8 * per * nseg) {
      v.clear();
      v.shrink_to_fit();
    }
  };
  trim(ends, 2);
  trim(views, 1);
  trim(tl_parent, 2);
  trim(tl_nodes, 2);
  ends.clear();
  views.clear();
  ends.reserve(2 * n);
  views.reserve(n);
  for (int64_t i = 0; i < n; i++) {
    V3 c{x[i], y[i], z[i]};
    double h = 0.5 * length[i];
    V3 ha{cab[i] * h, sab[i] * h, salp[i] * h};
    V3 a = sub(c, ha);
    V3 b{c.x + ha.x, c.y + ha.y, c.z + ha.z};
    views.push_back(View{i, a, b, c, radius[i], tags[i]});
    double thr = norm3(sub(b, a)) * kSmin;
    ends.push_back(End{a, 2 * i, thr});
    ends.push_back(End{b, 2 * i + 1, thr});
  }
  auto axis_of = [](auto& items) {
    V3 lo = items[0].p, hi = lo;
    for (size_t i = 1; i < items.size(); i++) {
      lo = V3{std::min(lo.x, items[i].p.x), std::min(lo.y, items[i].p.y), std::min(lo.z, items[i].p.z)};
      hi = V3{std::max(hi.x, items[i].p.x), std::max(hi.y, items[i].p.y), std::max(hi.z, items[i].p.z)};
    }
    double e[3] = {hi.x - lo.x, hi.y - lo.y, hi.z - lo.z};
    int ax = 0;
    for (int k = 1; k < 3; k++)
      if (e[k] > e[ax]) ax = k;
    return ax;
  };
  auto coord = [](const V3& v, int ax) { return ax == 0 ? v.x : (ax == 1 ? v.y : v.z); };

  // node classes (union-find over ends)
  std::vector<int64_t>& parent = tl_parent;
  parent.resize(2 * n);
  std::iota(parent.begin(), parent.end(), 0);
  auto root = [&](int64_t e) {
    while (parent[e] != e) {
      parent[e] = parent[parent[e]];
      e = parent[e];
    }
    return e;
  };
  double thr_max = 0.0;
  for (auto& e : ends) thr_max = std::max(thr_max, e.thr);
  // Candidate pairs come from a grid of cubes no smaller than the largest
  // interaction distance: the box of half-width `reach` around an item meets
  // at most two cubes along each axis, and every pair within that distance
  // is among the items found there.  Without a usable cube size the pairs
  // come from a sweep along the widest axis.  visit(worker, a, p) sees each
  // candidate pair once, a < p; with the grid the items are split over
  // worker threads, each visiting the pairs of its own items.
  const int nworkers = host_workers(2 * n, 512);
  // cell_factor: cell edge over reach (>= 2; larger for sparse points, so
  // that a query meets fewer cells)
  auto grid_pairs = [&](size_t count, auto pos, double reach, double cell_factor, int workers, auto visit) {
    if (std::isfinite(reach) && reach > 0.0 && count > 256) {
      // reused by the two searches and by later structures; workers use the
      // reference, not the thread_local name
      static thread_local FlatGrid tl_pair_grid;
      FlatGrid& grid = tl_pair_grid;
      const double cell = cell_factor * reach;
      grid.build(count, cell, pos);
      const double r2 = reach * reach * 3.0;
      auto range = [&](int w, size_t i0, size_t i1) {
        for (size_t i = i0; i < i1; i++) {
          const V3 v = pos(i);
          const int64_t x0 = EndGrid::idx(v.x - reach, cell), x1 = EndGrid::idx(v.x + reach, cell);
          const int64_t y0 = EndGrid::idx(v.y - reach, cell), y1 = EndGrid::idx(v.y + reach, cell);
          const int64_t z0 = EndGrid::idx(v.z - reach, cell), z1 = EndGrid::idx(v.z + reach, cell);
          for (int64_t a = x0; a <= x1; a++)
            for (int64_t b = y0; b <= y1; b++)
              for (int64_t c = z0; c <= z1; c++) {
                const auto rg = grid.find(EndGrid::key(a, b, c));
                for (int64_t q = rg.first; q < rg.second; q++) {
                  const int64_t j = grid.order[q];
                  if ((size_t)j <= i) continue;
                  const V3 u = pos((size_t)j);
                  const double dx = u.x - v.x, dy = u.y - v.y, dz = u.z - v.z;
                  if (dx * dx + dy * dy + dz * dz > r2) continue;  // farther than any pair of interest
                  visit(w, i, (size_t)j);
                }
              }
        }
      };
      parallel_chunks((int64_t)count, count < 4096 ? 1 : workers,
                      [&](int w, int64_t i0, int64_t i1) { range(w, (size_t)i0, (size_t)i1); });
      return;
    }
    std::vector<size_t> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::vector<V3> pts(count);
    for (size_t i = 0; i < count; i++) pts[i] = pos(i);
    struct P {
      V3 p;
    };
    std::vector<P> tmp(count);
    for (size_t i = 0; i < count; i++) tmp[i].p = pts[i];
    const int ax = count ? axis_of(tmp) : 0;
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t l, size_t r) { return coord(pts[l], ax) < coord(pts[r], ax); });
    for (size_t a = 0; a < count; a++)
      for (size_t p = a + 1; p < count && coord(pts[order[p]], ax) - coord(pts[order[a]], ax) <= reach; p++)
        visit(0, std::min(order[a], order[p]), std::max(order[a], order[p]));
  };
  // node classes: pairs of ends in contact, collected per worker, then joined
  {
    std::vector<std::vector<std::pair<size_t, size_t>>> touch(nworkers);
    grid_pairs(ends.size(), [&](size_t i) { return ends[i].p; }, thr_max, 4.0, nworkers,
               [&](int w, size_t a, size_t p) {
                 double t = std::max(ends[a].thr, ends[p].thr);
                 if (norm_l1(sub(ends[a].p, ends[p].p)) <= t) touch[w].push_back({a, p});
               });
    for (auto& lst : touch)
      for (auto& pr : lst) parent[root(ends[pr.second].idx)] = root(ends[pr.first].idx);
  }
  std::vector<std::pair<int64_t, int64_t>>& nodes = tl_nodes;
  nodes.resize(n);
  for (int64_t i = 0; i < n; i++) nodes[i] = {root(2 * i), root(2 * i + 1)};
  auto one_node = [&](int64_t s, int64_t t) {
    auto& A = nodes[s];
    auto& B = nodes[t];
    int shared = int(A.first == B.first || A.first == B.second) + int(A.second == B.first || A.second == B.second);
    return shared == 1;
  };
  // distance from a point to a segment axis, clamped to the segment
  auto axis_distance = [](const View& w, const V3& q) {
    double a0x = w.a.x, a0y = w.a.y, a0z = w.a.z, a1x = w.b.x, a1y = w.b.y, a1z = w.b.z;
    double sq = (a1x - a0x) * (a1x - a0x) + (a1y - a0y) * (a1y - a0y) + (a1z - a0z) * (a1z - a0z);
    double sa = (a1x * q.x + a1y * q.y + a1z * q.z - a0x * a1x - a0x * q.x - a0y * a1y - a0y * q.y -
                 a0z * a1z - a0z * q.z + a0x * a0x + a0y * a0y + a0z * a0z) / sq;
    if (sa < 0) sa = 0.0;
    if (sa > 1.0) sa = 1.0;
    V3 pt{a0x + (a1x - a0x) * sa, a0y + (a1y - a0y) * sa, a0z + (a1z - a0z) * sa};
    return norm3(sub(pt, q));
  };
  for (auto& v : views) {
    const V3 d = sub(v.b, v.a);
    if (d.x * d.x + d.y * d.y + d.z * d.z == 0.0) fail("nec_wire::axis_distance(): zero-length wire");
  }
  double reach = 0.0;
  for (auto& v : views) reach = std::max(reach, 0.5 * norm3(sub(v.b, v.a)) + v.r);
  // a centre inside a segment lies within `reach` of that segment's centre;
  // every violation is collected per worker
  struct Hit {
    int64_t inside, container;
    double d;
  };
  std::vector<std::vector<Hit>> hits(nworkers);
  grid_pairs(views.size(), [&](size_t i) { return views[i].c; }, reach, 2.0, nworkers, [&](int w, size_t a, size_t p) {
    if (!overlap_fatal_ || one_node(views[a].idx, views[p].idx)) return;
    const View* pairs[2][2] = {{&views[a], &views[p]}, {&views[p], &views[a]}};
    for (auto& pr : pairs) {
      const View& inside = *pr[0];
      const View& container = *pr[1];
      double d = axis_distance(container, inside.c);
      if (d > container.r) continue;
      hits[w].push_back(Hit{inside.idx, container.idx, d});
    }
  });
  size_t nhits = 0;
  for (auto& h : hits) nhits += h.size();
  if (nhits == 0) return;
  // The reported violation is the first of the reference's sweep
  // (c_geometry.cpp:1608-1633): centres in a stable order along their
  // widest axis, pairs by (anchor, probe) in that order, the anchor's centre
  // tested against the probe first.  The order is needed only here.
  V3 lo = views[0].c, hi = lo;
  for (auto& v : views) {
    lo = V3{std::min(lo.x, v.c.x), std::min(lo.y, v.c.y), std::min(lo.z, v.c.z)};
    hi = V3{std::max(hi.x, v.c.x), std::max(hi.y, v.c.y), std::max(hi.z, v.c.z)};
  }
  const double ext[3] = {hi.x - lo.x, hi.y - lo.y, hi.z - lo.z};
  int ax = 0;
  for (int k = 1; k < 3; k++)
    if (ext[k] > ext[ax]) ax = k;
  std::vector<int64_t> sorted(views.size()), rank(views.size());
  std::iota(sorted.begin(), sorted.end(), 0);
  std::stable_sort(sorted.begin(), sorted.end(),
                   [&](int64_t l, int64_t r) { return coord(views[l].c, ax) < coord(views[r].c, ax); });
  for (size_t q = 0; q < sorted.size(); q++) rank[views[sorted[q]].idx] = (int64_t)q;
  auto key = [&](const Hit& h) {
    const int64_t ri = rank[h.inside], rc = rank[h.container];
    return std::make_tuple(std::min(ri, rc), std::max(ri, rc), ri < rc ? 0 : 1);
  };
  const Hit* first = nullptr;
  for (auto& lst : hits)
    for (auto& h : lst)
      if (!first || key(h) < key(*first)) first = &h;
  const View& inside = views[first->inside];
  const View& container = views[first->container];
  char buf[256];
  snprintf(buf, sizeof(buf),
           "GEOMETRY DATA ERROR -- SEGMENT #%lld (TAG ID #%d) MIDPOINT LIES WITHIN "
           "SEGMENT #%lld (TAG ID #%d) AT DISTANCE %.5f RADIUS %.5f",
           (long long)(inside.idx + 1), inside.tag, (long long)(container.idx + 1), container.tag, first->d,
           container.r);
  throw nec_error(buf);
}

// geometry_complete, c_geometry.cpp:454-612 (wire part).
void Geometry::complete(int gpflag) {
  if (completed) fail("GEOMETRY ALREADY COMPLETE");
  if (np == 0) fail("Geometry has no wires or patches.");
  if (n <= 1)
    fail("GEOMETRY HAS ONE OR FEWER SEGMENTS and no patches. Please send bug "
         "report. This causes an error that we're trying to fix.");
  build_connections(gpflag);
  resolve_junctions();

  length.resize(n);
  cab.resize(n);
  sab.resize(n);
  salp.resize(n);
  for (int64_t i = 0; i < n; i++) {
    double xw1 = x2[i] - x[i];
    double yw1 = y2[i] - y[i];
    double zw1 = z2[i] - z[i];
    x[i] = (x[i] + x2[i]) * .5;
    y[i] = (y[i] + y2[i]) * .5;
    z[i] = (z[i] + z2[i]) * .5;
    double xw2 = xw1 * xw1 + yw1 * yw1 + zw1 * zw1;
    double yw2 = std::sqrt(xw2);
    yw2 = (xw2 / yw2 + yw2) * .5;
    length[i] = yw2;
    cab[i] = xw1 / yw2;
    sab[i] = yw1 / yw2;
    xw2 = zw1 / yw2;
    if (xw2 > 1.) xw2 = 1.;
    if (xw2 < -1.) xw2 = -1.;
    salp[i] = xw2;
    if (length[i] <= 1.e-20 || radius[i] <= 0.) fail("SEGMENT DATA ERROR");
  }
  check_overlaps();
  x_m_.assign(x.begin(), x.begin() + n);
  y_m_.assign(y.begin(), y.begin() + n);
  z_m_.assign(z.begin(), z.begin() + n);
  si_m_.assign(length.begin(), length.begin() + n);
  bi_m_.assign(radius.begin(), radius.begin() + n);
  completed = true;
}

// Scale to wavelengths, c_geometry.cpp:3389-3418.
void Geometry::frequency_scale(double freq_mhz) {
  double fr = (1.0e6 * freq_mhz) / speed_of_light();
  for (int64_t i = 0; i < n; i++) {
    x[i] = x_m_[i] * fr;
    y[i] = y_m_[i] * fr;
    z[i] = z_m_[i] * fr;
    length[i] = si_m_[i] * fr;
    radius[i] = bi_m_[i] * fr;
  }
}

// Per-segment terms used by sbf/tbf (c_geometry.cpp:2798-2812, 3132-3146,
// 2871-2886).  Two "1 - cos(2d)" forms appear in the reference and round
// differently: segments reached through a connection use 1 - cdh^2 + sdh^2,
// the segment a basis function is centred on uses 1 - (cdh^2 - sdh^2).
void Geometry::prepare_basis() {
  terms_.resize(n);
  for (int64_t i = 0; i < n; i++) {
    SegTerms& t = terms_[i];
    double d = kPi * length[i];
    t.sdh = std::sin(d);
    t.cdh = std::cos(d);
    t.sd = 2.0 * t.sdh * t.cdh;
    t.cd = t.cdh * t.cdh - t.sdh * t.sdh;
    if (d <= 0.015) {
      double omc = 4. * d * d;
      omc = ((1.3888889e-3 * omc - 4.1666666667e-2) * omc + .5) * omc;
      t.omc_link = omc;
      t.omc_self = omc;
    } else {
      t.omc_link = 1. - t.cdh * t.cdh + t.sdh * t.sdh;
      t.omc_self = 1. - t.cd;
    }
    t.aj = 1. / (std::log(1. / (kPi * radius[i])) - .577215664);
    double qp = kPi * radius[i];
    double xxi = qp * qp;
    t.xxi = qp * (1. - .5 * xxi) / (1. - xxi);
  }
}

// sbf, c_geometry.cpp:3102-3297.
void Geometry::sbf(int i, int is, double* aa, double* bb, double* cc) const {
  *aa = 0.;
  *bb = 0.;
  *cc = 0.;
  int june = 0, count = 0, njun1 = 0;
  double pp = 0., pm = 0.;
  const int ix = i - 1;
  int jcox = icon1[ix];
  if (jcox > kPatchConnection) jcox = i;
  int jend = -1, iend = -1;
  double sig = -1.;
  do {
    if (jcox != 0) {
      if (jcox < 0)
        jcox = -jcox;
      else {
        sig = -sig;
        jend = -jend;
      }
      const int jcoxx = jcox - 1;
      count++;
      const SegTerms& t = terms_[jcoxx];
      pp -= t.omc_link / t.sd * t.aj;
      if (jcox == is) {
        *aa = t.aj / t.sd * sig;
        *bb = t.aj / (2. * t.cdh);
        *cc = -t.aj / (2. * t.sdh) * sig;
        june = iend;
      }
      if (jcox != i) {
        jcox = (jend != 1) ? icon1[jcoxx] : icon2[jcoxx];
        if (std::abs(jcox) != i) {
          if (jcox == 0) fail("SBF - SEGMENT CONNECTION ERROR FOR SEGMENT ", i);
          continue;
        }
      } else if (jcox == is) {
        *bb = -*bb;
      }
      if (iend == 1) break;
    }
    pm = -pp;
    pp = 0.;
    njun1 = count;
    jcox = icon2[ix];
    if (jcox > kPatchConnection) jcox = i;
    jend = 1;
    iend = 1;
    sig = -1.;
  } while (jcox != 0);

  const int njun2 = count - njun1;
  const SegTerms& t = terms_[ix];
  const double sdh = t.sdh, cdh = t.cdh, sd = t.sd, cd = t.cd, omc = t.omc_self;
  const double ap = t.aj, aj = t.aj, xxi = t.xxi;
  if (njun1 == 0) {
    if (njun2 == 0) {
      *aa = -1.;
      *cc = 1. / (cdh - xxi * sdh);
      return;
    }
    double qp = -(omc + xxi * sd) / (sd * (ap + xxi * pp) + cd * (xxi * ap - pp));
    if (june == 1) {
      *aa = -*aa * qp;
      *bb = *bb * qp;
      *cc = -*cc * qp;
      if (i != is) return;
    }
    *aa -= 1.;
    double d = cd - xxi * sd;
    *bb += (sdh + ap * qp * (cdh - xxi * sdh)) / d;
    *cc += (cdh + ap * qp * (sdh + xxi * cdh)) / d;
    return;
  }
  if (njun2 == 0) {
    double qm = (omc + xxi * sd) / (sd * (aj - xxi * pm) + cd * (pm + xxi * aj));
    if (june == -1) {
      *aa = *aa * qm;
      *bb = *bb * qm;
      *cc = *cc * qm;
      if (i != is) return;
    }
    *aa -= 1.;
    double d = cd - xxi * sd;
    *bb += (aj * qm * (cdh - xxi * sdh) - sdh) / d;
    *cc += (cdh - aj * qm * (sdh + xxi * cdh)) / d;
    return;
  }
  double qp = sd * (pm * pp + aj * ap) + cd * (pm * ap - pp * aj);
  double qm = (ap * omc - pp * sd) / qp;
  qp = -(aj * omc + pm * sd) / qp;
  if (june != 0) {
    if (june < 0) {
      *aa = *aa * qm;
      *bb = *bb * qm;
      *cc = *cc * qm;
    } else {
      *aa = -*aa * qp;
      *bb = *bb * qp;
      *cc = -*cc * qp;
    }
    if (i != is) return;
  }
  *aa -= 1.;
  *bb += (aj * qm + ap * qp) * sdh / sd;
  *cc += (aj * qm - ap * qp) * cdh / sd;
}

// trio, c_geometry.cpp:2982-3100: every basis function with support on
// source segment j, the segment's own basis function last.
void Geometry::trio(int j, std::vector<BasisEntry>& out) const {
  out.clear();
  BasisEntry e;
  const int jx = j - 1;
  int jend = 0, iend = 0;
  int jcox = icon1[jx];
  if (jcox <= kPatchConnection) {
    jend = -1;
    iend = -1;
  }
  if (jcox == 0 || jcox > kPatchConnection) {
    jcox = icon2[jx];
    if (jcox <= kPatchConnection) {
      jend = 1;
      iend = 1;
    }
    if (jcox == 0 || jcox > kPatchConnection) {
      sbf(j, j, &e.a, &e.b, &e.c);
      e.basis = j;
      out.push_back(e);
      return;
    }
  }
  do {
    if (jcox < 0)
      jcox = -jcox;
    else
      jend = -jend;
    const int jcoxx = jcox - 1;
    if (jcox != j) {
      sbf(jcox, j, &e.a, &e.b, &e.c);
      e.basis = jcox;
      out.push_back(e);
      jcox = (jend != 1) ? icon1[jcoxx] : icon2[jcoxx];
      if (jcox == 0) fail("TRIO - SEGMENT CONNENTION ERROR FOR SEGMENT ", j);
      continue;
    }
    if (iend == 1) break;
    jcox = icon2[jx];
    if (jcox > kPatchConnection) break;
    jend = 1;
    iend = 1;
  } while (jcox != 0);
  sbf(j, j, &e.a, &e.b, &e.c);
  e.basis = j;
  out.push_back(e);
}

// tbf, c_geometry.cpp:2763-2980: the basis function centred on segment i
// over every segment it covers (connected ends first, segment i last).
// Entries carry the covered segment in .basis.
void Geometry::tbf(int i, int icap, std::vector<BasisEntry>& out) const {
  out.clear();
  double pp = 0.0, pm = 0.0;
  int njun1 = 0;
  const int ix = i - 1;
  int jcox = icon1[ix];
  if (jcox > kPatchConnection) jcox = i;
  int jend = -1, iend = -1;
  double sig = -1.0;
  do {
    if (jcox != 0) {
      if (jcox < 0)
        jcox = -jcox;
      else {
        sig = -sig;
        jend = -jend;
      }
      const int jcoxx = jcox - 1;
      const SegTerms& t = terms_[jcoxx];
      pp = pp - t.omc_link / t.sd * t.aj;
      BasisEntry e;
      e.basis = jcox;
      e.a = t.aj / t.sd * sig;
      e.b = t.aj / (2. * t.cdh);
      e.c = -t.aj / (2. * t.sdh) * sig;
      out.push_back(e);
      if (jcox != i) {
        jcox = (jend == 1) ? icon2[jcoxx] : icon1[jcoxx];
        if (std::abs(jcox) != i) {
          if (jcox != 0) continue;
          fail("TBF - SEGMENT CONNECTION ERROR FOR SEGMENT ", i);
        }
      } else {
        out.back().b = -out.back().b;
      }
      if (iend == 1) break;
    }
    pm = -pp;
    pp = 0.;
    njun1 = (int)out.size();
    jcox = icon2[ix];
    if (jcox > kPatchConnection) jcox = i;
    jend = 1;
    iend = 1;
    sig = -1.;
  } while (jcox != 0);

  const int jsno = (int)out.size();
  const int njun2 = jsno - njun1;
  const SegTerms& t = terms_[ix];
  const double sdh = t.sdh, cdh = t.cdh, sd = t.sd, cd = t.cd, omc = t.omc_self;
  const double ap = t.aj, aj = t.aj;
  const double xxi = (icap == 0) ? 0. : t.xxi;
  BasisEntry self;
  self.basis = i;
  self.a = -1.;
  if (njun1 == 0) {
    if (njun2 == 0) {
      self.b = 0.;
      self.c = 1. / (cdh - xxi * sdh);
      out.push_back(self);
      return;
    }
    double qp = -(omc + xxi * sd) / (sd * (ap + xxi * pp) + cd * (xxi * ap - pp));
    double d = cd - xxi * sd;
    self.b = (sdh + ap * qp * (cdh - xxi * sdh)) / d;
    self.c = (cdh + ap * qp * (sdh + xxi * cdh)) / d;
    for (int k = 0; k < njun2; k++) {
      out[k].a = -out[k].a * qp;
      out[k].b = out[k].b * qp;
      out[k].c = -out[k].c * qp;
    }
    out.push_back(self);
    return;
  }
  if (njun2 == 0) {
    double qm = (omc + xxi * sd) / (sd * (aj - xxi * pm) + cd * (pm + xxi * aj));
    double d = cd - xxi * sd;
    self.b = (aj * qm * (cdh - xxi * sdh) - sdh) / d;
    self.c = (cdh - aj * qm * (sdh + xxi * cdh)) / d;
    for (int k = 0; k < njun1; k++) {
      out[k].a = out[k].a * qm;
      out[k].b = out[k].b * qm;
      out[k].c = out[k].c * qm;
    }
    out.push_back(self);
    return;
  }
  double qp = sd * (pm * pp + aj * ap) + cd * (pm * ap - pp * aj);
  double qm = (ap * omc - pp * sd) / qp;
  qp = -(aj * omc + pm * sd) / qp;
  self.b = (aj * qm + ap * qp) * sdh / sd;
  self.c = (aj * qm - ap * qp) * cdh / sd;
  for (int k = 0; k < njun1; k++) {
    out[k].a = out[k].a * qm;
    out[k].b = out[k].b * qm;
    out[k].c = out[k].c * qm;
  }
  for (int k = njun1; k < jsno; k++) {
    out[k].a = -out[k].a * qp;
    out[k].b = out[k].b * qp;
    out[k].c = -out[k].c * qp;
  }
  out.push_back(self);
}

// c_geometry.cpp:3449-3458.
int Geometry::test_ek_approximation(int seg1, int seg2) const {
  double ratio = radius[seg2] / radius[seg1];
  double xi = std::fabs(cab[seg1] * cab[seg2] + sab[seg1] * sab[seg2] + salp[seg1] * salp[seg2]);
  if (xi < 0.999999 || std::fabs(ratio - 1.0) > 1.e-6) return 2;
  return 0;
}

}  // namespace necb
