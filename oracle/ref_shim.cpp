/*
 * Test-harness shim around the UNMODIFIED NEC2++ reference, compiled from the
 * reference's own sources by oracle/Makefile into oracle/_ref/libnecpp_ref.so.
 *
 * This file is test infrastructure.  It is only loaded by tests/, the CPU
 * baseline leg of bench.py and the fixture generator in tests/golden/.  It
 * exposes, over plain C, the pieces of the reference that the public C API
 * (src/libnecpp.h) does not reach:
 *   - c_geometry::helix (src/c_geometry.cpp:698-826; only in the C++ API,
 *     src/nec_context.h:449-450),
 *   - the segment arrays and the connection tables icon1/icon2
 *     (src/c_geometry.h:201-219),
 *   - the per-source-segment basis tables from c_geometry::trio
 *     (src/c_geometry.cpp:2982-3100),
 *   - the unfactored interaction matrix produced by nec_context::cmset
 *     (src/nec_context.cpp:2077-2204), the LU factors and pivots left in the
 *     public members cm / ip (src/nec_context.h:834-842),
 *   - the currents and current coefficients (src/nec_context.h:846-849),
 *   - the far-field sum ffld (src/nec_context.cpp:6639-6888),
 *   - the Sommerfeld ground tables and their interpolation cache
 *     (src/c_ggrid.h:36-76).
 *
 * cmset is a private member; it is reached through the standard
 * explicit-instantiation access idiom (a member pointer named in an explicit
 * template instantiation), which leaves the reference's headers untouched.
 */
#include "nec_context.h"
#include "c_geometry.h"
#include "libnecpp.h"

#include <complex>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

namespace {

template <typename Tag, typename Tag::type M>
struct member_access {
  friend typename Tag::type access_member(Tag) { return M; }
};

struct cmset_tag {
  typedef void (nec_context::*type)(int64_t, complex_array&, nec_float);
  friend type access_member(cmset_tag);
};
template struct member_access<cmset_tag, &nec_context::cmset>;

struct ggrid_tag {
  typedef c_ggrid nec_ground::*type;
  friend type access_member(ggrid_tag);
};
template struct member_access<ggrid_tag, &nec_ground::_ggrid>;

c_ggrid& ggrid_of(nec_context* ctx) { return ctx->ground.*access_member(ggrid_tag()); }

}  // namespace

extern "C" {

/* nec_create (src/libNEC.cpp:33-38) constructed in zero-filled storage.
   Probe helper: decides whether a crash depends on members the reference
   leaves uninitialised. */
nec_context* ref_create_zeroed(void) {
  void* mem = calloc(1, sizeof(nec_context));
  nec_context* ctx = new (mem) nec_context();
  ctx->initialize();
  return ctx;
}

long ref_helix(nec_context* ctx, int tag, int nseg, double s, double hl,
               double a1, double b1, double a2, double b2, double rad) {
  try {
    ctx->helix(tag, nseg, s, hl, a1, b1, a2, b2, rad);
  } catch (const nec_exception&) {
    return 1;
  }
  return 0;
}

long ref_n_segments(nec_context* ctx) {
  return (long)ctx->get_geometry()->n_segments;
}

/* Segment arrays as they stand now (metres right after geometry_complete,
   wavelengths after a simulation has scaled them). */
void ref_segments(nec_context* ctx, double* x, double* y, double* z,
                  double* si, double* bi, double* cab, double* sab,
                  double* salp, int* tags, int* icon1, int* icon2) {
  c_geometry* g = ctx->get_geometry();
  for (int64_t i = 0; i < g->n_segments; i++) {
    x[i] = g->x[i];
    y[i] = g->y[i];
    z[i] = g->z[i];
    si[i] = g->segment_length[i];
    bi[i] = g->segment_radius[i];
    cab[i] = g->cab[i];
    sab[i] = g->sab[i];
    salp[i] = g->salp[i];
    tags[i] = g->segment_tags[i];
    icon1[i] = g->icon1[i];
    icon2[i] = g->icon2[i];
  }
}

/* Segment end points (x,y,z) and (x2,y2,z2) after connection snapping. */
void ref_segment_ends(nec_context* ctx, double* x1, double* y1, double* z1,
                      double* x2, double* y2, double* z2) {
  c_geometry* g = ctx->get_geometry();
  for (int64_t i = 0; i < g->n_segments; i++) {
    x1[i] = g->x[i] - 0.5 * g->segment_length[i] * g->cab[i];
    y1[i] = g->y[i] - 0.5 * g->segment_length[i] * g->sab[i];
    z1[i] = g->z[i] - 0.5 * g->segment_length[i] * g->salp[i];
    x2[i] = g->x[i] + 0.5 * g->segment_length[i] * g->cab[i];
    y2[i] = g->y[i] + 0.5 * g->segment_length[i] * g->sab[i];
    z2[i] = g->z[i] + 0.5 * g->segment_length[i] * g->salp[i];
  }
}

/* Basis table of source segment j (1-based) from trio(): returns jsno and
   writes jsno entries of jco (1-based basis index) and ax/bx/cx. */
int ref_trio(nec_context* ctx, int j, int* jco, double* ax, double* bx,
             double* cx) {
  c_geometry* g = ctx->get_geometry();
  g->trio(j);
  for (int k = 0; k < g->jsno; k++) {
    jco[k] = g->jco[k];
    ax[k] = g->ax[k];
    bx[k] = g->bx[k];
    cx[k] = g->cx[k];
  }
  return g->jsno;
}

/* Basis function i (1-based) across segments from tbf(i, icap). */
int ref_tbf(nec_context* ctx, int i, int icap, int* jco, double* ax,
            double* bx, double* cx) {
  c_geometry* g = ctx->get_geometry();
  g->tbf(i, icap);
  for (int k = 0; k < g->jsno; k++) {
    jco[k] = g->jco[k];
    ax[k] = g->ax[k];
    bx[k] = g->bx[k];
    cx[k] = g->cx[k];
  }
  return g->jsno;
}

double ref_wavelength(nec_context* ctx) { return ctx->_wavelength; }

/* Refill the interaction matrix with the reference's own cmset at the
   frequency and ground of the last simulation and copy it out.  The layout
   is the reference's: out[basis + obs*n] (interleaved re, im). */
long ref_fill(nec_context* ctx, double* out) {
  try {
    int64_t n = ctx->neq;
    (ctx->*access_member(cmset_tag()))(n, ctx->cm, ctx->rkh);
    for (int64_t k = 0; k < n * n; k++) {
      out[2 * k] = ctx->cm[k].real();
      out[2 * k + 1] = ctx->cm[k].imag();
    }
  } catch (const nec_exception&) {
    return 1;
  }
  return 0;
}

/* The Sommerfeld ground tables of the last frequency (c_ggrid::sommerfeld,
   src/c_ggrid.cpp:164-288): ar1 (440), ar2 (340), ar3 (288) complex values,
   interleaved re/im, and the complex permittivity they were made for. */
void ref_somm_tables(nec_context* ctx, double* out, double* epscf) {
  c_ggrid& g = ggrid_of(ctx);
  int64_t k = 0;
  for (const complex_array* a : {&g.m_ar1, &g.m_ar2, &g.m_ar3})
    for (int64_t i = 0; i < a->size(); i++, k++) {
      out[2 * k] = (*a)[i].real();
      out[2 * k + 1] = (*a)[i].imag();
    }
  epscf[0] = g.m_epscf.real();
  epscf[1] = g.m_epscf.imag();
}

/* Reset the interpolation cache to the state a new context starts with
   (c_ggrid::initialize, src/c_ggrid.h:45-61; the tables are kept). */
void ref_somm_interp_reset(nec_context* ctx) { ggrid_of(ctx).initialize(); }

/* One call of c_ggrid::interpolate (src/c_ggrid.cpp:38-162) through the
   context's cache: f = erv, ezv, erh, eph interleaved. */
void ref_somm_interpolate(nec_context* ctx, double x, double y, double* f) {
  nec_complex a, b, c, d;
  ggrid_of(ctx).interpolate(x, y, &a, &b, &c, &d);
  const nec_complex v[4] = {a, b, c, d};
  for (int k = 0; k < 4; k++) {
    f[2 * k] = v[k].real();
    f[2 * k + 1] = v[k].imag();
  }
}

/* Near-field pattern `index` (nfpat, src/nec_context.cpp:5068-5186): its
   kind (0 electric, 1 magnetic) and point count; with non-null buffers the
   points (metres, 3 per point) and fields (3 complex per point). */
long ref_near_field(nec_context* ctx, long index, int* nfeh, double* xyz, double* f) {
  nec_near_field_pattern* p = ctx->get_near_field_pattern(index);
  if (!p) return -1;
  std::vector<nec_float> x = p->get_x(), y = p->get_y(), z = p->get_z();
  std::vector<nec_complex> fx = p->get_field_x(), fy = p->get_field_y(), fz = p->get_field_z();
  if (nfeh) *nfeh = p->get_nfeh();
  const long np = (long)x.size();
  for (long i = 0; xyz && i < np; i++) {
    xyz[3 * i] = x[i];
    xyz[3 * i + 1] = y[i];
    xyz[3 * i + 2] = z[i];
  }
  for (long i = 0; f && i < np; i++) {
    const nec_complex v[3] = {fx[i], fy[i], fz[i]};
    for (int k = 0; k < 3; k++) {
      f[6 * i + 2 * k] = v[k].real();
      f[6 * i + 2 * k + 1] = v[k].imag();
    }
  }
  return np;
}

/* LU factors (column-major, in place) and the 1-based permutation left by the
   last factorisation. */
void ref_lu(nec_context* ctx, double* out, int* ip) {
  int64_t n = ctx->neq;
  for (int64_t k = 0; k < n * n; k++) {
    out[2 * k] = ctx->cm[k].real();
    out[2 * k + 1] = ctx->cm[k].imag();
  }
  for (int64_t k = 0; k < n; k++) ip[k] = ctx->ip[k];
}

/* Segment-centre currents (current_vector, in units of the reference,
   i.e. amperes divided by wavelength) and the current coefficients. */
void ref_currents(nec_context* ctx, double* cur, double* air, double* aii,
                  double* bir, double* bii, double* cir, double* cii) {
  int64_t n = ctx->get_geometry()->n_segments;
  for (int64_t i = 0; i < n; i++) {
    cur[2 * i] = ctx->current_vector[i].real();
    cur[2 * i + 1] = ctx->current_vector[i].imag();
    air[i] = ctx->air[i];
    aii[i] = ctx->aii[i];
    bir[i] = ctx->bir[i];
    bii[i] = ctx->bii[i];
    cir[i] = ctx->cir[i];
    cii[i] = ctx->cii[i];
  }
}

/* Far-field sum at one direction (radians), from the last solution. */
void ref_ffld(nec_context* ctx, double thet, double phi, double* eth,
              double* eph) {
  nec_complex a, b;
  ctx->ffld(thet, phi, &a, &b, ctx->_wavelength);
  eth[0] = a.real();
  eth[1] = a.imag();
  eph[0] = b.real();
  eph[1] = b.imag();
}

}  // extern "C"
