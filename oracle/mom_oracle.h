/*
 * mom_oracle -- CPU restatement of the NEC2++ thin-wire hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the GPU path is compared
 * against; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load it.  The product (libnecpp_b200.so) never calls it.
 *
 * Plain C99 with GCC complex arithmetic (the same builtins libstdc++'s
 * std::complex<double> uses), compiled without contraction or fast-math, so
 * it reproduces the reference's rounding.  Pinned against the reference build
 * (oracle/_ref) and the committed golden fixtures by tests/test_oracle.py.
 */
#ifndef MOM_ORACLE_H
#define MOM_ORACLE_H
#include <stdint.h>

/* Interpolation cache of the Sommerfeld tables (the reference's c_ggrid
   m_ip_* members, src/c_ggrid.h:70-76). */
typedef struct mo_interp {
  int ix, iy, ixs, iys, igrs, ixeg, iyeg;
  int nxm2, nym2, nxms, nyms, nd, ndp;
  double dx, dy, xs, ys, xz, yz;
  double a[32], b[32], c[32], d[32]; /* 4x4 complex each */
} mo_interp;

typedef struct mo_structure {
  int64_t n;
  const double *x, *y, *z, *s, *b, *cab, *sab, *salp; /* wavelengths */
  const int32_t* trio_ptr;                           /* n+1 */
  const int32_t* trio_basis;                         /* 0-based */
  const double *trio_a, *trio_b, *trio_c;
  const int32_t *ind1, *ind2; /* extended-kernel end flags (or NULL) */
  double rkh;
  int use_exk;
  int ground; /* 0 none, 1 perfect, 2 reflection coefficient, 3 Sommerfeld/Norton */
  double zrati_re, zrati_im, frati_re, frati_im;
  double eta;
  /* impedance loading per segment (n complex, re/im interleaved; the
     reference's zarray after load(), src/nec_context.cpp:1861-2072), or NULL */
  const double* zload;
  /* Sommerfeld ground tables (1068 complex: grids of 11x10, 17x5, 9x8 points,
     4 functions each; mo_sommerfeld) for pairs closer than ~1 wavelength to
     the image, or NULL; the interpolation cache they are read through and
     whether it keeps the reference's state between points */
  const double* somm;
  mo_interp* interp;
  int interp_stateful;
} mo_structure;

/* Fill: z[obs*n + basis] (interleaved re, im); returns status bits
   (1 step-size limited, 4 Sommerfeld table path needed). */
int mo_fill(const mo_structure* s, double* z);
/* Unblocked LU with partial pivoting in place; piv[k] = row swapped with k. */
int mo_lu(int64_t n, double* a, int32_t* piv);
/* Solve with the factors: b overwritten by the solution. */
void mo_solve(int64_t n, const double* lu, const int32_t* piv, double* b);
/* Current coefficients (6n: air aii bir bii cir cii) and segment-centre
   currents cur (n complex) from the basis amplitudes x (n complex). */
void mo_coefficients(const mo_structure* s, const double* x, double* abc, double* cur);
/* Sommerfeld ground tables for relative permittivity epr, conductivity sig
   (S/m; negative: the imaginary part itself) at this wavelength (m); eta is
   the medium impedance.  tables: 1068 complex; epscf: the complex
   permittivity used.  Returns 1 when an integral did not converge. */
int mo_sommerfeld(double epr, double sig, double wavelength, double eta, double* tables, double* epscf);
int64_t mo_interp_size(void);
void mo_interp_init(mo_interp* s);
/* The four interpolated functions (erv, ezv, erh, eph; complex) at
   R = x (wavelengths), theta = y (radians). */
void mo_interpolate(mo_interp* s, const double* tables, double x, double y, int stateful, double* f);
/* Near electric (nefld) and magnetic (nhfld) field at a point (wavelengths)
   from current coefficients abc: out = 3 complex (x, y, z), interleaved. */
void mo_nefld(const mo_structure* s, const double* abc, double x, double y, double z, double* out);
void mo_nhfld(const mo_structure* s, const double* abc, double x, double y, double z, double* out);
/* Far field at (thet, phi) radians: eth, eph (complex, interleaved). */
void mo_ffld(const mo_structure* s, const double* abc, double thet, double phi, double* eth,
             double* eph);

#endif
