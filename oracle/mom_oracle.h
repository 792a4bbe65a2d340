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
/* Far field at (thet, phi) radians: eth, eph (complex, interleaved). */
void mo_ffld(const mo_structure* s, const double* abc, double thet, double phi, double* eth,
             double* eph);

#endif
