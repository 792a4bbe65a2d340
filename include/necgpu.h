/*
 * necgpu -- C-ABI of the sm_100a kernels behind the NEC2++ thin-wire hot path.
 *
 * The host library (libnecpp_b200.so, which also exports the libnecpp.h API)
 * calls these at the three points where NEC2++ runs its hot path:
 *
 *   nec_context::structure_segment_loading  (src/nec_context.cpp:1523-1558)
 *       cmset (fill, 2077-2204) + factrs (LU, src/matrix_algebra.cpp:319-338)
 *       -> necgpu_set_structure, necgpu_fill, necgpu_factor
 *   nec_context::netwk_compute_currents     (src/nec_context.cpp:4850-4935)
 *       solves (src/matrix_algebra.cpp:351-503) +
 *       c_geometry::get_current_coefficients (src/c_geometry.cpp:3299-3387)
 *       -> necgpu_solve
 *   nec_context::excitation_compute_far_field (src/nec_context.cpp:1761-1790)
 *       ffld (6639-6888) inside nec_radiation_pattern::analyze
 *       (src/nec_radiation_pattern.cpp:209-450)
 *       -> necgpu_pattern
 *
 * Plain pointers and sizes only.  Every function returns 0 on success and a
 * non-zero NECGPU_* status on failure; necgpu_last_error() gives the text.
 * There is no CPU fallback: without a usable CUDA device necgpu_create fails.
 */
#ifndef NECGPU_H
#define NECGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum necgpu_status {
  NECGPU_OK = 0,
  NECGPU_ERR_CUDA = 1,        /* a CUDA call failed */
  NECGPU_ERR_ARG = 2,         /* bad argument or call order */
  NECGPU_ERR_SINGULAR = 3,    /* zero pivot met in the factorisation */
  NECGPU_ERR_NONFINITE = 4,   /* NaN / Inf in the matrix or solution */
  NECGPU_ERR_REFINE = 5,      /* iterative refinement did not converge */
  NECGPU_ERR_UNSUPPORTED = 6, /* a kernel path this build does not provide */
  NECGPU_ERR_NO_DEVICE = 7
};

enum necgpu_precision {
  NECGPU_FP64 = 0,  /* complex128 fill, LU and solve */
  NECGPU_MIXED = 1  /* complex64 LU (tensor-core trailing update) + FP64 refinement */
};

enum necgpu_ground {
  NECGPU_GROUND_NONE = 0,
  NECGPU_GROUND_PERFECT = 1,
  NECGPU_GROUND_REFLECTION = 2, /* finite ground, reflection-coefficient approximation */
  NECGPU_GROUND_SOMMERFELD = 3  /* finite ground, Sommerfeld/Norton (Norton branch) */
};

/* One structure at one frequency.  Lengths are in wavelengths, as after
 * c_geometry::frequency_scale.  Basis tables are the per-source-segment lists
 * of c_geometry::trio (src/c_geometry.cpp:2982-3100) in CSR form with
 * 0-based basis indices. */
typedef struct necgpu_structure {
  int64_t n;
  const double *x, *y, *z, *length, *radius, *cab, *sab, *salp;
  const int32_t* trio_ptr; /* n+1 */
  const int32_t* trio_basis;
  const double *trio_a, *trio_b, *trio_c;
  const int32_t* ek_ind1; /* extended-kernel end flags per source segment (or NULL) */
  const int32_t* ek_ind2;
  double rkh;   /* far-pair threshold in wavelengths (KH card) */
  int32_t use_exk;
  int32_t ground; /* necgpu_ground */
  double zrati_re, zrati_im; /* 1/sqrt(eps_c) */
  double frati_re, frati_im; /* image scale factor */
  double eta;   /* wave impedance of the medium, sqrt(mu/eps) (src/electromag.cpp:31-35) */
} necgpu_structure;

typedef struct necgpu_engine necgpu_engine;

/* Replaces: nothing in the reference (the reference has no device state);
 * owned per nec_context and released by nec_delete (src/libNEC.cpp:40-42). */
int necgpu_create(necgpu_engine** out, int device);
int necgpu_destroy(necgpu_engine* e);
/* Engine reuse between short-lived users (nec_context does this): acquire
 * takes the device's pooled engine if there is one (else creates one);
 * release returns an engine to the pool, one per device, keeping its
 * streams, buffers and captured LU graph but none of its results, tables
 * or statistics.  An engine whose settings were changed (stream, timing,
 * refinement, pivoting, update format, tuning, resident inputs) or that ran
 * a test, batch, matrix or allocation-free entry point is destroyed
 * instead, as is one whose stream reports an error. */
int necgpu_acquire(necgpu_engine** out, int device);
int necgpu_release(necgpu_engine* e);
const char* necgpu_last_error(const necgpu_engine* e);

/* Use the given cudaStream_t (as void*) for all work; NULL = the engine's own
 * stream. */
int necgpu_set_stream(necgpu_engine* e, void* stream);

/* Upload one structure (host arrays, copied). */
int necgpu_set_structure(necgpu_engine* e, const necgpu_structure* s);

/* Impedance loading of the structure set last (n complex: the reference's
 * zarray, lambda x impedance per unit length, from load(),
 * src/nec_context.cpp:1861-2072), applied by every later necgpu_fill as
 * cmset does (2127-2142); NULL removes it.  necgpu_set_structure clears it. */
int necgpu_set_loads(necgpu_engine* e, const double* zload);

/* Sommerfeld ground (structure ground type 3): computes on the device the
   tables of the ground's reflected field for complex relative permittivity
   eps_re + j eps_im (the reference's epscf) at the structure's medium
   impedance; the next fills integrate them for segment pairs within
   0.95 wavelength^2 (squared distance) of their image.  Replaces
   c_ggrid::sommerfeld (src/c_ggrid.cpp:164-288) as called from
   nec_ground::calculate_antenna_environment (src/nec_ground.cpp:204-209).
   The tables belong to one structure and frequency: call after every
   necgpu_set_structure.  The interpolation cache that the fill reads them
   through persists across fills, as the reference's does
   (src/c_ggrid.cpp:38-162). */
int necgpu_set_sommerfeld(necgpu_engine* e, double eps_re, double eps_im);
/* The tables (1068 complex, interleaved re/im: grids of 11x10, 17x5 and
   9x8 points, 4 functions each, in the reference's m_ar1..m_ar3 layout). */
int necgpu_copy_sommerfeld(necgpu_engine* e, double* tables);
/* Returns the interpolation cache to the state of a new context. */
int necgpu_reset_interpolation(necgpu_engine* e);

/* Near field of the last solution at npts points (pts: x, y, z per point in
   wavelengths): magnetic = 0 the electric field (nefld,
   src/nec_context.cpp:4304-4490), 1 the magnetic field (nhfld, 5189-5265).
   fields: 3 complex per point (x, y, z; interleaved re/im), in the units of
   the reference's nec_near_field_pattern.  With Sommerfeld ground the points
   are taken in the given order through the tables' interpolation cache, as
   nfpat takes them. */
int necgpu_near_field(necgpu_engine* e, int magnetic, int npts, const double* pts, double* fields);

/* Replaces cmset (src/nec_context.cpp:2077-2204) for wires: fills Z on the
 * device, row-major, Z[obs*n + basis] = field at obs due to basis (the
 * reference's cm layout). */
int necgpu_fill(necgpu_engine* e);

/* Announce the precision of the factorisations that follow the next fills
 * (-1: unknown, the default).  With NECGPU_MIXED the fill also writes the
 * complex64 copy the mixed LU factors, and the factorisation skips its
 * demotion pass (not for loaded structures, whose loads are applied to the
 * FP64 matrix after the fill).  Results are the same either way. */
int necgpu_set_fill_precision(necgpu_engine* e, int precision);

/* Replaces factrs/lu_decompose (src/matrix_algebra.cpp:217-266, 319-338):
 * LU with partial pivoting of the filled Z in the requested precision. */
int necgpu_factor(necgpu_engine* e, int precision);

/* Replaces solves/solve (src/matrix_algebra.cpp:271-307, 351-503) and
 * get_current_coefficients (src/c_geometry.cpp:3299-3387).  rhs: n complex
 * (interleaved re,im) applied field; cur: n complex segment-centre currents
 * (the reference's current_vector after the call); abc: if not NULL, 6*n
 * doubles air,aii,bir,bii,cir,cii.  Mixed precision refines the solution in
 * FP64 against the FP64 Z until the relative residual drops below tol. */
int necgpu_solve(necgpu_engine* e, const double* rhs, double* cur, double* abc);

/* Replaces the ffld loop of nec_radiation_pattern::analyze
 * (src/nec_context.cpp:6639-6888, src/nec_radiation_pattern.cpp:281-283):
 * far field of the last solution at n_dir directions (radians).
 * eth/eph: n_dir complex each.  ksymp/ground describe the image (the ground
 * of necgpu_structure is used). */
int necgpu_pattern(necgpu_engine* e, int n_dir, const double* theta,
                   const double* phi, double* eth, double* eph);

/* Refinement controls for NECGPU_MIXED (defaults: 1e-13, 30). */
int necgpu_set_refinement(necgpu_engine* e, double tol, int max_iter);
/* Pivoting of the NECGPU_MIXED factorisation.  1 (default): pivots chosen
 * inside each 64-row diagonal block; the FP64 refinement absorbs the extra
 * growth, and a refinement that stalls above 1e-10 (or a zero pivot in a
 * block) refactors with 0: partial pivoting over the whole column, the
 * reference's choice.  NECGPU_FP64 always uses partial pivoting. */
int necgpu_set_pivoting(necgpu_engine* e, int mode);
/* Operand format of the NECGPU_MIXED factorisation's tensor-core update.
 * 1: complex64 operands split into BF16 hi/lo parts, three products per
 * pair (~2^-16 relative); 2: one TF32 pass (~2^-11 relative, two thirds of
 * the tensor-core time; the refinement takes a step or more extra);
 * 0 (default): TF32 from 10,240 unknowns on (NECPP_B200_TF32_MIN_N), split
 * BF16 below that and, for the rest of the engine's life, after a TF32
 * factorisation whose refinement needed more than 5 steps or stalled (the
 * solve then refactors with split BF16).  The environment variable
 * NECPP_B200_TC_FORMAT (bf16x3, tf32, auto) sets it at engine creation. */
int necgpu_set_update_format(necgpu_engine* e, int format);
/* Format (1 or 2) of the held NECGPU_MIXED factors; 0 when none are held. */
int necgpu_update_format(const necgpu_engine* e);

/* Diagnostics of the last necgpu_solve / necgpu_factor. */
enum necgpu_kernel_class {
  NECGPU_K_FILL = 0,
  NECGPU_K_PANEL = 1,   /* LU panel factorisation */
  NECGPU_K_LASWP = 2,   /* row interchanges */
  NECGPU_K_TRSM = 3,    /* U12 = L11^-1 A12 */
  NECGPU_K_GEMM = 4,    /* trailing update A22 -= L21 U12 */
  NECGPU_K_TRSV = 5,    /* triangular solves */
  NECGPU_K_RESID = 6,   /* FP64 refinement residual */
  NECGPU_K_PATTERN = 7, /* far-field sum */
  NECGPU_K_OTHER = 8,
  NECGPU_K_COUNT = 9
};

typedef struct necgpu_stats {
  int refine_iters;
  double refine_residual;   /* final ||b - Z x|| / ||b|| (FP64) */
  double ms_fill, ms_factor, ms_solve, ms_pattern; /* last timings (0 if not timed) */
  int64_t launches;         /* kernels launched by the engine since create */
  int64_t h2d_bytes, d2h_bytes; /* host<->device bytes copied since create (or acquire) */
  /* per kernel class, accumulated while kernel timing is on: CUDA-event time
     of every launch (ms), launch count, algorithmic flops of the launches */
  double k_ms[NECGPU_K_COUNT];
  int64_t k_launches[NECGPU_K_COUNT];
  double k_flops[NECGPU_K_COUNT];
  /* pivoting of the last mixed factorisation: 0 partial (whole column),
     1 block-local (64-row diagonal block; refined in FP64, falls back to 0) */
  int pivoting;
  /* near-ground fills (Sommerfeld tables): rounds of the last fill's column
     scan (1: every column was right from a fresh interpolation cache) */
  int near_passes;
} necgpu_stats;
int necgpu_get_stats(const necgpu_engine* e, necgpu_stats* out);
/* 1: time each stage (fill / factor / solve / pattern) with CUDA events.
   2: additionally time every kernel launch by class (events around each
      launch on the stream it runs on; accumulated into k_ms / k_launches).
   3: additionally keep a trace of every timed launch (necgpu_get_trace). */
int necgpu_enable_timing(necgpu_engine* e, int on);
/* Clears the per-class sums and the trace; the next traced launch sets the
   trace's time origin. */
int necgpu_reset_kernel_stats(necgpu_engine* e);

/* One launch of the trace: class (necgpu_kernel_class), stream (0 the
   engine's, 2 the lookahead's far update, 3 the U12 panel solves, 4 the
   panel solves and updates below the next panel's rows, 1 other),
   start and end in ms after the trace origin, its algorithmic work (the unit
   of its class) and the launch expression (truncated). */
typedef struct necgpu_trace_rec {
  int cls;
  int stream;
  float start_ms, end_ms;
  double work;
  char name[48];
} necgpu_trace_rec;
/* Copies up to cap records of the trace (timing level 3, read after the
   stages have synchronised) and returns how many there are. */
int necgpu_get_trace(necgpu_engine* e, necgpu_trace_rec* out, int cap);
/* Make the last right-hand side and direction list passed to necgpu_solve /
   necgpu_pattern the resident inputs of necgpu_step_resident. */
int necgpu_reuse_last_inputs(necgpu_engine* e);

/* Device-resident access for benchmarks and tests: pointers into the engine's
 * own device buffers (valid until the next set_structure / destroy). */
int necgpu_device_z(necgpu_engine* e, void** z_fp64, int64_t* ld);
/* Copy the filled (unfactored) Z to the host: n*n complex, out[basis + obs*n],
 * the layout of the reference's cm after cmset.  Only valid between
 * necgpu_fill and necgpu_factor(NECGPU_FP64) (which factors in place). */
int necgpu_copy_z(necgpu_engine* e, double* host_out);

/* Benchmark support: keep one right-hand side and one direction list
 * resident, then run fill -> factor -> solve -> coefficients -> far field
 * entirely on the device (no host transfers; one status read at the end). */
int necgpu_set_resident(necgpu_engine* e, const double* rhs, int n_dir, const double* theta,
                        const double* phi);
int necgpu_step_resident(necgpu_engine* e, int precision);
/* Copy results of the last resident step (cur: n complex, eth/eph: n_dir complex). */
int necgpu_read_resident(necgpu_engine* e, double* cur, double* eth, double* eph);

/* Allocation-free solve.  No counterpart in the reference (its solves runs on
 * host arrays the caller already owns); this is an addition for callers that
 * must not allocate.
 *
 * The same solution as necgpu_solve on the held factors (FP64, or mixed with
 * its FP64 refinement), but rhs_dev (n complex), cur_dev (n complex) and
 * abc_dev (6*n doubles, or NULL) are device memory of the engine's device,
 * and every scratch vector lives in one static device array of 1,574,144
 * bytes per device, sized for n <= 16384 unknowns; larger n is rejected with
 * NECGPU_ERR_ARG.  No call after the first allocates host or device memory
 * on success (a failure stores its message in the engine).  Who needs it: a
 * caller that reserved the device's memory up front for its own pool (a
 * frequency sweep or an optimiser holding thousands of matrices, a PyTorch
 * process whose caching allocator owns the HBM) and calls the solver inside
 * its inner loop, where a cudaMalloc can fail or fragment that pool and a
 * cudaFree waits for the whole device, stalling the caller's other streams.
 *
 * Each buffer must lie inside one device allocation: one that runs past the
 * end of its allocation is rejected with NECGPU_ERR_ARG.  A sub-allocation of
 * a caching allocator (PyTorch's, say) can only be checked against the end of
 * the segment that holds it, so the lengths above stay the caller's duty.
 *
 * The first call on a device does the set-up, with that device current:
 * it looks up the static array, zeroes the sweep flag words (they must start
 * at zero; nothing else in the array needs to), loads every kernel the call
 * can launch in either precision (under CUDA's lazy module loading a kernel
 * takes device memory when it is first loaded), and sets the kernels'
 * attributes.  Make that first call before any stream capture.  The work
 * runs on the engine's stream; the call returns when it has finished
 * (mixed refinement also waits once per refinement step).  The engine's own
 * solution (for necgpu_pattern) is left as it was.
 *
 * All engines on one device share the one array and its host-side sweep
 * counter: calls that overlap in time on the same device (from two threads,
 * or two engines on different streams) race on the array and give wrong
 * results.  Serialise them.
 *
 * If the mixed refinement stalls on block-pivoted factors, the call fails
 * with NECGPU_ERR_REFINE instead of refactoring (which would allocate);
 * necgpu_solve refactors with partial pivoting, after which this call
 * converges. */
int necgpu_solve_noalloc(necgpu_engine* e, const double* rhs_dev, double* cur_dev, double* abc_dev);

/* ---- adjoint gradients (no counterpart in the reference; they serve the
 * gradient extension of the host library, nec_gradient) ---- */

/* Copy the basis amplitudes x of the last necgpu_solve (n complex; Z x = e). */
int necgpu_copy_solution(necgpu_engine* e, double* x);

/* Solve Z^T w_k = phi_k for nrhs right-hand sides (n complex each, host
 * arrays) on the held mixed-precision factors: the transposed factors and
 * diagonal-block inverses drive the same triangular sweeps, refined in FP64
 * against Z^T to the refinement tolerance.  NECGPU_ERR_UNSUPPORTED after an
 * FP64 factorisation (it overwrites Z). */
int necgpu_adjoint_solve(necgpu_engine* e, int nrhs, const double* phi, double* w);

/* E_theta = phi_t^T x and E_phi = phi_p^T x: the far field of one direction
 * (radians) as linear functionals of the basis amplitudes (n complex each). */
int necgpu_pattern_weights(necgpu_engine* e, double theta, double phi, double* phi_t, double* phi_p);

/* For each of nstruct perturbed copies of the held structure (same segment
 * count, basis-table layout and medium; geometry and coefficients may
 * differ): zx[s][k] = w_k^T Z_s x for the nw <= 4 vectors w (nw x n complex)
 * and the held solution x, from a fill of Z_s contracted on the fly (Z_s is
 * not stored); efar[s] = (E_theta, E_phi) of x on structure s at one
 * direction.  zx: nstruct x nw complex; efar: nstruct x 2 complex. */
int necgpu_perturbed_terms(necgpu_engine* e, int nstruct, const necgpu_structure* structs, int nw, const double* w,
                           double theta, double phi, double* zx, double* efar);

/* ---- batched sweeps (no counterpart in the reference, which solves one
 * structure per context; this serves frequency sweeps and optimiser
 * populations of small structures) ---- */

/* Solve nprob independent structures (2..640 segments each; one medium,
 * ground and kernel setting for all) in one pass: fill, complex64 LU with
 * partial pivoting, solve refined in FP64 against the FP64 matrix,
 * segment-centre currents, far field at ndir directions (radians; 0 for
 * none).  rhs / cur: the problems' vectors concatenated (sum n complex).
 * gain (or NULL): nprob x ndir power gain in dB, normalised by the input
 * power of the one voltage source of each problem (feed: 0-based segment,
 * volt: complex source voltage, wavelength in metres, per problem).
 * eth / eph (both or neither): nprob x ndir complex fields.  status[p]:
 * 0 ok, 1 singular, 2 non-finite, 3 refinement above 1e-6; residual[p]
 * (or NULL): final relative FP64 residual. */
int necgpu_batch_solve(necgpu_engine* e, int nprob, const necgpu_structure* structs, const double* rhs,
                       const int* feed, const double* volt, const double* wavelength, int ndir, const double* theta,
                       const double* phi, double* cur, float* gain, double* eth, double* eph, int* status,
                       double* residual);

/* Diagnostic: apply one complex64 update C -= A B (m x n, inner kb) to a
 * seeded random matrix with the tensor-core kernel and with the CUDA-core
 * FP32 kernel; report max |difference| and max |reference| over C. */
int necgpu_check_tc_gemm(necgpu_engine* e, int m, int n, int kb, unsigned seed, double* max_abs_diff,
                         double* max_abs_ref);

/* Dense complex solve of a caller's matrix, without a structure: the
 * replacement of factrs + solves (src/matrix_algebra.cpp:319-338, 351-503)
 * for a matrix that does not come from the fill.  z: n x n complex
 * (interleaved re, im), row-major, z[i*n + j] the coefficient of x_j in
 * equation i; b: n complex; x: n complex out.  NECGPU_FP64 factors with
 * partial pivoting; NECGPU_MIXED factors the complex64 copy (block-local
 * pivoting, with the partial-pivot refactor when a diagonal block has no
 * usable pivot or the refinement stalls) and refines in FP64 against z.
 * residual (may be NULL) receives the final relative residual of the mixed
 * refinement (0 for FP64).  An exactly singular matrix fails with
 * NECGPU_ERR_SINGULAR (or NECGPU_ERR_NONFINITE), never with a non-finite x.
 * Any structure the engine held is dropped, and the engine holds none
 * afterwards.  n <= 65536. */
int necgpu_matrix_solve(necgpu_engine* e, int64_t n, const double* z, const double* b, int precision, double* x,
                        double* residual);

/* ---- tuning of the mixed-precision LU (no counterpart in the reference,
 * whose Eigen LU has fixed blocking, src/matrix_algebra.cpp:243-251) ----
 *
 * outer          columns per outer block of the block-pivoted LU: 64-wide
 *                inner panels inside it, one tensor-core trailing update of
 *                inner dimension `outer` per block (multiple of 64, 64..1024)
 * lookahead_sms  SMs kept for the next outer block's panels while the far
 *                part of the trailing update runs beside them (0: no
 *                lookahead; at most 127)
 * gemm_group     m-tiles per band of the tensor-core update's tile walk
 *                (1..1024)
 *
 * The values a factorisation uses are, in order of precedence: the
 * environment (NECPP_B200_OUTER, NECPP_B200_LOOKAHEAD_SMS,
 * NECPP_B200_LOOKAHEAD=0, NECPP_B200_GEMM_GROUP), an explicit
 * necgpu_set_tuning, the row of the tuning table for the precision and n,
 * the built-in defaults (256, 48, 16).  The tuning table is the text file
 * tuning.tsv beside the library (written by the autotuner,
 * necpp_b200/tune.py), or the file named by NECPP_B200_TUNING ("none": no
 * table).  Its rows are "precision n_max outer lookahead_sms gemm_group
 * [measurement]" with precision "mixed" or "fp64"; a size uses the row with
 * the smallest n_max >= n, else the row with the largest n_max. */
typedef struct necgpu_tuning {
  int outer;
  int lookahead_sms;
  int gemm_group;
} necgpu_tuning;

/* Fix the engine's tuning (NULL: back to the table and defaults). */
int necgpu_set_tuning(necgpu_engine* e, const necgpu_tuning* t);

/* The tuning a factorisation of n unknowns in `precision` would use now. */
int necgpu_get_tuning(const necgpu_engine* e, int precision, int64_t n, necgpu_tuning* out);

/* Host-only lookup in a tuning table (path NULL: the library's table, as
 * above).  Returns 0 and fills *out when a row applies, NECGPU_ERR_ARG when
 * the table is missing, unreadable, malformed or has no row for the
 * precision (out then holds the defaults).  Needs no device. */
int necgpu_tuning_lookup(const char* path, int precision, int64_t n, necgpu_tuning* out);

/* Measured FP64 throughput of this device in TFLOP/s, the denominator of the
 * FP64 kernels' rooflines: kind 0 = FP64 FMA on the CUDA cores (the fill and
 * pattern arithmetic), kind 1 = FP64 tensor-core MMA (mma.sync m8n8k4, the
 * FP64 LU's trailing update).  A register-only loop over 4 CTAs per SM, best
 * of three timed launches.  Measurement support; no counterpart in the
 * reference. */
int necgpu_measure_peak(necgpu_engine* e, int kind, double* tflops);

/* Self-check of the block-pivoted complex64 LU of the mixed path: factors a
 * seeded random n x n matrix (n <= 4096) on the engine's buffers and reports
 * the componentwise backward error max |P A - L U|_ij / (|L| |U|)_ij, max |A|
 * and how many of the n interchanges moved a row.  The engine must hold no
 * structure, and holds none afterwards.  Test support; it has no counterpart
 * in the reference. */
int necgpu_check_block_lu(necgpu_engine* e, int n, unsigned seed, double* backward_err, double* max_abs,
                          int* interchanges);

#ifdef __cplusplus
}
#endif
#endif /* NECGPU_H */
