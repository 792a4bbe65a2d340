/*
 * libnecpp.h -- the NEC2++ C API, served by libnecpp_b200.so.
 *
 * Same names, argument meanings, return values and error behaviour as the
 * reference's src/libnecpp.h (line numbers below): functions return 0 on
 * success and 1 on error with the message available from
 * nec_error_message(); result accessors return -999.0 when no result exists.
 * The fill, LU factor/solve and far-field sum behind nec_xq_card /
 * nec_rp_card run on a B200 GPU (include/necgpu.h); there is no CPU path.
 *
 * Cards outside the thin-wire hot path (patches SP/SC, symmetry GX, loads LD,
 * networks NT/TL, near fields NE/NH, coupling CP, cliffs GD, plot PL,
 * EX type 5) exist and return 1 with a message saying so.
 */
#ifndef LIBNECPP_B200_H
#define LIBNECPP_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#ifndef __cplusplus
typedef struct nec_context nec_context;
#else
namespace necb { class Context; }
typedef necb::Context nec_context;
#endif

/* src/libnecpp.h:60 */
nec_context* nec_create(void);
/* src/libnecpp.h:65 */
long nec_delete(nec_context* in_context);
/* src/libnecpp.h:94-97 */
long nec_wire(nec_context* in_context, int tag_id, int segment_count,
              double xw1, double yw1, double zw1, double xw2, double yw2, double zw2,
              double rad, double rdel, double rrad);
/* src/libnecpp.h:116-118 (patches: not in the hot path, returns 1) */
long nec_sp_card(nec_context* in_context, int ns, double x1, double y1, double z1,
                 double x2, double y2, double z2);
/* src/libnecpp.h:132-134 (patches: returns 1) */
long nec_sc_card(nec_context* in_context, int i2, double x3, double y3, double z3,
                 double x4, double y4, double z4);
/* src/libnecpp.h:154-156 (angles in degrees) */
long nec_gm_card(nec_context* in_context, int itsi, int nrpt, double rox, double roy,
                 double roz, double xs, double ys, double zs, int its);
/* src/libnecpp.h:190 (symmetry: returns 1) */
long nec_gx_card(nec_context* in_context, int i1, int i2);
/* src/libnecpp.h:201 */
long nec_geometry_complete(nec_context* in_context, int gpflag);
/* src/libnecpp.h:214 (the reference's benchmark decks; returns 0 and sets the
   error message: the reference's own benchmark geometry fails its overlap
   check in the version this build follows) */
long nec_benchmark(void);
/* src/libnecpp.h:220 */
const char* nec_error_message(void);
/* src/libnecpp.h:240 */
long nec_medium_parameters(nec_context* in_context, double permittivity, double permeability);
/* src/libnecpp.h:264 */
long nec_gn_card(nec_context* in_context, int iperf, int nradl, double epse, double sig,
                 double tmp3, double tmp4, double tmp5, double tmp6);
/* src/libnecpp.h:274 */
long nec_fr_card(nec_context* in_context, int in_ifrq, int in_nfrq, double in_freq_mhz,
                 double in_del_freq);
/* src/libnecpp.h:282 */
long nec_ek_card(nec_context* in_context, int itmp1);
/* src/libnecpp.h:303: impedance loading (types 0-5: series / parallel RLC,
   per metre, fixed impedance, wire conductivity) */
long nec_ld_card(nec_context* in_context, int ldtyp, int ldtag, int ldtagf, int ldtagt,
                 double tmp1, double tmp2, double tmp3);
/* src/libnecpp.h:330 */
long nec_ex_card(nec_context* in_context, int extype, int i2, int i3, int i4, double tmp1,
                 double tmp2, double tmp3, double tmp4, double tmp5, double tmp6);
/* src/libnecpp.h:349 */
long nec_excitation_voltage(nec_context* in_context, int tag, int segment, double v_real,
                            double v_imag);
/* src/libnecpp.h:365 */
long nec_excitation_current(nec_context* in_context, double x, double y, double z, double a,
                            double beta, double moment);
/* src/libnecpp.h:384-385 */
long nec_excitation_planewave(nec_context* in_context, int n_theta, int n_phi, double theta,
                              double phi, double eta, double dtheta, double dphi,
                              double pol_ratio);
/* src/libnecpp.h:387-388: transmission lines (Z0 < 0 crosses the line;
   length <= 0 takes the distance between the two port segments) and
   two-port networks given by their short-circuit admittances */
long nec_tl_card(nec_context* in_context, int itmp1, int itmp2, int itmp3, int itmp4,
                 double tmp1, double tmp2, double tmp3, double tmp4, double tmp5, double tmp6);
long nec_nt_card(nec_context* in_context, int itmp1, int itmp2, int itmp3, int itmp4,
                 double tmp1, double tmp2, double tmp3, double tmp4, double tmp5, double tmp6);
/* src/libnecpp.h:406 */
long nec_xq_card(nec_context* in_context, int itmp1);
/* src/libnecpp.h:408 (cliff: returns 1) */
long nec_gd_card(nec_context* in_context, double tmp1, double tmp2, double tmp3, double tmp4);
/* src/libnecpp.h:483-487 */
long nec_rp_card(nec_context* in_context, int calc_mode, int n_theta, int n_phi,
                 int output_format, int normalization, int D, int A, double theta0,
                 double phi0, double delta_theta, double delta_phi, double radial_distance,
                 double gain_norm);
/* src/libnecpp.h:505-507 */
long nec_pt_card(nec_context* in_context, int itmp1, int itmp2, int itmp3, int itmp4);
long nec_pq_card(nec_context* in_context, int itmp1, int itmp2, int itmp3, int itmp4);
/* src/libnecpp.h:509 */
long nec_kh_card(nec_context* in_context, double tmp1);
/* src/libnecpp.h:510-511: near electric / magnetic field over a grid of
   points (near = 0 rectangular in metres, 1 spherical in degrees); results
   through nec_near_field */
long nec_ne_card(nec_context* in_context, int itmp1, int itmp2, int itmp3, int itmp4,
                 double tmp1, double tmp2, double tmp3, double tmp4, double tmp5, double tmp6);
long nec_nh_card(nec_context* in_context, int itmp1, int itmp2, int itmp3, int itmp4,
                 double tmp1, double tmp2, double tmp3, double tmp4, double tmp5, double tmp6);
/* src/libnecpp.h:514-515 (coupling / plot: return 1) */
long nec_cp_card(nec_context* in_context, int itmp1, int itmp2, int itmp3, int itmp4);
long nec_pl_card(nec_context* in_context, char* ploutput_filename, int itmp1, int itmp2,
                 int itmp3, int itmp4);

/* src/libnecpp.h:537-606: result accessors (-999.0 when absent) */
double nec_gain(nec_context* in_context, int freq_index, int theta_index, int phi_index);
double nec_gain_max(nec_context* in_context, int freq_index);
double nec_gain_min(nec_context* in_context, int freq_index);
double nec_gain_mean(nec_context* in_context, int freq_index);
double nec_gain_sd(nec_context* in_context, int freq_index);
double nec_gain_rhcp_max(nec_context* in_context, int freq_index);
double nec_gain_rhcp_min(nec_context* in_context, int freq_index);
double nec_gain_rhcp_mean(nec_context* in_context, int freq_index);
double nec_gain_rhcp_sd(nec_context* in_context, int freq_index);
double nec_gain_lhcp_max(nec_context* in_context, int freq_index);
double nec_gain_lhcp_min(nec_context* in_context, int freq_index);
double nec_gain_lhcp_mean(nec_context* in_context, int freq_index);
double nec_gain_lhcp_sd(nec_context* in_context, int freq_index);
double nec_impedance_real(nec_context* in_context, int freq_index);
double nec_impedance_imag(nec_context* in_context, int freq_index);
double nec_impedance_real_indexed(nec_context* in_context, int freq_index, int feed_index);
double nec_impedance_imag_indexed(nec_context* in_context, int freq_index, int feed_index);

/* ---- Extensions (no C-API counterpart in the reference) ---------------- */

/* nec_context::helix (src/nec_context.h:449-450; only in the reference's C++
   API): GH card. */
long nec_helix(nec_context* in_context, int tag_id, int segment_count, double s, double hl,
               double a1, double b1, double a2, double b2, double rad);
/* Precision of the GPU factor/solve: 0 = complex128 (default), 1 = mixed
   (complex64 LU with tensor-core trailing update + FP64 refinement). */
long nec_set_precision(nec_context* in_context, int precision);
/* c_geometry::set_intersection_check / set_intersection_fatal
   (src/c_geometry.h:148-154). */
long nec_set_intersection_check(nec_context* in_context, int enable, int fatal);
/* Segment count after geometry_complete. */
long nec_segment_count(nec_context* in_context);
/* Scale the completed geometry to wavelengths at freq_mhz, as the frequency
   loop does (c_geometry::frequency_scale, src/c_geometry.cpp:3389-3418);
   host-only, for inspecting the basis tables. */
long nec_frequency_scale(nec_context* in_context, double freq_mhz);
/* Segment-centre currents in amperes of result index (n complex, re/im
   interleaved), i.e. nec_structure_currents::get_current(). Returns n or -1. */
long nec_get_currents(nec_context* in_context, int index, double* out, long capacity);
/* Segment tables after geometry_complete (metres): x,y,z centres, lengths,
   radii, direction cosines, tags, icon1, icon2 (each n long). */
long nec_get_segments(nec_context* in_context, double* x, double* y, double* z, double* si,
                      double* bi, double* cab, double* sab, double* salp, int* tags,
                      int* icon1, int* icon2);
/* trio(j) basis table of source segment j (1-based) at the scaling of the
   last frequency run; writes up to cap entries, returns the count. */
long nec_get_trio(nec_context* in_context, int j, int* jco, double* ax, double* bx,
                  double* cx, long cap);
/* Build, on the host only, the structure tables the GPU receives at
   freq_mhz: scaling, ground constants, trio basis tables, extended-kernel
   flags (for inspection and for driving include/necgpu.h directly). */
long nec_prepare_structure(nec_context* in_context, double freq_mhz);
/* Copy those tables out: seg (8n: x y z length radius cab sab salp, in
   wavelengths), tptr (n+1), tbasis (nt, 0-based), tabc (3nt: a b c),
   ind (2n: EK end flags), params (10: rkh, use_exk, ground, zrati re/im,
   frati re/im, eta, complex permittivity re/im of a finite ground).  Any pointer may be NULL; returns nt or -1. */
long nec_get_structure(nec_context* in_context, double* seg, int* tptr, int* tbasis, double* tabc,
                       int* ind, double* params);
/* Applied-field right-hand side of the current excitation at the prepared
   frequency (nec_context::etmns, src/nec_context.cpp:3488-3550): n complex,
   interleaved; host only. */
long nec_get_rhs(nec_context* in_context, double* out);
/* Impedance loading (n complex: lambda x impedance per unit length, the
   reference's zarray) of the structure prepared last; zeros if unloaded. */
long nec_get_loads(nec_context* in_context, double* out);
/* Near-field pattern `index` (0-based, in the order NE/NH requests ran;
   the reference's nec_context::get_near_field_pattern): returns its point
   count, or -1 if it does not exist.  nfeh receives 0 (electric) or 1
   (magnetic); with non-null buffers, xyz the points (metres, 3 per point)
   and fields 3 complex per point (x, y, z; re/im interleaved; V/m or A/m). */
long nec_near_field(nec_context* in_context, int index, int* nfeh, double* xyz, double* fields);
/* Runs a NEC input deck (nec2++'s card images: comments, geometry up to GE,
   program-control cards to EN; several jobs separated by NX) and writes the
   antenna input, power budget, radiation pattern and near-field sections of
   nec2++'s text output to output_path (standard output if NULL or empty).
   Returns 0, or 1 with the message in nec_deck_error(). */
long nec_run_deck(const char* input_path, const char* output_path);
const char* nec_deck_error(void);
/* Number of NT/TL networks on the context (0 if none). */
long nec_network_count(nec_context* in_context);
/* The context's GPU engine (include/necgpu.h), created on first use; NULL
   with nec_error_message() set when no usable device exists. */
void* nec_gpu_engine(nec_context* in_context);
/* Adjoint gradients (no counterpart in the reference).  After an XQ or RP
   card has solved `base` (one voltage source, mixed precision), returns
   value[3] = {Re Zin, Im Zin, gain in dB at (theta, phi)} and
   grad[3*k + i] = d value[i] / d p_k for nparam geometry parameters p_k.
   plus[k] / minus[k] are contexts holding the same cards with parameter k
   moved by +h[k] / -h[k] (geometry complete and excitation given, not
   solved).  One transposed solve per output on the held factors; the
   matrix derivative is recomputed tile by tile from the perturbed
   structures and never stored. */
long nec_gradient(nec_context* base, int nparam, nec_context** plus, nec_context** minus, const double* h,
                  double theta_deg, double phi_deg, double* value, double* grad);
/* Refinement diagnostics of the last solve (mixed precision). */
long nec_last_refinement(nec_context* in_context, int* iters, double* residual);
/* Complex far field E_theta / E_phi (V/m x wavelength, as stored by the
   reference's nec_radiation_pattern) of result index. */
long nec_get_pattern_fields(nec_context* in_context, int index, double* e_theta,
                            double* e_phi, long capacity);

#ifdef __cplusplus
}
#endif
#endif /* LIBNECPP_B200_H */
