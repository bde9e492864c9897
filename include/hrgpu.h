/*
 * hrgpu.h -- C ABI of the B200 (sm_100a) fermion hot path for HiRep.
 *
 * Plain C, plain pointers and sizes.  One process drives one GPU; the library
 * keeps HiRep's "global state" model (one lattice, one gauge field, one clover
 * term, one force accumulator), like LibHR does through Include/global.h.
 *
 * Fields passed to the operators are DEVICE pointers in the library's device
 * layout (structure-of-arrays, checkerboarded; see hrgpu_spinor_bytes).  Host
 * fields in HiRep's own layout (Include/spinor_field.h:37-56, site order from
 * LibHR/Geometry/geometry_mpi_eo.c) cross the boundary through
 * hrgpu_spinor_upload / hrgpu_spinor_download, which translate the site order
 * and the layout exactly.
 *
 * Every entry point returns 0 on success and a non-zero HRGPU_E* code on
 * failure; hrgpu_last_error() gives the message.  (HiRep's own convention is
 * error() -> exit, LibHR/Error/error.c:21-37; the drop-in layer maps a non-zero
 * status onto that.)
 *
 * Each declaration names the reference interface it replaces (file:line in
 * sofiemartins/HiRep).
 */
#ifndef HRGPU_H
#define HRGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* parities: HiRep's glat_even / glat_odd / glattice (Include/global.h:105-107) */
enum { HRGPU_EVEN = 0, HRGPU_ODD = 1, HRGPU_FULL = 2 };
/* precisions: spinor_field / spinor_field_flt (Include/spinor_field.h:50-51) */
enum { HRGPU_DOUBLE = 0, HRGPU_FLOAT = 1 };
/* representations: REPR_FUNDAMENTAL / _ADJOINT / _SYMMETRIC / _ANTISYMMETRIC (Make/MkFlags) */
enum { HRGPU_FUND = 0, HRGPU_ADJ = 1, HRGPU_SYM = 2, HRGPU_ASYM = 3 };
/* operators for the inverters: the spinor_operator argument of cg_mshift (Include/inverters.h:14) */
enum {
  HRGPU_OP_G5DPHI_SQ = 0,       /* g5Dphi_sq(mass)        Dphi.c:1001-1019, full lattice   */
  HRGPU_OP_G5DPHI_EOPRE_SQ = 1, /* g5Dphi_eopre_sq(mass)  Dphi.c:988-998, even sites       */
  HRGPU_OP_G5CPHI_EOPRE_SQ = 2, /* g5Cphi_eopre_sq(mass)  Dphi.c:1263-1272, even sites     */
  HRGPU_OP_G5CPHI_SQ = 3,       /* g5Cphi_sq(mass)        Dphi.c:1226-1235, full lattice   */
  /* not positive (the g5QMR / MINRES operators; eopre ones also for hrgpu_apply_op_batch) */
  HRGPU_OP_DPHI_EOPRE = 4,      /* Dphi_eopre(mass)       Dphi.c:874-907                   */
  HRGPU_OP_G5DPHI_EOPRE = 5,    /* g5Dphi_eopre(mass)     Dphi.c:950-985                   */
  HRGPU_OP_CPHI_EOPRE = 6,      /* Cphi_eopre(mass)       Dphi.c:1240-1255                 */
  HRGPU_OP_G5CPHI_EOPRE = 7,    /* g5Cphi_eopre(mass)     Dphi.c:1257-1261                 */
  HRGPU_OP_DPHI = 8,            /* Dphi(mass)             Dphi.c:703-783, full lattice     */
  HRGPU_OP_CPHI = 9             /* Cphi(mass)             Dphi.c:1215-1221, full lattice   */
};
/* status codes */
enum {
  HRGPU_OK = 0,
  HRGPU_E_CUDA = 1,      /* a CUDA call failed                          */
  HRGPU_E_ARG = 2,       /* invalid argument                            */
  HRGPU_E_STATE = 3,     /* called before the state it needs was set    */
  HRGPU_E_NF = 4,        /* no kernel instantiated for this NF          */
  HRGPU_E_NOCONV = 5,    /* inverter stopped at max_iter (not fatal)    */
  HRGPU_E_BREAKDOWN = 6  /* inverter breakdown: a non-finite source, norm or
                            residual, or zero curvature <p, M p> (a NaN field or a
                            singular system); the solution is garbage (fatal)  */
};

/* ---------------------------------------------------------------- setup -- */
/* process/device setup: replaces the device part of setup_process (LibHR/Geometry/process_init.c:56-146) */
int hrgpu_init(int device);
/* lattice: geometry_init (LibHR/Geometry/geometry_init.c:243-338) for one GPU.
 * ipt is HiRep's site map ipt[((t*X+x)*Y+y)*Z+z] (Include/global.h:96,103) and is
 * imported bit-exactly; ng/repr fix NG, NF and the representation (Make/MkFlags:1-75). */
int hrgpu_lattice_init(int T, int X, int Y, int Z, int ng, int repr, const int *ipt);
/* HiRep's serial site numbering (LibHR/Geometry/geometry_mpi_eo.c:1919-1953 with
 * NP_T=NP_X=NP_Y=NP_Z=1): fills ipt[V] and, when non-NULL, iup[4V] and idn[4V]
 * exactly as Include/global.h:96-100 holds them.  Host-only, no GPU needed. */
int hrgpu_geometry(int T, int X, int Y, int Z, int *ipt, int *iup, int *idn);
/* frees every device buffer (the atexit frees of Dphi.c:45-73, field_alloc.c) */
int hrgpu_finalize(void);
const char *hrgpu_last_error(void);
int hrgpu_nf(void);
/* the basis T_A of su(NG) in which forces and momenta are expanded (autosun's
 * generators, Tr T_A T_B = delta_AB / 2): T[A][i][j] complex, A < NG*NG-1 */
int hrgpu_algebra_generators(double *T);
/* bytes of one device spinor field of the given parity and precision */
size_t hrgpu_spinor_bytes(int par, int prec);
/* all work is issued on this stream; NULL is the legacy default stream (stream 0).
 * Until this is called the library uses a stream of its own. */
int hrgpu_set_stream(void *cuda_stream);
int hrgpu_synchronize(void);

/* --------------------------------------------------------- gauge fields -- */
/* u_gauge upload (Include/global.h:143, HiRep layout [V][4][NG*NG] complex) */
int hrgpu_gauge_set(const double *u_host);
/* represent_gauge_field (LibHR/Update/representation.c:391-468) on the device, then
 * the antiperiodic-T link sign (LibHR/Utils/boundary_conditions.c:321-341) and,
 * with a clover term, compute_clover_term; also refreshes the float copy (assign_ud2u_f) */
int hrgpu_represent_gauge_field(int bc_t_antiperiodic);
/* SU(3) fundamental and SU(2) adjoint links: after represent_gauge_field has
 * checked that every link's row 2 equals s conj(r0 x r1) (adjoint: s (r0 x r1))
 * to 1e-14 (s = -1 on the links with the antiperiodic time sign), the
 * single-field hopping kernels load rows 0 and 1 only and rebuild row 2.
 * hrgpu_gauge_set_f runs the same check, trying the antiperiodic sign first.
 * The SU(3) symmetric and SU(4) antisymmetric representations (NF = 6): after
 * represent_gauge_field the single-field hopping kernel of variant 6 may
 * build each represented link from the fundamental one (9 or 16 complex
 * numbers read instead of 36), until the fundamental links are written again
 * (hrgpu_gauge_set, update_gauge_field, project_gauge_field,
 * read_gauge_field) or represented links are uploaded; the autotuner times it
 * against the other variants.
 * mode: 0 full links (any other group or representation, a field that fails
 * the check), 1 rebuilt, 2 rebuilt with the antiperiodic sign, 3 built from
 * the fundamental links, 4 the same with the antiperiodic sign.  No
 * counterpart in the reference, which reads the full links. */
int hrgpu_link_recon(int *mode);
/* allow (1, default) or forbid (0) the reconstruction modes above */
int hrgpu_set_link_recon(int on);
/* u_gauge_f upload: the represented field as HiRep holds it ([V][4][NF*NF], complex,
 * or real for the adjoint representation) */
int hrgpu_gauge_set_f(const void *uf_host);
int hrgpu_gauge_get_f(void *uf_host);
/* assign_ud2u_f (LibHR/Utils/single_double_utils.c:70-87) */
int hrgpu_assign_ud2u_f(void);

/* ------------------------------------------------------- spinor fields -- */
/* host (HiRep layout, HiRep site order) <-> device layout; prec selects
 * suNf_spinor (double) or suNf_spinor_flt (float) */
int hrgpu_spinor_upload(void *dev, const void *host, int par, int prec);
int hrgpu_spinor_download(void *host, const void *dev, int par, int prec);
/* assign_sd2s / assign_s2sd (LibHR/Utils/single_double_utils.c:89-115) */
int hrgpu_assign_sd2s(void *out_flt, const void *in_dbl, int par);
int hrgpu_assign_s2sd(void *out_dbl, const void *in_flt, int par);

/* ------------------------------------------------------ Dirac operator -- */
/* Dphi_ (LibHR/Update/Dphi.c:193-374): out_par EVEN/ODD reads the other parity,
 * FULL reads a full field.  Hopping term with the -1/2 included. */
int hrgpu_Dphi_(void *out, int out_par, const void *in);
int hrgpu_Dphi(double m0, void *out, const void *in);             /* Dphi.c:703-783   */
int hrgpu_g5Dphi(double m0, void *out, const void *in);           /* Dphi.c:785-867   */
int hrgpu_g5Dphi_sq(double m0, void *out, const void *in);        /* Dphi.c:1001-1019 */
int hrgpu_Dphi_eopre(double m0, void *out, const void *in);       /* Dphi.c:874-907   */
int hrgpu_Dphi_oepre(double m0, void *out, const void *in);       /* Dphi.c:914-948   */
int hrgpu_g5Dphi_eopre(double m0, void *out, const void *in);     /* Dphi.c:950-985   */
int hrgpu_g5Dphi_eopre_sq(double m0, void *out, const void *in);  /* Dphi.c:988-998   */
/* Dphi_eopre for callers that cannot let the library allocate device memory
 * (a host framework that owns the GPU through its own memory pool).  Same
 * result as hrgpu_Dphi_eopre, but the odd temporary lives in a 32 MiB static
 * device array of the library instead of a cudaMalloc'd buffer; lattices whose
 * odd FP64 field needs more are rejected with HRGPU_E_ARG.  The first call on a
 * device looks up the array's address (make it before any stream capture); calls
 * that overlap on the GPU share the array and race.  No counterpart in the
 * reference. */
int hrgpu_Dphi_eopre_noalloc(double m0, void *out, const void *in);
/* single precision: LibHR/Update/Dphi_flt.c:162-593 */
int hrgpu_Dphi_flt_(void *out, int out_par, const void *in);
int hrgpu_Dphi_flt(double m0, void *out, const void *in);
int hrgpu_g5Dphi_flt(double m0, void *out, const void *in);
int hrgpu_g5Dphi_sq_flt(double m0, void *out, const void *in);
int hrgpu_Dphi_eopre_flt(double m0, void *out, const void *in);
int hrgpu_g5Dphi_eopre_flt(double m0, void *out, const void *in);
int hrgpu_g5Dphi_eopre_sq_flt(double m0, void *out, const void *in);
/* Hopping-kernel variant: 0 = one thread per site, 1 = two threads per site
 * (spin split), 2 and 3 = the same with registers capped for 4 blocks per SM,
 * 4 = one thread per site with cp.async-pipelined loads, 5 = one thread per site
 * with the time halo staged in shared memory by bulk (TMA) copies (4 and 5: NF <= 4
 * complex, NF = 3 real; 5 also needs time slabs of a multiple of 128 sites per
 * parity), 6 = one thread per site building the SU(3) symmetric or SU(4)
 * antisymmetric links from the fundamental ones (link modes 3 and 4 of
 * hrgpu_link_recon; the FP32 operators from a float copy of the fundamental
 * links made with the FP32 represented ones), -1 = autotune on first use (default).  hrgpu_hop_tuning
 * reports the variant chosen for (precision, epilogue 0..2) and the per-launch
 * times it measured (ms has room for 7 values; -1 marks a variant not built for
 * this NF, lattice or link mode); precision 2 is the FP32 operator reading BF16
 * links.
 * Tuning controls of this library; they have no counterpart in the reference. */
int hrgpu_set_hop_variant(int variant);
int hrgpu_hop_tuning(int prec, int epilogue, int *chosen, float *ms);
/* whole-lattice FP64 hopping kernels launched with programmatic dependent
 * launch (default 1: the next hop's blocks start in the SMs the previous hop's
 * last wave leaves idle); 0 launches them plainly */
int hrgpu_set_hop_pdl(int on);
/* Storage of the links read by the FP32 operators (the _flt operators, the
 * inner solves of cg_mshift_flt): HRGPU_LINKS_F32 (default, assign_ud2u_f's
 * copy) or HRGPU_LINKS_BF16 (a BF16 copy rounded from the FP64 links, FP32
 * arithmetic).  BF16 halves the link bytes of the FP32 operator and makes its
 * result differ from the FP32 one at the 1e-3 level; the FP64 defect
 * correction of cg_mshift_flt still reaches the FP64 tolerance.  An experiment
 * of this library, not in the reference. */
enum { HRGPU_LINKS_F32 = 0, HRGPU_LINKS_BF16 = 1 };
int hrgpu_set_flt_link_storage(int kind);
/* getMVM (Dphi.c:105-113): hopping applications / 2 since the last call */
unsigned long hrgpu_getMVM(void);

/* set_dirac_mass / get_dirac_mass and the global-mass operators H2, H, D
 * (LibHR/Update/D_update.c:12-95, UPDATE_EO build; clover forms when a clover
 * term is set) */
int hrgpu_set_dirac_mass(double mass);
double hrgpu_get_dirac_mass(void);
int hrgpu_H2(void *out, const void *in);
int hrgpu_H(void *out, const void *in);
int hrgpu_D(void *out, const void *in);

/* ------------------------------------------------------------ host fields -- */
/* An even-odd preconditioned operator (op 4..7: Dphi_eopre, g5Dphi_eopre,
 * Cphi_eopre, g5Cphi_eopre; Dphi.c:874-985, :1240-1261) applied to an even host
 * field in HiRep's layout ([VH][4][NF] complex in ipt order, complex128 for
 * HRGPU_DOUBLE, complex64 for HRGPU_FLOAT), result written to host_out.  The
 * field is moved in chunks whose copies overlap the hops on the time slabs
 * already complete (bit-identical to upload + operator + download).  Host
 * buffers should be pinned (cudaHostAlloc / cudaHostRegister) for the copies to
 * overlap. */
int hrgpu_apply_op_host(int op, double mass, void *host_out, const void *host_in, int prec);
int hrgpu_set_host_chunks(int chunks); /* chunks of the pipeline (default 10; 1 = no overlap) */
/* With pinned buffers the operator runs as a cached CUDA graph per (operator,
 * mass, buffers, ...).  Form 0 (default): when a graph is made, the pipelined
 * form and the plain sequence (one copy each way around the whole-lattice
 * operator) are both captured and timed, the faster is used first, the first 32
 * calls for that graph alternate the two (timed on the device) and the one with
 * the lower median is kept, and 32 calls alternate them again after every 1024
 * calls; 1 forces the pipeline, 2 the plain sequence.  No HiRep counterpart
 * (host-field transport). */
int hrgpu_set_host_form(int form);
/* the form chosen for the last graph made (1 pipelined, 2 sequential, -1 none
 * yet) and the times behind the choice (ms: the replays when the graph was made,
 * then the trial calls' medians once a round of them is done; -1 if not timed) */
int hrgpu_host_form(int *form, float *ms_pipelined, float *ms_sequential);

/* ---------------------------------------------------------------- clover -- */
int hrgpu_clover_init(double csw);                  /* clover_init, clover_tools.c:360-373        */
/* the same with the exponential clover term of WITH_EXPCLOVER (Dphi.c:1292-1482,
 * LibHR/Utils/clover_exp.c): diagonal (4+m) exp(A/(4+m)), inverse
 * exp(-A/(4+m))/(4+m); every Cphi operator and force_fermion_core then use it
 * (force_fermion_core.c:484-772), and force_clover_logdet adds nothing (the
 * blocks are traceless: det D_oo is constant). */
int hrgpu_expclover_init(double csw);
int hrgpu_compute_clover_term(void);                /* compute_clover_term, clover_tools.c:333-341 */
int hrgpu_compute_ldl_decomp(double sigma);         /* compute_ldl_decomp, clover_tools.c:343-358  */
int hrgpu_clover_term_get(void *cl_host);           /* cl_term in HiRep layout [V][4][NF*NF] complex */
int hrgpu_Cphi(double mass, void *out, const void *in);            /* Dphi.c:1215-1221 */
int hrgpu_g5Cphi(double mass, void *out, const void *in);          /* Dphi.c:1223-1227 */
int hrgpu_g5Cphi_sq(double mass, void *out, const void *in);       /* Dphi.c:1229-1238 */
int hrgpu_Cphi_eopre(double mass, void *out, const void *in);      /* Dphi.c:1240-1255 */
int hrgpu_g5Cphi_eopre(double mass, void *out, const void *in);    /* Dphi.c:1257-1261 */
int hrgpu_g5Cphi_eopre_sq(double mass, void *out, const void *in); /* Dphi.c:1263-1272 */
int hrgpu_Cphi_diag(double mass, void *out, const void *in, int par);     /* Dphi.c:1274-1280 */
int hrgpu_Cphi_diag_inv(double mass, void *out, const void *in, int par); /* Dphi.c:1282-1288 */
/* float clover operator for the mixed-precision solver (no float clover in the reference) */
int hrgpu_g5Cphi_eopre_flt(double mass, void *out, const void *in);
int hrgpu_g5Cphi_eopre_sq_flt(double mass, void *out, const void *in);

/* -------------------------------------------------------- linear algebra -- */
/* LibHR/Inverters/TMPL/linear_algebra.c.sdtmpl (declared in
 * Include/TMPL/linear_algebra.h.sdtmpl:6-95), instantiated for double (_f) and
 * float (_f_flt) by LibHR/Inverters/linear_algebra.c:20-59.  par gives the
 * geometry of the fields; prec = HRGPU_DOUBLE or HRGPU_FLOAT.  Reductions
 * accumulate in double in a fixed order (deterministic) and return on the host. */
int hrgpu_spinor_field_prod_re(int par, int prec, const void *s1, const void *s2, double *res);
int hrgpu_spinor_field_prod_im(int par, int prec, const void *s1, const void *s2, double *res);
int hrgpu_spinor_field_prod(int par, int prec, const void *s1, const void *s2, double *res_re_im);
int hrgpu_spinor_field_g5_prod_re(int par, int prec, const void *s1, const void *s2, double *res);
int hrgpu_spinor_field_g5_prod_im(int par, int prec, const void *s1, const void *s2, double *res);
int hrgpu_spinor_field_sqnorm(int par, int prec, const void *s1, double *res);
int hrgpu_spinor_field_mul_add_assign(int par, int prec, void *s1, double r, const void *s2);
int hrgpu_spinor_field_mulc_add_assign(int par, int prec, void *s1, double c_re, double c_im, const void *s2);
int hrgpu_spinor_field_g5_mulc_add_assign(int par, int prec, void *s1, double c_re, double c_im, const void *s2);
int hrgpu_spinor_field_mul(int par, int prec, void *s1, double r, const void *s2);
int hrgpu_spinor_field_mulc(int par, int prec, void *s1, double c_re, double c_im, const void *s2);
int hrgpu_spinor_field_add(int par, int prec, void *r, const void *s1, const void *s2);
int hrgpu_spinor_field_sub(int par, int prec, void *r, const void *s1, const void *s2);
int hrgpu_spinor_field_add_assign(int par, int prec, void *s1, const void *s2);
int hrgpu_spinor_field_sub_assign(int par, int prec, void *s1, const void *s2);
int hrgpu_spinor_field_copy(int par, int prec, void *s1, const void *s2);
int hrgpu_spinor_field_zero(int par, int prec, void *s1);
int hrgpu_spinor_field_minus(int par, int prec, void *s1, const void *s2);
int hrgpu_spinor_field_lc(int par, int prec, void *s1, double r1, const void *s2, double r2, const void *s3);
int hrgpu_spinor_field_lc_add_assign(int par, int prec, void *s1, double r1, const void *s2, double r2, const void *s3);
int hrgpu_spinor_field_clc(int par, int prec, void *s1, double c1_re, double c1_im, const void *s2,
                           double c2_re, double c2_im, const void *s3);
int hrgpu_spinor_field_clc_add_assign(int par, int prec, void *s1, double c1_re, double c1_im, const void *s2,
                                      double c2_re, double c2_im, const void *s3);
int hrgpu_spinor_field_g5(int par, int prec, void *s1, const void *s2);
int hrgpu_spinor_field_g5_assign(int par, int prec, void *s1);
int hrgpu_spinor_field_g0(int par, int prec, void *s1, const void *s2);
int hrgpu_spinor_field_g1(int par, int prec, void *s1, const void *s2);
int hrgpu_spinor_field_g2(int par, int prec, void *s1, const void *s2);
int hrgpu_spinor_field_g3(int par, int prec, void *s1, const void *s2);
int hrgpu_spinor_field_lc1(int par, int prec, double c1, void *s1, const void *s2);
int hrgpu_spinor_field_lc2(int par, int prec, double c1, double c2, void *s1, const void *s2);
int hrgpu_spinor_field_lc3(int par, int prec, double c1, double c2, const void *s1, const void *s2, void *s3);

/* ------------------------------------------------------------- inverters -- */
/* cg_mshift (LibHR/Inverters/cg_mshift.c:147-195): out[i] = (M - shift[i])^-1 in,
 * M selected by op at the given mass; err2 is HiRep's squared relative residual;
 * with n == 1 out[0] is the initial guess.  *iters gets the MVM count as HiRep
 * counts it (including the final true-residual checks). */
int hrgpu_cg_mshift(int op, double mass, int n, const double *shift, double err2, int max_iter,
                    const void *in, void *const *out, int *iters);
/* cg_mshift_flt (LibHR/Inverters/cg_mshift_flt.c:144-276): FP64 defect correction
 * around an FP32 multi-shift CG on the float twin of op (clover included). */
int hrgpu_cg_mshift_flt(int op, double mass, int n, const double *shift, double err2, int max_iter,
                        const void *in, void *const *out, int *iters);

/* g5QMR_mshift (LibHR/Inverters/g5QMR_mshift.c:481-542) for the gamma_5-hermitian
 * Dirac operator D (op: HRGPU_OP_DPHI_EOPRE, _CPHI_EOPRE, _DPHI, _CPHI):
 * out[i] = (D - shift[i])^-1 in; with n == 1 out[0] is the initial guess.
 * Unconverged shifts are solved again alone, then by MINRES on g5 (D - shift)
 * as in the reference.  *iters gets the MVM count as HiRep counts it. */
int hrgpu_g5QMR_mshift(int op, double mass, int n, const double *shift, double err2, int max_iter,
                       const void *in, void *const *out, int *iters);
/* MINRES (LibHR/Inverters/MINRES.c:160-172) for a hermitian op (g5Dphi_eopre,
 * g5Cphi_eopre and the squared operators); trial may be NULL (start from zero). */
int hrgpu_MINRES(int op, double mass, double err2, int max_iter, const void *in, void *out, const void *trial,
                 int *iters);
/* chronological initial guess, MRE (LibHR/Update/mre.c): a handle keeps the
 * last max (<= 15) solutions of two sequences p = 0, 1 of fields of parity par.
 * mre_guess builds the guess from them for DD = op (mre.c:230-268), keeping the
 * reference's convention (the coefficients solve A x = conj(b) with
 * A[j][i] = <DD v_i, v_j>, b_i = <v_i, pf>); a singular system gives out = 0.
 * hrgpu_mre_init returns NULL on error (message in hrgpu_last_error). */
void *hrgpu_mre_init(int max, int par);
int hrgpu_mre_store(void *mre, int p, const void *in);
int hrgpu_mre_guess(void *mre, int p, void *out, int op, double mass, const void *pf);
int hrgpu_mre_free(void *mre);

/* ------------------------------------------------------------ HMC pieces -- */
/* The gauge-side pieces of an HMC step on the device (HiRep's drivers --
 * integrator, monomials, accept/reject -- stay host code calling these).
 * Momenta: HiRep's suN_momenta, host layout [V][4][NG*NG-1] in HiRep's site
 * order; the library keeps one device copy. */
int hrgpu_momenta_set(const double *host);
int hrgpu_momenta_get(double *host);
/* Random draws on the device.  HiRep draws with ranlux on the host
 * (rlxd_init, LibHR/Random/ranlxd.c; gauss, LibHR/Random/gauss.c); here the
 * generator is Philox4x32-10 with Box-Muller Gaussians, keyed by
 * hrgpu_random_seed (the counterpart of rlxd_init's seed; a seed replays its
 * sequence of draws).  The numbers differ from ranlux's, the distributions
 * are the same.
 * gaussian_momenta: LibHR/Update/random_momenta.c:18-38 (fills the device
 * momenta: N(0,1)/sqrt(C(fund)) per generator component).
 * gaussian_spinor_field: LibHR/Update/random_spinor_field.c:14-36 (N(0,1)/sqrt(2)
 * per real component of a device field of parity par; FP32: the FP64 draw
 * rounded); padding sites are zero. */
int hrgpu_random_seed(unsigned long long seed);
int hrgpu_gaussian_momenta(void);
int hrgpu_gaussian_spinor_field(int par, int prec, void *s);
/* the fundamental links, host layout of hrgpu_gauge_set */
int hrgpu_gauge_get(double *u_host);
/* force0 (LibHR/Update/force0.c:22-99): momenta += -dt beta/NG proj(U staples^+) */
int hrgpu_force0(double dt, double beta);
/* update_gauge_field (LibHR/Update/field_update.c:18-66): U <- exp(dt mom) U on
 * every link (ExpX), reunitarised every 17th call (project_to_suNg,
 * suN_utils.c:76-150), then represent_gauge_field (and the clover term) with the
 * time boundary condition of the last hrgpu_represent_gauge_field */
int hrgpu_update_gauge_field(double dt);
int hrgpu_project_gauge_field(void);
/* local_hmc_action (LibHR/Update/local_action.c:19-90) into a device per-site
 * field: NEW sets it to 1/2 C(F) |mom|^2 - beta/NG (sum of the 6 plaquettes),
 * DELTA to that minus its previous content; pf_local_action adds |pf|^2 of a
 * pseudofermion of parity par; local_action_sum returns the sum over sites
 * (fixed-order reduction) and local_action_get the field ([V], HiRep order). */
enum { HRGPU_ACTION_NEW = 0, HRGPU_ACTION_DELTA = 1 };
int hrgpu_local_hmc_action(int type, double beta);
int hrgpu_pf_local_action(const void *pf, int par);
/* clover_la_logdet (clover_tools.c:312-331): local action -= nf log det D_oo on
 * the odd sites (the standard clover monomial's log-det term; refused for the
 * exponential clover term, whose det D_oo is constant) */
int hrgpu_clover_la_logdet(double nf, double mass);
int hrgpu_local_action_sum(double *sum);
int hrgpu_local_action_get(double *host);
/* avr_plaquette (LibHR/Observables/avr_plaquette.c): mean of Re Tr P / NG */
int hrgpu_avr_plaquette(double *plaq);
/* fermion_force_end (force_fermion_core.c:964-993) adding into the device momenta */
int hrgpu_fermion_force_end_momenta(double dt);

/* ------------------------------------------------------------- gauge IO -- */
/* write_gauge_field / read_gauge_field (LibHR/IO/archive.c:26-457,
 * archive_su2quat.c): HiRep's big-endian file (NG, T, X, Y, Z, the average
 * plaquette, then the links of each site in (t, x, y, z) order, z fastest; SU(2)
 * as quaternions, read in either form) to and from the device's fundamental
 * links.  The reader refuses another NG or lattice size and reports the stored
 * and the recomputed plaquette (the reference warns when they differ by more
 * than 1e-12); call hrgpu_represent_gauge_field afterwards. */
int hrgpu_write_gauge_field(const char *filename);
int hrgpu_read_gauge_field(const char *filename, double *plaq_file, double *plaq_read);

/* ------------------------------------------------------ batched (multi-RHS) -- */
/* HiRep has no batched interface; these entry points serve its callers that
 * hold many sources at once (calc_prop.c:210-289 loops cg_mshift over the 4*NF
 * spin-colour point sources; force_rhmc.c:24-112 solves one source for many
 * shifts).  A batch of nb even-parity fields is one device buffer in tiles of 4
 * fields (the last tile padded) and blocks of 8 sites: element (component c,
 * site n, field f) at
 *   (((f/4) * ld/8 + n/8) * 4NF + c) * 32 + (n%8) * 4 + f%4,
 * where a single field has its element (c, n) at c*ld + n (ld: a multiple of 32).  hrgpu_batch_bytes
 * gives its size (0 if not initialised or nb <= 0).  pack/unpack move nb
 * separate device fields (the layout of hrgpu_spinor_upload) into a batch and
 * back; nb <= 64. */
size_t hrgpu_batch_bytes(int prec, int nb);
int hrgpu_batch_pack(void *batch, const void *const *fields, int nb, int prec);
int hrgpu_batch_unpack(void *const *fields, const void *batch, int nb, int prec);
/* one even-odd operator (HRGPU_OP_G5DPHI_EOPRE_SQ, _G5CPHI_EOPRE_SQ, _DPHI_EOPRE,
 * _G5DPHI_EOPRE, _CPHI_EOPRE, _G5CPHI_EOPRE) on every field of a batch; the
 * result of each field is that of the single-field operator, to rounding. */
int hrgpu_apply_op_batch(int op, int prec, double mass, void *out, const void *in, int nb);
/* batch hopping kernel variants (0, 1, 2: one thread per site and field with
 * the register budget of 1, 3, 4 resident blocks per SM; 3: the link products
 * on the tensor cores, tcgen05 kind::tf32 with three products for FP32
 * accuracy, FP32 and complex NF = 6 only, nb <= 32; 4: the same with the
 * neighbours prefetched into shared memory two sites ahead, nb <= 16; 3 and 4
 * run only when pinned; 5: variant 0 with the link products in packed FP32 FMAs,
 * complex representations in FP32 only): -1 (default) autotunes variants 0-2
 * and 5 per precision, epilogue and nb at first use; hrgpu_batch_tuning reports
 * the choice (-1: not tuned yet) and the tuning times in ms (6 entries, -1 for a
 * variant not timed). */
int hrgpu_set_batch_variant(int variant);
int hrgpu_batch_tuning(int prec, int epilogue, int nb, int *chosen, float *ms);
/* cg_mshift for many sources at once (op: g5Dphi_eopre_sq or g5Cphi_eopre_sq).
 * Source s (in[s], a separate FP64 even field) is solved for its nshift[s]
 * shifts: with o_s = nshift[0] + ... + nshift[s-1], out[o_s + i] =
 * (M - shift[o_s + i])^-1 in[s], every system from a zero start (unlike
 * hrgpu_cg_mshift with n == 1).  nsrc <= 32, total systems <= 64.  One Krylov
 * space per source (the multi-shift recursion of cg_mshift.c:24-145), all
 * sources advanced by one batched operator per iteration, the iteration replayed
 * from a captured CUDA graph.  flt = 0: FP64 throughout, then HiRep's true
 * residual check and single-shift restarts (cg_mshift.c:122-179); flt = 1:
 * FP64 defect correction around batched FP32 solves.  Its first round is
 * cg_mshift_flt's (cg_mshift_flt.c:144-276): one multi-shift solve per source;
 * later rounds correct every unconverged system from its own residual (one
 * single-shift Krylov space each), because after an FP32 solve the residuals of
 * different shifts are collinear only up to FP32 noise.  iters[s] (nsrc
 * entries) gets the batched iterations in which source s had a system running,
 * plus its residual evaluations. */
int hrgpu_cg_mshift_batch(int op, double mass, int nsrc, const int *nshift, const double *shift, double err2,
                          int max_iter, const void *const *in, void *const *out, int flt, int *iters);

/* ----------------------------------------------------------------- force -- */
int hrgpu_fermion_force_begin(void);                    /* force_fermion_core.c:935-962 */
/* force_fermion_core (force_fermion_core.c:788-928, UPDATE_EO build): Xs, Ys are
 * full-lattice device fields; with auto_fill_odd their odd halves are overwritten
 * by D_oe (times D_oo^-1 with clover) of the even halves, as in the reference. */
int hrgpu_force_fermion_core(void *Xs, void *Ys, int auto_fill_odd, double dt, double residue);
int hrgpu_force_clover_logdet(double mass, double residue); /* force_fermion_core.c:777-781; no-op for expclover */
/* kernel of the hopping part of force_fermion_core for complex NF <= 6 and real
 * NF = 3: 1 = one thread per link; 2 = two threads per link in two warps (one
 * per pairing of X and Y) with the algebra projection from a constant-memory
 * table; 3 = 2 with the link and the spinor at x prefetched into L2; 4 = 2
 * building the SU(3) symmetric or SU(4) antisymmetric links from the
 * fundamental ones (link modes 3 and 4 of hrgpu_link_recon; elsewhere 2); 5 =
 * 2 with the link staged in shared memory by cp.async; 6 = 5 with the spinor
 * at x staged too (5 and 6: complex links; real ones run 2); 0 = the default
 * (5 for complex links, 2 for real ones).  A tuning control of this library;
 * it has no counterpart in the reference. */
int hrgpu_set_force_variant(int variant);
/* fermion_force_end (force_fermion_core.c:964-993): clover derivative, then adds the
 * accumulated force to the host momentum field force[V][4][NG*NG-1] (HiRep layout) */
int hrgpu_fermion_force_end(double dt, double *force_host);
int hrgpu_clover_force_get(void *host); /* cl_force in HiRep layout [V][6][NF*NF] complex */
/* the accumulator itself, HiRep layout (for tests) */
int hrgpu_force_sum_get(double *host);

#ifdef __cplusplus
}
#endif
#endif
