/*
 * hr_oracle.h -- CPU oracle for the HiRep fermion hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the algorithms of
 * HiRep's LibHR (sofiemartins/HiRep) for the even-odd Wilson/clover Dirac
 * operator, the spinor linear algebra, the multi-shift CG inverters and the
 * pseudofermion force.  It is the checker the GPU library is compared against;
 * nothing in the product links it.  Every function cites the reference file and
 * line range it restates.
 *
 * Conventions (all follow HiRep):
 *   - site indices are HiRep's: even sites [0,V/2), odd sites [V/2,V)
 *     (LibHR/Geometry/geometry_mpi_eo.c walk, serial build);
 *   - a spinor is 4 x NF complex doubles, stored site-major (Include/spinor_field.h:37-56);
 *   - a field of parity 0 (even) holds sites [0,V/2), parity 1 (odd) holds
 *     [V/2,V) at offset ix-V/2, parity 2 (full) holds [0,V);
 *   - the represented link U(ix,mu) is NF x NF row-major at [4*ix+mu]
 *     (Include/field_ordering.h:10), complex, or real for the adjoint
 *     representation (Make/Utils/write_suN_headers.pl:33-36).
 */
#ifndef HR_ORACLE_H
#define HR_ORACLE_H

#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_FUND = 0, ORC_ADJ = 1, ORC_SYM = 2, ORC_ASYM = 3 };
enum { ORC_EVEN = 0, ORC_ODD = 1, ORC_FULL = 2 };

/* lattice / representation setup */
int orc_init(int T, int X, int Y, int Z, int ng, int repr);
int orc_nf(void);
int orc_real_links(void);
int orc_volume(void);
void orc_geometry(int *ipt, int *iup, int *idn);
void orc_set_threads(int n);

/* algebra (Make/Utils/autosun) */
int orc_group_dim(void);
void orc_generators(double complex *gT, double complex *rT, double *norms);
void orc_group_represent(void *v, const double complex *u);
void orc_algebra_project(double *h, const void *m);
void orc_fund_algebra_project(double *h, const double complex *m);
void orc_fund_algebra_represent(double complex *m, const double *h);
void orc_represent_gauge_field(void *uf, const double complex *u, int bc_t_antiperiodic);

/* gauge fields used by the operators (pointers are kept, not copied) */
void orc_set_gauge(const void *uf);
void orc_set_gauge_flt(const void *uf_flt);
void orc_set_mass(double m);

/* Wilson operator, double (LibHR/Update/Dphi.c) */
void orc_Dphi_(double complex *out, int out_par, const double complex *in, int in_par);
void orc_Dphi(double m0, double complex *out, const double complex *in);
void orc_g5Dphi(double m0, double complex *out, const double complex *in);
void orc_g5Dphi_sq(double m0, double complex *out, const double complex *in);
void orc_Dphi_eopre(double m0, double complex *out, const double complex *in);
void orc_Dphi_oepre(double m0, double complex *out, const double complex *in);
void orc_g5Dphi_eopre(double m0, double complex *out, const double complex *in);
void orc_g5Dphi_eopre_sq(double m0, double complex *out, const double complex *in);

/* Wilson operator, single (LibHR/Update/Dphi_flt.c) */
void orc_Dphi_flt_(float complex *out, int out_par, const float complex *in, int in_par);
void orc_Dphi_flt(double m0, float complex *out, const float complex *in);
void orc_g5Dphi_flt(double m0, float complex *out, const float complex *in);
void orc_g5Dphi_sq_flt(double m0, float complex *out, const float complex *in);
void orc_Dphi_eopre_flt(double m0, float complex *out, const float complex *in);
void orc_g5Dphi_eopre_flt(double m0, float complex *out, const float complex *in);
void orc_g5Dphi_eopre_sq_flt(double m0, float complex *out, const float complex *in);

/* clover (LibHR/Update/clover_tools.c, Dphi.c:1081-1290) */
void orc_expclover_init(double csw);
void orc_clover_init(double csw);
void orc_compute_clover_term(void);
void orc_compute_ldl_decomp(double sigma0);
void orc_get_clover_term(double complex *cl);
void orc_get_clover_ldl(double complex *ldl);
void orc_Cphi_(double mass, double complex *out, const double complex *in, int par, int assign);
void orc_Cphi_inv_(double mass, double complex *out, const double complex *in, int par, int assign);
void orc_Cphi(double mass, double complex *out, const double complex *in);
void orc_g5Cphi(double mass, double complex *out, const double complex *in);
void orc_g5Cphi_sq(double mass, double complex *out, const double complex *in);
void orc_Cphi_eopre(double mass, double complex *out, const double complex *in);
void orc_g5Cphi_eopre(double mass, double complex *out, const double complex *in);
void orc_g5Cphi_eopre_sq(double mass, double complex *out, const double complex *in);
void orc_Cphi_diag(double mass, double complex *out, const double complex *in, int par);
void orc_Cphi_diag_inv(double mass, double complex *out, const double complex *in, int par);

/* linear algebra (LibHR/Inverters/TMPL/linear_algebra.c.sdtmpl), n = number of sites */
double orc_sqnorm(int n, const double complex *s);
double orc_prod_re(int n, const double complex *a, const double complex *b);
double orc_prod_im(int n, const double complex *a, const double complex *b);
double orc_g5_prod_re(int n, const double complex *a, const double complex *b);
double orc_g5_prod_im(int n, const double complex *a, const double complex *b);
void orc_mul_add_assign(int n, double complex *s1, double r, const double complex *s2);
void orc_g5(int n, double complex *s1, const double complex *s2);
void orc_gamma(int mu, int n, double complex *s1, const double complex *s2);
float orc_sqnorm_flt_site(const float complex *s);

/* inverters (LibHR/Inverters/cg_mshift.c, cg_mshift_flt.c) */
enum {
  ORC_OP_G5DPHI_SQ = 0, ORC_OP_G5DPHI_EOPRE_SQ = 1, ORC_OP_G5CPHI_EOPRE_SQ = 2, ORC_OP_G5CPHI_SQ = 3,
  ORC_OP_DPHI_EOPRE = 4, ORC_OP_G5DPHI_EOPRE = 5, ORC_OP_CPHI_EOPRE = 6, ORC_OP_G5CPHI_EOPRE = 7,
  ORC_OP_DPHI = 8, ORC_OP_CPHI = 9
};
int orc_cg_mshift(int op, int n, const double *shift, double err2, int max_iter,
                  const double complex *in, double complex *out);
int orc_cg_mshift_flt(int op, int n, const double *shift, double err2, int max_iter,
                      const double complex *in, double complex *out);
/* g5QMR_mshift, MINRES (LibHR/Inverters/g5QMR_mshift.c, MINRES.c) and the MRE guess (LibHR/Update/mre.c) */
int orc_g5QMR_mshift(int op, int n, const double *shift, double err2, int max_iter,
                     const double complex *in, double complex *out);
int orc_MINRES(int op, int g5, double sh, double err2, int max_iter, const double complex *in,
               double complex *out, const double complex *trial);
void orc_mre_guess(int op, int max, const double complex *s, double complex *out, const double complex *pf);

/* force (LibHR/Update/force_fermion_core.c) */
void orc_fermion_force_begin(void);
void orc_force_fermion_core(double complex *Xs, double complex *Ys, int auto_fill_odd, double dt, double residue);
void orc_clover_la_logdet(double nf, double mass, double *la);
void orc_force_clover_logdet(double mass, double residue);
void orc_fermion_force_end(double dt, double *force);
void orc_get_force_sum(double *f);
void orc_get_clover_force(double complex *cf);

/* HMC pieces (LibHR/Update/force0.c, staples.c, field_update.c, local_action.c, suN_utils.c) */
void orc_force0(double dt, double beta, const double complex *u, double *mom);
void orc_update_gauge_field(double dt, double complex *u, const double *mom);
void orc_project_gauge_field(double complex *u);
void orc_local_hmc_action(double beta, const double complex *u, const double *mom, double *loc);

/* gauge utilities used by tests */
double orc_avr_plaquette(const double complex *u);

#ifdef __cplusplus
}
#endif
#endif
