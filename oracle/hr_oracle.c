/*
 * hr_oracle.c -- CPU oracle for the HiRep fermion hot path (TEST INFRASTRUCTURE).
 *
 * A plain-C restatement of HiRep's LibHR algorithms for the serial (no MPI)
 * build, with NG, NF and the representation chosen at run time instead of at
 * compile time.  Used only by tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py, as the checker.  The GPU library never calls it.
 *
 * Each section cites the reference file:line it restates (paths relative to the
 * HiRep source tree).
 */
#include "hr_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;
typedef float complex fcplx;

/* ------------------------------------------------------------------------- */
/* global state (mirrors Include/global.h for the serial build)              */
/* ------------------------------------------------------------------------- */
static int T_, X_, Y_, Z_, V_, VH_;
static int *ipt_ = NULL, *iup_ = NULL, *idn_ = NULL;
static int NG_, NF_, REPR_, REAL_, DIMG_;
static cplx *gT_ = NULL;   /* group generators T_A, NG x NG, DIMG of them        */
static cplx *rT_ = NULL;   /* represented generators R(iT_A), NF x NF            */
static double fund_norm2_, repr_norm2_;
static const void *uf_ = NULL;     /* represented links, double                  */
static const void *uf_flt_ = NULL; /* represented links, float                   */
static double static_mass_ = 0.0;

/* clover state (LibHR/Update/clover_tools.c:17-20, Include/global.h) */
static double csw_ = 0.0;
static double sigma_ = 0xF00F;
static cplx *cl_term_ = NULL;  /* [V][4][NF*NF]                                  */
static cplx *cl_ldl_ = NULL;   /* [V][2][NF*(2NF+1)]  (up, dn)                   */
static cplx *cl_force_ = NULL; /* [V][6][NF*NF]  (real part only for real reps)  */
static double *force_sum_ = NULL; /* [V][4][DIMG]                               */

#define SPN (4 * NF_) /* complex numbers per spinor */

void orc_set_threads(int n)
{
#ifdef _OPENMP
  omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* ------------------------------------------------------------------------- */
/* geometry: serial even-odd walk                                             */
/* LibHR/Geometry/geometry_mpi_eo.c:449-498 (walk_on_lattice, level 4, path   */
/* blocks PB_T..PB_Z = 2 from Include/global.h:64-67), :713-729               */
/* (set_border_pointer: ids in walk order), :1327-1352 (fix_next_neightbours) */
/* For NP_*=1 dir_mask puts X innermost, then Y, Z and T outermost            */
/* (:286-330), so blocks are walked T,Z,Y,X outer->inner and sites inside a   */
/* 2^4 block likewise.  Even sites are walked first (set_inner(even)), then   */
/* odd (:1919-1953).                                                          */
/* ------------------------------------------------------------------------- */
static int overlexi(int t, int x, int y, int z)
{
  t = (t + T_) % T_; x = (x + X_) % X_; y = (y + Y_) % Y_; z = (z + Z_) % Z_;
  return t + T_ * (x + X_ * (y + Y_ * z));
}

static void build_geometry(void)
{
  int *map = malloc(sizeof(int) * V_);
  for (int i = 0; i < V_; i++) map[i] = -1;
  int id = 0;
  for (int eo = 0; eo < 2; eo++)
    for (int bt = 0; bt < T_; bt += 2)
      for (int bz = 0; bz < Z_; bz += 2)
        for (int by = 0; by < Y_; by += 2)
          for (int bx = 0; bx < X_; bx += 2)
            for (int dt = 0; dt < 2 && bt + dt < T_; dt++)
              for (int dz = 0; dz < 2 && bz + dz < Z_; dz++)
                for (int dy = 0; dy < 2 && by + dy < Y_; dy++)
                  for (int dx = 0; dx < 2 && bx + dx < X_; dx++)
                  {
                    int t = bt + dt, x = bx + dx, y = by + dy, z = bz + dz;
                    if ((t + x + y + z) % 2 != eo) continue;
                    int l = overlexi(t, x, y, z);
                    if (map[l] == -1) map[l] = id++;
                  }
  for (int z = 0; z < Z_; z++)
    for (int y = 0; y < Y_; y++)
      for (int x = 0; x < X_; x++)
        for (int t = 0; t < T_; t++)
        {
          int ix = map[overlexi(t, x, y, z)];
          ipt_[((t * X_ + x) * Y_ + y) * Z_ + z] = ix;
          iup_[4 * ix + 0] = map[overlexi(t + 1, x, y, z)];
          idn_[4 * ix + 0] = map[overlexi(t - 1, x, y, z)];
          iup_[4 * ix + 1] = map[overlexi(t, x + 1, y, z)];
          idn_[4 * ix + 1] = map[overlexi(t, x - 1, y, z)];
          iup_[4 * ix + 2] = map[overlexi(t, x, y + 1, z)];
          idn_[4 * ix + 2] = map[overlexi(t, x, y - 1, z)];
          iup_[4 * ix + 3] = map[overlexi(t, x, y, z + 1)];
          idn_[4 * ix + 3] = map[overlexi(t, x, y, z - 1)];
        }
  free(map);
}

/* ------------------------------------------------------------------------- */
/* generators: Make/Utils/autosun/sun.h:27-74 (group T_A, scaled by 1/2,      */
/* Tnorm = 1/2), fundamental.h:18-30, adjoint.h:20-61, symmetric.h:20-66,     */
/* antisymmetric.h:20-62 (representation basis e and R(iT_A), iTnorm),        */
/* representation.h:30-58 (algebra_project: h_A = Re Tr[R(iT_A)^+ m]/iTnorm) */
/* ------------------------------------------------------------------------- */
static void mat_mul(int n, cplx *c, const cplx *a, const cplx *b)
{
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
    {
      cplx s = 0;
      for (int k = 0; k < n; k++) s += a[i * n + k] * b[k * n + j];
      c[i * n + j] = s;
    }
}

static cplx mat_trace(int n, const cplx *a)
{
  cplx s = 0;
  for (int i = 0; i < n; i++) s += a[i * n + i];
  return s;
}

static void build_generators(void)
{
  int N = NG_;
  DIMG_ = N * N - 1;
  gT_ = calloc((size_t)DIMG_ * N * N, sizeof(cplx));
  int A = 0;
  for (int a = 0; a < N; a++)
    for (int b = 0; b < N; b++)
    {
      cplx *t = gT_ + (size_t)A * N * N;
      if (a > b) { t[a * N + b] = 1.0; t[b * N + a] = 1.0; A++; }
      else if (a < b) { t[a * N + b] = I; t[b * N + a] = -I; A++; }
      else if (a != 0)
      {
        double n = sqrt(2. / (a * (a + 1.)));
        for (int k = 0; k < a; k++) t[k * N + k] = n;
        t[a * N + a] = -a * n;
        A++;
      }
    }
  for (int i = 0; i < DIMG_ * N * N; i++) gT_[i] *= 0.5;
  fund_norm2_ = 0.5;

  int F = NF_;
  rT_ = calloc((size_t)DIMG_ * F * F, sizeof(cplx));
  cplx *tmp = malloc(sizeof(cplx) * N * N), *tmp1 = malloc(sizeof(cplx) * N * N);
  cplx *e = NULL;
  if (REPR_ == ORC_FUND)
  {
    for (int C = 0; C < DIMG_; C++)
      for (int k = 0; k < N * N; k++) rT_[(size_t)C * F * F + k] = I * gT_[(size_t)C * N * N + k];
    repr_norm2_ = 0.5;
  }
  else if (REPR_ == ORC_ADJ)
  {
    e = calloc((size_t)F * N * N, sizeof(cplx));
    for (int C = 0; C < F; C++)
      for (int k = 0; k < N * N; k++) e[(size_t)C * N * N + k] = gT_[(size_t)C * N * N + k] / sqrt(0.5);
    for (int C = 0; C < DIMG_; C++)
      for (int a = 0; a < F; a++)
      {
        /* tmp = -e_a T_C + T_C e_a */
        mat_mul(N, tmp, e + (size_t)a * N * N, gT_ + (size_t)C * N * N);
        mat_mul(N, tmp1, gT_ + (size_t)C * N * N, e + (size_t)a * N * N);
        for (int k = 0; k < N * N; k++) tmp[k] = tmp1[k] - tmp[k];
        for (int b = 0; b < F; b++)
        {
          cplx *t2 = malloc(sizeof(cplx) * N * N);
          mat_mul(N, t2, tmp, e + (size_t)b * N * N);
          cplx tr = mat_trace(N, t2);
          free(t2);
          rT_[(size_t)C * F * F + b * F + a] = -cimag(tr);
        }
      }
    repr_norm2_ = 2. * 0.5 * N;
  }
  else
  {
    e = calloc((size_t)F * N * N, sizeof(cplx));
    int C = 0;
    if (REPR_ == ORC_SYM)
    {
      for (int a = 0; a < N; a++)
      {
        for (int b = 0; b < a; b++)
        {
          e[(size_t)C * N * N + a * N + b] = sqrt(.5);
          e[(size_t)C * N * N + b * N + a] = sqrt(.5);
          C++;
        }
        e[(size_t)C * N * N + a * N + a] = 1.0;
        C++;
      }
    }
    else
    {
      for (int a = 1; a < N; a++)
        for (int b = 0; b < a; b++)
        {
          e[(size_t)C * N * N + a * N + b] = sqrt(.5);
          e[(size_t)C * N * N + b * N + a] = -sqrt(.5);
          C++;
        }
    }
    cplx fac = (REPR_ == ORC_SYM) ? 2.0 * I : -2.0 * I;
    for (C = 0; C < DIMG_; C++)
      for (int a = 0; a < F; a++)
      {
        mat_mul(N, tmp, e + (size_t)a * N * N, gT_ + (size_t)C * N * N);
        for (int b = 0; b < F; b++)
        {
          mat_mul(N, tmp1, tmp, e + (size_t)b * N * N);
          rT_[(size_t)C * F * F + a * F + b] = fac * mat_trace(N, tmp1);
        }
      }
    repr_norm2_ = (REPR_ == ORC_SYM) ? (N + 2.) * 0.5 : (N - 2.) * 0.5;
  }
  free(e);
  free(tmp);
  free(tmp1);
}

int orc_group_dim(void) { return DIMG_; }

void orc_generators(cplx *gT, cplx *rT, double *norms)
{
  if (gT) memcpy(gT, gT_, sizeof(cplx) * DIMG_ * NG_ * NG_);
  if (rT) memcpy(rT, rT_, sizeof(cplx) * DIMG_ * NF_ * NF_);
  if (norms) { norms[0] = fund_norm2_; norms[1] = repr_norm2_; }
}

/* h_A = Re Tr[R(iT_A)^+ m] / C(R)   (autosun/representation.h:36-58) */
void orc_algebra_project(double *h, const void *m)
{
  int F = NF_;
  for (int A = 0; A < DIMG_; A++)
  {
    const cplx *t = rT_ + (size_t)A * F * F;
    double s = 0;
    if (REAL_)
    {
      const double *mr = (const double *)m;
      for (int k = 0; k < F * F; k++) s += creal(t[k]) * mr[k];
    }
    else
    {
      const cplx *mc = (const cplx *)m;
      for (int k = 0; k < F * F; k++) s += creal(conj(t[k]) * mc[k]);
    }
    h[A] = s / repr_norm2_;
  }
}

/* autosun/sun.h:203-241 */
void orc_fund_algebra_project(double *h, const cplx *m)
{
  int N = NG_;
  for (int A = 0; A < DIMG_; A++)
  {
    double s = 0;
    for (int k = 0; k < N * N; k++) s += creal(conj(I * gT_[(size_t)A * N * N + k]) * m[k]);
    h[A] = s / fund_norm2_;
  }
}

/* m = sum_A h_A iT_A  (autosun/sun.h:181-200) */
void orc_fund_algebra_represent(cplx *m, const double *h)
{
  int N = NG_;
  for (int k = 0; k < N * N; k++) m[k] = 0;
  for (int A = 0; A < DIMG_; A++)
    for (int k = 0; k < N * N; k++) m[k] += h[A] * I * gT_[(size_t)A * N * N + k];
}

/* ------------------------------------------------------------------------- */
/* group representation: LibHR/Update/representation.c:16-200               */
/* (_group_represent2, explicit formulas per representation)                 */
/* ------------------------------------------------------------------------- */
#define XG(m, a, b) ((m)[(a) * NG_ + (b)])
#define XF(m, a, b) ((m)[(a) * NF_ + (b)])

void orc_group_represent(void *v, const cplx *u)
{
  int N = NG_;
  cplx *mf = malloc(sizeof(cplx) * N * N);
  if (REPR_ == ORC_FUND)
  {
    memcpy(v, u, sizeof(cplx) * N * N);
  }
  else if (REPR_ == ORC_ADJ)
  {
    double *vf = (double *)v;
    int A = 0;
    for (int a = 0; a < N; a++)
      for (int b = (a == 0) ? 1 : 0; b < N; b++)
      {
        for (int i = 0; i < N; i++)
          for (int j = i; j < N; j++)
          {
            if (a > b)
              XG(mf, i, j) = XG(u, i, a) * conj(XG(u, j, b)) + XG(u, i, b) * conj(XG(u, j, a));
            else if (a < b)
              XG(mf, i, j) = I * (XG(u, i, a) * conj(XG(u, j, b))) - I * (XG(u, i, b) * conj(XG(u, j, a)));
            else
            {
              XG(mf, i, j) = -a * XG(u, i, a) * conj(XG(u, j, a));
              for (int k = 0; k < a; k++) XG(mf, i, j) += XG(u, i, k) * conj(XG(u, j, k));
              XG(mf, i, j) *= sqrt(2. / (a * (a + 1.)));
            }
          }
        int C = 0;
        for (int c = 0; c < N; c++)
          for (int d = (c == 0) ? 1 : 0; d < N; d++)
          {
            if (c > d)
              XF(vf, C, A) = creal(XG(mf, d, c));
            else if (c < d)
              XF(vf, C, A) = cimag(XG(mf, c, d));
            else
            {
              XF(vf, C, A) = -c * creal(XG(mf, c, c));
              for (int k = 0; k < c; k++) XF(vf, C, A) += creal(XG(mf, k, k));
              XF(vf, C, A) *= sqrt(.5 / (c * (c + 1.)));
            }
            C++;
          }
        A++;
      }
  }
  else if (REPR_ == ORC_SYM)
  {
    const double st = sqrt(2.);
    cplx *vf = (cplx *)v;
    int A = 0;
    for (int a = 0; a < N; a++)
    {
      for (int b = 0; b < a; b++)
      {
        for (int i = 0; i < N; i++)
          for (int j = i; j < N; j++)
            XG(mf, i, j) = XG(u, i, a) * XG(u, j, b) + XG(u, i, b) * XG(u, j, a);
        int C = 0;
        for (int c = 0; c < N; c++)
        {
          for (int d = 0; d < c; d++) { XF(vf, C, A) = XG(mf, d, c); C++; }
          XF(vf, C, A) = XG(mf, c, c) / st;
          C++;
        }
        A++;
      }
      for (int i = 0; i < N; i++)
        for (int j = i; j < N; j++) XG(mf, i, j) = XG(u, i, a) * XG(u, j, a);
      int C = 0;
      for (int c = 0; c < N; c++)
      {
        for (int d = 0; d < c; d++) { XF(vf, C, A) = XG(mf, d, c) * st; C++; }
        XF(vf, C, A) = XG(mf, c, c);
        C++;
      }
      A++;
    }
  }
  else
  {
    cplx *vf = (cplx *)v;
    int A = 0;
    for (int a = 1; a < N; a++)
      for (int b = 0; b < a; b++)
      {
        for (int i = 0; i < N; i++)
          for (int j = i; j < N; j++)
            XG(mf, i, j) = XG(u, i, a) * XG(u, j, b) - XG(u, i, b) * XG(u, j, a);
        int C = 0;
        for (int c = 1; c < N; c++)
          for (int d = 0; d < c; d++) { XF(vf, C, A) = -XG(mf, d, c); C++; }
        A++;
      }
  }
  free(mf);
}

/* represent_gauge_field (representation.c:391-468) followed by the          */
/* antiperiodic-T sign on U(t=0,mu=0) (Utils/boundary_conditions.c:321-341)   */
void orc_represent_gauge_field(void *uf, const cplx *u, int bc_t_antiperiodic)
{
  int F = NF_, N = NG_;
  size_t lsz = REAL_ ? sizeof(double) * F * F : sizeof(cplx) * F * F;
#pragma omp parallel for
  for (int ix = 0; ix < V_; ix++)
    for (int mu = 0; mu < 4; mu++)
      orc_group_represent((char *)uf + lsz * (4 * (size_t)ix + mu), u + (size_t)(4 * ix + mu) * N * N);
  if (bc_t_antiperiodic)
  {
    for (int x = 0; x < X_; x++)
      for (int y = 0; y < Y_; y++)
        for (int z = 0; z < Z_; z++)
        {
          int ix = ipt_[((0 * X_ + x) * Y_ + y) * Z_ + z];
          if (REAL_)
          {
            double *p = (double *)uf + (size_t)(4 * ix) * F * F;
            for (int k = 0; k < F * F; k++) p[k] = -p[k];
          }
          else
          {
            cplx *p = (cplx *)uf + (size_t)(4 * ix) * F * F;
            for (int k = 0; k < F * F; k++) p[k] = -p[k];
          }
        }
  }
}

int orc_init(int T, int X, int Y, int Z, int ng, int repr)
{
  if (T <= 0 || X <= 0 || Y <= 0 || Z <= 0 || ng < 2 || repr < 0 || repr > 3) return -1;
  if (repr == ORC_ASYM && ng < 3) return -1;
  free(ipt_); free(iup_); free(idn_); free(gT_); free(rT_);
  free(cl_term_); free(cl_ldl_); free(cl_force_); free(force_sum_);
  cl_term_ = NULL; cl_ldl_ = NULL; cl_force_ = NULL; force_sum_ = NULL;
  T_ = T; X_ = X; Y_ = Y; Z_ = Z;
  V_ = T * X * Y * Z;
  VH_ = V_ / 2;
  ipt_ = malloc(sizeof(int) * V_);
  iup_ = malloc(sizeof(int) * 4 * V_);
  idn_ = malloc(sizeof(int) * 4 * V_);
  NG_ = ng;
  REPR_ = repr;
  REAL_ = (repr == ORC_ADJ);
  NF_ = (repr == ORC_FUND) ? ng : (repr == ORC_ADJ) ? ng * ng - 1 : (repr == ORC_SYM) ? ng * (ng + 1) / 2 : ng * (ng - 1) / 2;
  build_geometry();
  build_generators();
  uf_ = NULL;
  uf_flt_ = NULL;
  sigma_ = 0xF00F;
  return 0;
}

int orc_nf(void) { return NF_; }
int orc_real_links(void) { return REAL_; }
int orc_volume(void) { return V_; }

void orc_geometry(int *ipt, int *iup, int *idn)
{
  if (ipt) memcpy(ipt, ipt_, sizeof(int) * V_);
  if (iup) memcpy(iup, iup_, sizeof(int) * 4 * V_);
  if (idn) memcpy(idn, idn_, sizeof(int) * 4 * V_);
}

void orc_set_gauge(const void *uf) { uf_ = uf; }
void orc_set_gauge_flt(const void *uf) { uf_flt_ = uf; }
void orc_set_mass(double m) { static_mass_ = m; }

/* ------------------------------------------------------------------------- */
/* link x vector products: Make/Utils/write_suN_headers.pl:1414-1489          */
/* (_suNf_multiply r=U s) and :1628-1707 (_suNf_inverse_multiply r=U^+ s);    */
/* real links for the adjoint representation                                  */
/* ------------------------------------------------------------------------- */
static inline void link_mul(cplx *r, int ix, int mu, const cplx *s)
{
  int F = NF_;
  if (REAL_)
  {
    const double *u = (const double *)uf_ + (size_t)(4 * ix + mu) * F * F;
    for (int i = 0; i < F; i++)
    {
      cplx a = u[i * F] * s[0];
      for (int j = 1; j < F; j++) a += u[i * F + j] * s[j];
      r[i] = a;
    }
  }
  else
  {
    const cplx *u = (const cplx *)uf_ + (size_t)(4 * ix + mu) * F * F;
    for (int i = 0; i < F; i++)
    {
      cplx a = u[i * F] * s[0];
      for (int j = 1; j < F; j++) a += u[i * F + j] * s[j];
      r[i] = a;
    }
  }
}

static inline void link_dag_mul(cplx *r, int ix, int mu, const cplx *s)
{
  int F = NF_;
  if (REAL_)
  {
    const double *u = (const double *)uf_ + (size_t)(4 * ix + mu) * F * F;
    for (int i = 0; i < F; i++)
    {
      cplx a = u[i] * s[0];
      for (int j = 1; j < F; j++) a += u[j * F + i] * s[j];
      r[i] = a;
    }
  }
  else
  {
    const cplx *u = (const cplx *)uf_ + (size_t)(4 * ix + mu) * F * F;
    for (int i = 0; i < F; i++)
    {
      cplx a = s[0] * conj(u[i]);
      for (int j = 1; j < F; j++) a += s[j] * conj(u[j * F + i]);
      r[i] = a;
    }
  }
}

static inline void link_mul_flt(fcplx *r, int ix, int mu, const fcplx *s)
{
  int F = NF_;
  if (REAL_)
  {
    const float *u = (const float *)uf_flt_ + (size_t)(4 * ix + mu) * F * F;
    for (int i = 0; i < F; i++)
    {
      fcplx a = u[i * F] * s[0];
      for (int j = 1; j < F; j++) a += u[i * F + j] * s[j];
      r[i] = a;
    }
  }
  else
  {
    const fcplx *u = (const fcplx *)uf_flt_ + (size_t)(4 * ix + mu) * F * F;
    for (int i = 0; i < F; i++)
    {
      fcplx a = u[i * F] * s[0];
      for (int j = 1; j < F; j++) a += u[i * F + j] * s[j];
      r[i] = a;
    }
  }
}

static inline void link_dag_mul_flt(fcplx *r, int ix, int mu, const fcplx *s)
{
  int F = NF_;
  if (REAL_)
  {
    const float *u = (const float *)uf_flt_ + (size_t)(4 * ix + mu) * F * F;
    for (int i = 0; i < F; i++)
    {
      fcplx a = u[i] * s[0];
      for (int j = 1; j < F; j++) a += u[j * F + i] * s[j];
      r[i] = a;
    }
  }
  else
  {
    const fcplx *u = (const fcplx *)uf_flt_ + (size_t)(4 * ix + mu) * F * F;
    for (int i = 0; i < F; i++)
    {
      fcplx a = s[0] * conjf(u[i]);
      for (int j = 1; j < F; j++) a += s[j] * conjf(u[j * F + i]);
      r[i] = a;
    }
  }
}

static int par_base(int par) { return par == ORC_ODD ? VH_ : 0; }
static int par_end(int par) { return par == ORC_EVEN ? VH_ : V_; }


/* ------------------------------------------------------------------------- */
/* hopping term: LibHR/Update/Dphi.c:193-374 (Dphi_), chiral gamma basis      */
/* (Doc/hirep.tex:581-618).  The same body in float: Dphi_flt.c:162-364.      */
/* ------------------------------------------------------------------------- */
#define HOP_BODY(CT, MUL, DMUL, HALF)                                                   \
  int F = NF_;                                                                        \
  int ob = par_base(out_par), ib = par_base(in_par);                                  \
  _Pragma("omp parallel for") for (int ix = ob; ix < par_end(out_par); ix++)          \
  {                                                                                   \
    CT r[4][64], psi[64], psi2[64], chi[64], chi2[64];                                \
    const CT *s;                                                                      \
    int iy;                                                                           \
    /* +0 */                                                                          \
    iy = iup_[4 * ix + 0]; s = in + (size_t)(iy - ib) * 4 * F;                        \
    for (int i = 0; i < F; i++) { psi[i] = s[i] + s[2 * F + i]; psi2[i] = s[F + i] + s[3 * F + i]; } \
    MUL(chi, ix, 0, psi); MUL(chi2, ix, 0, psi2);                                     \
    for (int i = 0; i < F; i++) { r[0][i] = chi[i]; r[2][i] = chi[i]; r[1][i] = chi2[i]; r[3][i] = chi2[i]; } \
    /* -0 */                                                                          \
    iy = idn_[4 * ix + 0]; s = in + (size_t)(iy - ib) * 4 * F;                        \
    for (int i = 0; i < F; i++) { psi[i] = s[i] - s[2 * F + i]; psi2[i] = s[F + i] - s[3 * F + i]; } \
    DMUL(chi, iy, 0, psi); DMUL(chi2, iy, 0, psi2);                                   \
    for (int i = 0; i < F; i++) { r[0][i] += chi[i]; r[2][i] -= chi[i]; r[1][i] += chi2[i]; r[3][i] -= chi2[i]; } \
    /* +1 */                                                                          \
    iy = iup_[4 * ix + 1]; s = in + (size_t)(iy - ib) * 4 * F;                        \
    for (int i = 0; i < F; i++) { psi[i] = s[i] + I * s[3 * F + i]; psi2[i] = s[F + i] + I * s[2 * F + i]; } \
    MUL(chi, ix, 1, psi); MUL(chi2, ix, 1, psi2);                                     \
    for (int i = 0; i < F; i++) { r[0][i] += chi[i]; r[3][i] -= I * chi[i]; r[1][i] += chi2[i]; r[2][i] -= I * chi2[i]; } \
    /* -1 */                                                                          \
    iy = idn_[4 * ix + 1]; s = in + (size_t)(iy - ib) * 4 * F;                        \
    for (int i = 0; i < F; i++) { psi[i] = s[i] - I * s[3 * F + i]; psi2[i] = s[F + i] - I * s[2 * F + i]; } \
    DMUL(chi, iy, 1, psi); DMUL(chi2, iy, 1, psi2);                                   \
    for (int i = 0; i < F; i++) { r[0][i] += chi[i]; r[3][i] += I * chi[i]; r[1][i] += chi2[i]; r[2][i] += I * chi2[i]; } \
    /* +2 */                                                                          \
    iy = iup_[4 * ix + 2]; s = in + (size_t)(iy - ib) * 4 * F;                        \
    for (int i = 0; i < F; i++) { psi[i] = s[i] + s[3 * F + i]; psi2[i] = s[F + i] - s[2 * F + i]; } \
    MUL(chi, ix, 2, psi); MUL(chi2, ix, 2, psi2);                                     \
    for (int i = 0; i < F; i++) { r[0][i] += chi[i]; r[3][i] += chi[i]; r[1][i] += chi2[i]; r[2][i] -= chi2[i]; } \
    /* -2 */                                                                          \
    iy = idn_[4 * ix + 2]; s = in + (size_t)(iy - ib) * 4 * F;                        \
    for (int i = 0; i < F; i++) { psi[i] = s[i] - s[3 * F + i]; psi2[i] = s[F + i] + s[2 * F + i]; } \
    DMUL(chi, iy, 2, psi); DMUL(chi2, iy, 2, psi2);                                   \
    for (int i = 0; i < F; i++) { r[0][i] += chi[i]; r[3][i] -= chi[i]; r[1][i] += chi2[i]; r[2][i] += chi2[i]; } \
    /* +3 */                                                                          \
    iy = iup_[4 * ix + 3]; s = in + (size_t)(iy - ib) * 4 * F;                        \
    for (int i = 0; i < F; i++) { psi[i] = s[i] + I * s[2 * F + i]; psi2[i] = s[F + i] - I * s[3 * F + i]; } \
    MUL(chi, ix, 3, psi); MUL(chi2, ix, 3, psi2);                                     \
    for (int i = 0; i < F; i++) { r[0][i] += chi[i]; r[2][i] -= I * chi[i]; r[1][i] += chi2[i]; r[3][i] += I * chi2[i]; } \
    /* -3 */                                                                          \
    iy = idn_[4 * ix + 3]; s = in + (size_t)(iy - ib) * 4 * F;                        \
    for (int i = 0; i < F; i++) { psi[i] = s[i] - I * s[2 * F + i]; psi2[i] = s[F + i] + I * s[3 * F + i]; } \
    DMUL(chi, iy, 3, psi); DMUL(chi2, iy, 3, psi2);                                   \
    for (int i = 0; i < F; i++) { r[0][i] += chi[i]; r[2][i] += I * chi[i]; r[1][i] += chi2[i]; r[3][i] -= I * chi2[i]; } \
    CT *o = out + (size_t)(ix - ob) * 4 * F;                                          \
    for (int k = 0; k < 4; k++)                                                       \
      for (int i = 0; i < F; i++) o[k * F + i] = HALF * r[k][i];                      \
  }

void orc_Dphi_(cplx *out, int out_par, const cplx *in, int in_par)
{
  HOP_BODY(cplx, link_mul, link_dag_mul, -0.5)
}

void orc_Dphi_flt_(fcplx *out, int out_par, const fcplx *in, int in_par)
{
  HOP_BODY(fcplx, link_mul_flt, link_dag_mul_flt, -0.5f)
}

/* ------------------------------------------------------------------------- */
/* spinor linear algebra: LibHR/Inverters/TMPL/linear_algebra.c.sdtmpl       */
/* (per-site products in the field's precision, accumulated in double)        */
/* ------------------------------------------------------------------------- */
double orc_sqnorm(int n, const cplx *s)
{
  double res = 0;
  size_t m = (size_t)n * SPN;
#pragma omp parallel for reduction(+ : res)
  for (int ix = 0; ix < n; ix++)
  {
    double p = 0;
    const cplx *a = s + (size_t)ix * SPN;
    for (int k = 0; k < SPN; k++) p += creal(a[k]) * creal(a[k]) + cimag(a[k]) * cimag(a[k]);
    res += p;
  }
  (void)m;
  return res;
}

double orc_prod_re(int n, const cplx *a, const cplx *b)
{
  double res = 0;
#pragma omp parallel for reduction(+ : res)
  for (int ix = 0; ix < n; ix++)
  {
    double p = 0;
    for (int k = 0; k < SPN; k++) p += creal(conj(a[(size_t)ix * SPN + k]) * b[(size_t)ix * SPN + k]);
    res += p;
  }
  return res;
}

double orc_prod_im(int n, const cplx *a, const cplx *b)
{
  double res = 0;
#pragma omp parallel for reduction(+ : res)
  for (int ix = 0; ix < n; ix++)
  {
    double p = 0;
    for (int k = 0; k < SPN; k++) p += cimag(conj(a[(size_t)ix * SPN + k]) * b[(size_t)ix * SPN + k]);
    res += p;
  }
  return res;
}

double orc_g5_prod_re(int n, const cplx *a, const cplx *b)
{
  double res = 0;
#pragma omp parallel for reduction(+ : res)
  for (int ix = 0; ix < n; ix++)
  {
    double p = 0;
    for (int k = 0; k < SPN; k++)
      p += (k < 2 * NF_ ? 1.0 : -1.0) * creal(conj(a[(size_t)ix * SPN + k]) * b[(size_t)ix * SPN + k]);
    res += p;
  }
  return res;
}

double orc_g5_prod_im(int n, const cplx *a, const cplx *b)
{
  double res = 0;
#pragma omp parallel for reduction(+ : res)
  for (int ix = 0; ix < n; ix++)
  {
    double p = 0;
    for (int k = 0; k < SPN; k++)
      p += (k < 2 * NF_ ? 1.0 : -1.0) * cimag(conj(a[(size_t)ix * SPN + k]) * b[(size_t)ix * SPN + k]);
    res += p;
  }
  return res;
}

void orc_mul_add_assign(int n, cplx *s1, double r, const cplx *s2)
{
  size_t m = (size_t)n * SPN;
#pragma omp parallel for
  for (size_t k = 0; k < m; k++) s1[k] += r * s2[k];
}

static void la_mul(int n, cplx *s1, double r, const cplx *s2)
{
  size_t m = (size_t)n * SPN;
#pragma omp parallel for
  for (size_t k = 0; k < m; k++) s1[k] = r * s2[k];
}

static void la_sub(int n, cplx *r, const cplx *a, const cplx *b)
{
  size_t m = (size_t)n * SPN;
#pragma omp parallel for
  for (size_t k = 0; k < m; k++) r[k] = a[k] - b[k];
}

static void la_add_assign(int n, cplx *a, const cplx *b)
{
  size_t m = (size_t)n * SPN;
#pragma omp parallel for
  for (size_t k = 0; k < m; k++) a[k] += b[k];
}

static void la_minus(int n, cplx *a, const cplx *b)
{
  size_t m = (size_t)n * SPN;
#pragma omp parallel for
  for (size_t k = 0; k < m; k++) a[k] = -b[k];
}

/* s1 = g5 s2: gamma_5 = diag(1,1,-1,-1) (write_suN_headers.pl:3112-3128) */
void orc_g5(int n, cplx *s1, const cplx *s2)
{
#pragma omp parallel for
  for (int ix = 0; ix < n; ix++)
    for (int k = 0; k < SPN; k++)
      s1[(size_t)ix * SPN + k] = (k < 2 * NF_) ? s2[(size_t)ix * SPN + k] : -s2[(size_t)ix * SPN + k];
}

/* s1 = g_mu s2 (Include/gamma_spinor.h:36-58) */
void orc_gamma(int mu, int n, cplx *s1, const cplx *s2)
{
  int F = NF_;
  static const int src[4][4] = {{2, 3, 0, 1}, {3, 2, 1, 0}, {3, 2, 1, 0}, {2, 3, 0, 1}};
  const cplx fac[4][4] = {{-1, -1, -1, -1}, {-I, -I, I, I}, {-1, 1, 1, -1}, {-I, I, I, -I}};
  for (int ix = 0; ix < n; ix++)
    for (int c = 0; c < 4; c++)
      for (int i = 0; i < F; i++)
        s1[(size_t)ix * SPN + c * F + i] = fac[mu][c] * s2[(size_t)ix * SPN + src[mu][c] * F + i];
}

/* float helpers (same template instantiated for float, _f_flt) */
static double la_sqnorm_flt(int n, const fcplx *s)
{
  double res = 0;
#pragma omp parallel for reduction(+ : res)
  for (int ix = 0; ix < n; ix++)
  {
    float p = 0;
    for (int k = 0; k < SPN; k++) p += crealf(s[(size_t)ix * SPN + k]) * crealf(s[(size_t)ix * SPN + k]) + cimagf(s[(size_t)ix * SPN + k]) * cimagf(s[(size_t)ix * SPN + k]);
    res += (double)p;
  }
  return res;
}

float orc_sqnorm_flt_site(const fcplx *s)
{
  float p = 0;
  for (int k = 0; k < SPN; k++) p += crealf(s[k]) * crealf(s[k]) + cimagf(s[k]) * cimagf(s[k]);
  return p;
}

static double la_prod_re_flt(int n, const fcplx *a, const fcplx *b)
{
  double res = 0;
#pragma omp parallel for reduction(+ : res)
  for (int ix = 0; ix < n; ix++)
  {
    float p = 0;
    for (int k = 0; k < SPN; k++) p += crealf(conjf(a[(size_t)ix * SPN + k]) * b[(size_t)ix * SPN + k]);
    res += (double)p;
  }
  return res;
}

static void la_mul_add_assign_flt(int n, fcplx *s1, float r, const fcplx *s2)
{
  size_t m = (size_t)n * SPN;
#pragma omp parallel for
  for (size_t k = 0; k < m; k++) s1[k] += r * s2[k];
}

static void la_mul_flt(int n, fcplx *s1, float r, const fcplx *s2)
{
  size_t m = (size_t)n * SPN;
#pragma omp parallel for
  for (size_t k = 0; k < m; k++) s1[k] = r * s2[k];
}

/* ------------------------------------------------------------------------- */
/* Wilson operators: Dphi.c:703-1019                                          */
/* ------------------------------------------------------------------------- */
void orc_Dphi(double m0, cplx *out, const cplx *in)
{
  orc_Dphi_(out, ORC_FULL, in, ORC_FULL);
  orc_mul_add_assign(V_, out, 4. + m0, in);
}

void orc_g5Dphi(double m0, cplx *out, const cplx *in)
{
  orc_Dphi(m0, out, in);
  orc_g5(V_, out, out);
}

void orc_g5Dphi_sq(double m0, cplx *out, const cplx *in)
{
  cplx *g = malloc(sizeof(cplx) * V_ * SPN);
  orc_g5Dphi(m0, g, in);
  orc_g5Dphi(m0, out, g);
  free(g);
}

static void eopre_core(double m0, cplx *out, const cplx *in, int outpar, int g5)
{
  int other = outpar == ORC_EVEN ? ORC_ODD : ORC_EVEN;
  cplx *tmp = malloc(sizeof(cplx) * VH_ * SPN);
  orc_Dphi_(tmp, other, in, outpar);
  orc_Dphi_(out, outpar, tmp, other);
  double rho = 4.0 + m0;
  rho *= -rho;
  orc_mul_add_assign(VH_, out, rho, in);
  la_minus(VH_, out, out);
  if (g5) orc_g5(VH_, out, out);
  free(tmp);
}

void orc_Dphi_eopre(double m0, cplx *out, const cplx *in) { eopre_core(m0, out, in, ORC_EVEN, 0); }
void orc_Dphi_oepre(double m0, cplx *out, const cplx *in) { eopre_core(m0, out, in, ORC_ODD, 0); }
void orc_g5Dphi_eopre(double m0, cplx *out, const cplx *in) { eopre_core(m0, out, in, ORC_EVEN, 1); }

void orc_g5Dphi_eopre_sq(double m0, cplx *out, const cplx *in)
{
  cplx *e = malloc(sizeof(cplx) * VH_ * SPN);
  orc_g5Dphi_eopre(m0, e, in);
  orc_g5Dphi_eopre(m0, out, e);
  free(e);
}

/* float versions: Dphi_flt.c:366-593 (rho in float) */
static void g5_flt(int n, fcplx *s)
{
  for (int ix = 0; ix < n; ix++)
    for (int k = 2 * NF_; k < SPN; k++) s[(size_t)ix * SPN + k] = -s[(size_t)ix * SPN + k];
}

void orc_Dphi_flt(double m0, fcplx *out, const fcplx *in)
{
  orc_Dphi_flt_(out, ORC_FULL, in, ORC_FULL);
  float rho = 4.f + (float)m0;
  la_mul_add_assign_flt(V_, out, rho, in);
}

void orc_g5Dphi_flt(double m0, fcplx *out, const fcplx *in)
{
  orc_Dphi_flt(m0, out, in);
  g5_flt(V_, out);
}

void orc_g5Dphi_sq_flt(double m0, fcplx *out, const fcplx *in)
{
  fcplx *g = malloc(sizeof(fcplx) * V_ * SPN);
  orc_g5Dphi_flt(m0, g, in);
  orc_g5Dphi_flt(m0, out, g);
  free(g);
}

static void eopre_flt_core(double m0, fcplx *out, const fcplx *in, int g5)
{
  fcplx *tmp = malloc(sizeof(fcplx) * VH_ * SPN);
  orc_Dphi_flt_(tmp, ORC_ODD, in, ORC_EVEN);
  orc_Dphi_flt_(out, ORC_EVEN, tmp, ORC_ODD);
  float rho = 4.0f + (float)m0;
  rho *= -rho;
  la_mul_add_assign_flt(VH_, out, rho, in);
  size_t m = (size_t)VH_ * SPN;
  for (size_t k = 0; k < m; k++) out[k] = -out[k];
  if (g5) g5_flt(VH_, out);
  free(tmp);
}

void orc_Dphi_eopre_flt(double m0, fcplx *out, const fcplx *in) { eopre_flt_core(m0, out, in, 0); }
void orc_g5Dphi_eopre_flt(double m0, fcplx *out, const fcplx *in) { eopre_flt_core(m0, out, in, 1); }

void orc_g5Dphi_eopre_sq_flt(double m0, fcplx *out, const fcplx *in)
{
  fcplx *e = malloc(sizeof(fcplx) * VH_ * SPN);
  orc_g5Dphi_eopre_flt(m0, e, in);
  orc_g5Dphi_eopre_flt(m0, out, e);
  free(e);
}

/* ------------------------------------------------------------------------- */
/* clover term: LibHR/Update/clover_tools.c                                   */
/* ------------------------------------------------------------------------- */
#define LDLN (NF_ * (2 * NF_ + 1)) /* packed lower-triangular 2NF x 2NF        */
#define CPX(x, i, j) ((x)[(i) * ((i) + 1) / 2 + (j)])

static int expclover_ = 0; /* WITH_EXPCLOVER: diagonal (4+m) exp(A/(4+m)) */

void orc_clover_init(double csw)
{
  expclover_ = 0;
  free(cl_term_); free(cl_ldl_); free(cl_force_);
  cl_term_ = calloc((size_t)V_ * 4 * NF_ * NF_, sizeof(cplx));
  cl_ldl_ = calloc((size_t)V_ * 2 * LDLN, sizeof(cplx));
  cl_force_ = calloc((size_t)V_ * 6 * NF_ * NF_, sizeof(cplx));
  csw_ = csw;
  sigma_ = 0xF00F;
}

/* exponential clover (Dphi.c:1292-1482, LibHR/Utils/clover_exp.c): the same
 * clover term, the diagonal (4+m) exp(A/(4+m)) and its inverse exp(-A/(4+m))/(4+m) */
void orc_expclover_init(double csw)
{
  orc_clover_init(csw);
  expclover_ = 1;
}

/* block b (0: [[s0, s1], [s1^+, -s0]], 1: the same from s2, s3) of site ix, dense 2NF x 2NF */
static void clover_block(cplx *m, int ix, int b)
{
  const int F = NF_, F2 = NF_ * NF_, n = 2 * NF_;
  const cplx *sa = cl_term_ + ((size_t)ix * 4 + 2 * b) * F2, *sb = sa + F2;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
    {
      cplx v;
      if (i < F && j < F) v = sa[i * F + j];
      else if (i < F) v = sb[i * F + (j - F)];
      else if (j < F) v = conj(sb[j * F + (i - F)]);
      else v = -sa[(i - F) * F + (j - F)];
      m[i * n + j] = v;
    }
}

/* exp(x) of an n x n matrix by its Taylor series, summed until the terms' norm
 * is below 1e-28 (clover_exp_taylor, clover_exp.c:364-396) */
static void taylor_exp(int n, cplx *e, const cplx *x)
{
  cplx term[n * n], tmp[n * n];
  for (int k = 0; k < n * n; k++) e[k] = term[k] = (k % (n + 1) == 0) ? 1.0 : 0.0;
  for (int j = 1; j < 200; j++)
  {
    mat_mul(n, tmp, term, x);
    double nrm = 0;
    for (int k = 0; k < n * n; k++)
    {
      term[k] = tmp[k] / j;
      e[k] += term[k];
      nrm += creal(term[k] * conj(term[k]));
    }
    if (sqrt(nrm) < 1e-28) break;
  }
}

/* out = (4+m)^s exp(s A/(4+m)) in on the chiral halves, s = +1 (Cphi_) or -1 (inverse) */
static void expclover_apply(double mass, cplx *out, const cplx *in, int par, int assign, int inverse)
{
  const int F = NF_, n = 2 * NF_;
  const double sig = 4. + mass, c = (inverse ? -1.0 : 1.0) / sig, scale = inverse ? 1.0 / sig : sig;
  const int b0 = par_base(par);
#pragma omp parallel for
  for (int ix = b0; ix < par_end(par); ix++)
  {
    const cplx *s = in + (size_t)(ix - b0) * SPN;
    cplx tmp[4 * 64];
    for (int b = 0; b < 2; b++)
    {
      cplx m[n * n], e[n * n];
      clover_block(m, ix, b);
      for (int k = 0; k < n * n; k++) m[k] *= c;
      taylor_exp(n, e, m);
      for (int i = 0; i < n; i++)
      {
        cplx v = 0;
        for (int j = 0; j < n; j++) v += e[i * n + j] * s[2 * b * F + j];
        tmp[2 * b * F + i] = scale * v;
      }
    }
    cplx *o = out + (size_t)(ix - b0) * SPN;
    for (int k = 0; k < SPN; k++)
      if (assign) o[k] += tmp[k]; else o[k] = tmp[k];
  }
}

/* a generic represented link as complex (real reps promoted) */
static void get_link(cplx *m, int ix, int mu)
{
  int F = NF_;
  if (REAL_)
  {
    const double *u = (const double *)uf_ + (size_t)(4 * ix + mu) * F * F;
    for (int k = 0; k < F * F; k++) m[k] = u[k];
  }
  else
    memcpy(m, (const cplx *)uf_ + (size_t)(4 * ix + mu) * F * F, sizeof(cplx) * F * F);
}

static void mm(cplx *c, const cplx *a, const cplx *b) { mat_mul(NF_, c, a, b); }
static void mmd(cplx *c, const cplx *a, const cplx *b) /* c = a b^+ */
{
  int n = NF_;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
    {
      cplx s = 0;
      for (int k = 0; k < n; k++) s += a[i * n + k] * conj(b[j * n + k]);
      c[i * n + j] = s;
    }
}
static void mdm(cplx *c, const cplx *a, const cplx *b) /* c = a^+ b */
{
  int n = NF_;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
    {
      cplx s = 0;
      for (int k = 0; k < n; k++) s += conj(a[k * n + i]) * b[k * n + j];
      c[i * n + j] = s;
    }
}
static void dagger(cplx *c, const cplx *a)
{
  int n = NF_;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) c[i * n + j] = conj(a[j * n + i]);
}

/* clover_tools.c:59-95 (four-leaf loop) */
static void clover_loop(int id, int mu, int nu, cplx *u)
{
  int F2 = NF_ * NF_;
  cplx s1[F2], s2[F2], s3[F2], a[F2], b[F2];
  int o1, o2, o3;
  o1 = iup_[4 * id + mu]; o2 = iup_[4 * id + nu];
  get_link(a, id, mu); get_link(b, o1, nu); mm(s1, a, b);
  get_link(a, id, nu); get_link(b, o2, mu); mm(s2, a, b);
  mmd(u, s1, s2);
  o1 = idn_[4 * id + mu]; o2 = iup_[4 * o1 + nu];
  get_link(a, o1, nu); get_link(b, o2, mu); mm(s1, a, b);
  get_link(a, id, nu); mmd(s2, a, s1);
  get_link(a, o1, mu); mm(s3, s2, a);
  for (int k = 0; k < F2; k++) u[k] += s3[k];
  o1 = idn_[4 * id + mu]; o2 = idn_[4 * id + nu]; o3 = idn_[4 * o1 + nu];
  get_link(a, o3, nu); get_link(b, o1, mu); mm(s1, a, b);
  get_link(a, o3, mu); mdm(s2, s1, a);
  get_link(a, o2, nu); mm(s3, s2, a);
  for (int k = 0; k < F2; k++) u[k] += s3[k];
  o1 = idn_[4 * id + nu]; o2 = iup_[4 * o1 + mu];
  get_link(a, o1, nu); get_link(b, o1, mu); mdm(s1, a, b);
  get_link(a, o2, nu); get_link(b, id, mu); mmd(s2, a, b);
  mm(s3, s1, s2);
  for (int k = 0; k < F2; k++) u[k] += s3[k];
}

/* clover_tools.c:161-206 */
void orc_compute_clover_term(void)
{
  int F = NF_, F2 = NF_ * NF_;
  double csw = -csw_ / 16.0;
#pragma omp parallel for
  for (int id = 0; id < V_; id++)
  {
    cplx tmp[6][F2];
    clover_loop(id, 0, 1, tmp[0]);
    clover_loop(id, 0, 2, tmp[1]);
    clover_loop(id, 0, 3, tmp[2]);
    clover_loop(id, 1, 2, tmp[3]);
    clover_loop(id, 1, 3, tmp[4]);
    clover_loop(id, 2, 3, tmp[5]);
    cplx *cl = cl_term_ + (size_t)id * 4 * F2;
    for (int i = 0; i < F; i++)
      for (int j = 0; j < F; j++)
      {
        int ij = i * F + j, ji = j * F + i;
        cplx at, bt, ct, dt;
        if (REAL_)
        {
          /* real-representation loops: the tmp matrices are real */
          double t0ij = creal(tmp[0][ij]), t0ji = creal(tmp[0][ji]);
          double t1ij = creal(tmp[1][ij]), t1ji = creal(tmp[1][ji]);
          double t2ij = creal(tmp[2][ij]), t2ji = creal(tmp[2][ji]);
          double t3ij = creal(tmp[3][ij]), t3ji = creal(tmp[3][ji]);
          double t4ij = creal(tmp[4][ij]), t4ji = creal(tmp[4][ji]);
          double t5ij = creal(tmp[5][ij]), t5ji = creal(tmp[5][ji]);
          at = I * (t2ji - t2ij);
          bt = I * (t3ij - t3ji);
          ct = t1ji - t1ij + I * (t0ji - t0ij);
          dt = t4ij - t4ji + I * (t5ji - t5ij);
        }
        else
        {
          at = I * (conj(tmp[2][ji]) - tmp[2][ij]);
          bt = I * (conj(tmp[3][ij]) - tmp[3][ji]);
          ct = I * (conj(tmp[0][ji]) - tmp[0][ij]) - tmp[1][ij] + conj(tmp[1][ji]);
          dt = tmp[4][ij] - conj(tmp[4][ji]) + I * (conj(tmp[5][ji]) - tmp[5][ij]);
        }
        cl[0 * F2 + ij] = csw * (at - conj(bt));
        cl[1 * F2 + ij] = csw * (ct - dt);
        cl[2 * F2 + ij] = -csw * (at + conj(bt));
        cl[3 * F2 + ij] = -csw * (ct + dt);
      }
  }
  sigma_ = 0xF00F;
}

void orc_get_clover_term(cplx *cl) { memcpy(cl, cl_term_, sizeof(cplx) * V_ * 4 * NF_ * NF_); }
void orc_get_clover_ldl(cplx *l) { memcpy(l, cl_ldl_, sizeof(cplx) * V_ * 2 * LDLN); }

/* clover_tools.c:97-114 */
static void ldl(int N, cplx *A)
{
  for (int i = 0; i < N; i++)
  {
    for (int k = 0; k < i; k++) CPX(A, i, i) -= conj(CPX(A, i, k)) * CPX(A, i, k) * creal(CPX(A, k, k));
    for (int j = i + 1; j < N; j++)
    {
      for (int k = 0; k < i; k++) CPX(A, j, i) -= conj(CPX(A, i, k)) * CPX(A, j, k) * creal(CPX(A, k, k));
      CPX(A, j, i) /= creal(CPX(A, i, i));
    }
  }
}

/* clover_tools.c:116-159, :343-358 (recomputed only when sigma changes) */
void orc_compute_ldl_decomp(double sigma0)
{
  if (sigma_ == sigma0) return;
  sigma_ = sigma0;
  int F = NF_, F2 = NF_ * NF_;
#pragma omp parallel for
  for (int id = 0; id < V_; id++)
  {
    cplx *A = cl_ldl_ + (size_t)id * 2 * LDLN, *B = A + LDLN;
    const cplx *cl = cl_term_ + (size_t)id * 4 * F2;
    for (int i = 0; i < F; i++)
    {
      int m = i + F;
      for (int j = 0; j < F; j++)
      {
        int n = j + F, ij = i * F + j, ji = j * F + i;
        CPX(A, m, j) = conj(cl[1 * F2 + ji]);
        CPX(B, m, j) = conj(cl[3 * F2 + ji]);
        if (i >= j)
        {
          CPX(A, i, j) = cl[0 * F2 + ij];
          CPX(A, m, n) = -cl[0 * F2 + ij];
          CPX(B, i, j) = cl[2 * F2 + ij];
          CPX(B, m, n) = -cl[2 * F2 + ij];
          if (i == j)
          {
            CPX(A, i, j) += sigma_;
            CPX(A, m, n) += sigma_;
            CPX(B, i, j) += sigma_;
            CPX(B, m, n) += sigma_;
          }
        }
      }
    }
    ldl(2 * F, A);
    ldl(2 * F, B);
  }
}

/* Dphi.c:1091-1146 */
void orc_Cphi_(double mass, cplx *out, const cplx *in, int par, int assign)
{
  if (expclover_)
  {
    expclover_apply(mass, out, in, par, assign, 0);
    return;
  }
  int F = NF_, F2 = NF_ * NF_;
  mass = 4. + mass;
  int b = par_base(par);
#pragma omp parallel for
  for (int ix = b; ix < par_end(par); ix++)
  {
    const cplx *s = in + (size_t)(ix - b) * SPN;
    const cplx *cl = cl_term_ + (size_t)ix * 4 * F2;
    const cplx *s0 = cl, *s1 = cl + F2, *s2 = cl + 2 * F2, *s3 = cl + 3 * F2;
    cplx tmp[4 * 64];
    for (int i = 0; i < F; i++)
    {
      cplx v1 = 0, v2 = 0;
      for (int j = 0; j < F; j++) { v1 += s0[i * F + j] * s[j]; v2 += s1[i * F + j] * s[F + j]; }
      tmp[i] = v1 + v2;
      v1 = 0; v2 = 0;
      for (int j = 0; j < F; j++) { v1 += s[j] * conj(s1[j * F + i]); v2 += s0[i * F + j] * s[F + j]; }
      tmp[F + i] = v1 - v2;
      v1 = 0; v2 = 0;
      for (int j = 0; j < F; j++) { v1 += s2[i * F + j] * s[2 * F + j]; v2 += s3[i * F + j] * s[3 * F + j]; }
      tmp[2 * F + i] = v1 + v2;
      v1 = 0; v2 = 0;
      for (int j = 0; j < F; j++) { v1 += s[2 * F + j] * conj(s3[j * F + i]); v2 += s2[i * F + j] * s[3 * F + j]; }
      tmp[3 * F + i] = v1 - v2;
    }
    cplx *o = out + (size_t)(ix - b) * SPN;
    for (int k = 0; k < SPN; k++)
    {
      tmp[k] += mass * s[k];
      if (assign) o[k] += tmp[k]; else o[k] = tmp[k];
    }
  }
}

/* Dphi.c:1148-1213 (LDL forward/back substitution) */
void orc_Cphi_inv_(double mass, cplx *out, const cplx *in, int par, int assign)
{
  if (expclover_)
  {
    expclover_apply(mass, out, in, par, assign, 1);
    return;
  }
  int N = 2 * NF_;
  mass = 4. + mass;
  orc_compute_ldl_decomp(mass);
  int b = par_base(par);
#pragma omp parallel for
  for (int ix = b; ix < par_end(par); ix++)
  {
    const cplx *up = cl_ldl_ + (size_t)ix * 2 * LDLN, *dn = up + LDLN;
    cplx x[4 * 64];
    memcpy(x, in + (size_t)(ix - b) * SPN, sizeof(cplx) * SPN);
    for (int i = 0; i < N; i++)
      for (int k = 0; k < i; k++)
      {
        int n = i * (i + 1) / 2 + k;
        x[i] -= up[n] * x[k];
        x[i + N] -= dn[n] * x[k + N];
      }
    for (int i = N - 1; i >= 0; i--)
    {
      int n = i * (i + 1) / 2 + i;
      x[i] = (1. / creal(up[n])) * x[i];
      x[i + N] = (1. / creal(dn[n])) * x[i + N];
      for (int k = i + 1; k < N; k++)
      {
        n = k * (k + 1) / 2 + i;
        x[i] -= conj(up[n]) * x[k];
        x[i + N] -= conj(dn[n]) * x[k + N];
      }
    }
    cplx *o = out + (size_t)(ix - b) * SPN;
    for (int k = 0; k < SPN; k++)
      if (assign) o[k] += x[k]; else o[k] = x[k];
  }
}

/* Dphi.c:1215-1290 */
void orc_Cphi(double mass, cplx *out, const cplx *in)
{
  orc_Dphi_(out, ORC_FULL, in, ORC_FULL);
  orc_Cphi_(mass, out, in, ORC_FULL, 1);
}

void orc_g5Cphi(double mass, cplx *out, const cplx *in)
{
  orc_Cphi(mass, out, in);
  orc_g5(V_, out, out);
}

void orc_g5Cphi_sq(double mass, cplx *out, const cplx *in)
{
  cplx *g = malloc(sizeof(cplx) * V_ * SPN);
  orc_g5Cphi(mass, g, in);
  orc_g5Cphi(mass, out, g);
  free(g);
}

void orc_Cphi_eopre(double mass, cplx *out, const cplx *in)
{
  cplx *otmp = malloc(sizeof(cplx) * VH_ * SPN);
  orc_Dphi_(otmp, ORC_ODD, in, ORC_EVEN);
  orc_Cphi_inv_(mass, otmp, otmp, ORC_ODD, 0);
  orc_Dphi_(out, ORC_EVEN, otmp, ORC_ODD);
  la_minus(VH_, out, out);
  orc_Cphi_(mass, out, in, ORC_EVEN, 1);
  free(otmp);
}

void orc_g5Cphi_eopre(double mass, cplx *out, const cplx *in)
{
  orc_Cphi_eopre(mass, out, in);
  orc_g5(VH_, out, out);
}

void orc_g5Cphi_eopre_sq(double mass, cplx *out, const cplx *in)
{
  cplx *e = malloc(sizeof(cplx) * VH_ * SPN);
  orc_g5Cphi_eopre(mass, e, in);
  orc_g5Cphi_eopre(mass, out, e);
  free(e);
}

void orc_Cphi_diag(double mass, cplx *out, const cplx *in, int par) { orc_Cphi_(mass, out, in, par, 0); }
void orc_Cphi_diag_inv(double mass, cplx *out, const cplx *in, int par) { orc_Cphi_inv_(mass, out, in, par, 0); }

/* ------------------------------------------------------------------------- */
/* multi-shift CG: LibHR/Inverters/cg_mshift.c:24-195                         */
/* ------------------------------------------------------------------------- */
static int op_sites(int op)
{
  return (op == ORC_OP_G5DPHI_SQ || op == ORC_OP_G5CPHI_SQ || op == ORC_OP_DPHI || op == ORC_OP_CPHI) ? V_ : VH_;
}

static void apply_op(int op, cplx *out, const cplx *in)
{
  switch (op)
  {
  case ORC_OP_G5DPHI_SQ: orc_g5Dphi_sq(static_mass_, out, in); break;
  case ORC_OP_G5DPHI_EOPRE_SQ: orc_g5Dphi_eopre_sq(static_mass_, out, in); break;
  case ORC_OP_G5CPHI_EOPRE_SQ: orc_g5Cphi_eopre_sq(static_mass_, out, in); break;
  case ORC_OP_G5CPHI_SQ: orc_g5Cphi_sq(static_mass_, out, in); break;
  case ORC_OP_DPHI_EOPRE: orc_Dphi_eopre(static_mass_, out, in); break;
  case ORC_OP_G5DPHI_EOPRE: orc_g5Dphi_eopre(static_mass_, out, in); break;
  case ORC_OP_CPHI_EOPRE: orc_Cphi_eopre(static_mass_, out, in); break;
  case ORC_OP_G5CPHI_EOPRE: orc_g5Cphi_eopre(static_mass_, out, in); break;
  case ORC_OP_DPHI: orc_Dphi(static_mass_, out, in); break;
  case ORC_OP_CPHI: orc_Cphi(static_mass_, out, in); break;
  }
}

static int cg_mshift_core(short *sflags, int op, int n, const double *shift, double err2, int max_iter,
                          const cplx *in, cplx *out)
{
  int ns = op_sites(op);
  size_t fsz = (size_t)ns * SPN;
  cplx *p = malloc(sizeof(cplx) * fsz * (n + 3));
  cplx *k = p + fsz * n, *r = k + fsz, *Mk = r + fsz;
  double *z1 = malloc(sizeof(double) * n), *z2 = malloc(sizeof(double) * n), *z3 = malloc(sizeof(double) * n);
  int cgiter = 0;
  double omega = 1., oldomega, gamma = 0., alpha, lambda, delta;
  double innorm2 = orc_sqnorm(ns, in);
  if (n == 1)
  {
    apply_op(op, Mk, out);
    ++cgiter;
    orc_mul_add_assign(ns, Mk, -shift[0], out);
    la_sub(ns, r, in, Mk);
  }
  else
    memcpy(r, in, sizeof(cplx) * fsz);
  memcpy(k, r, sizeof(cplx) * fsz);
  delta = orc_sqnorm(ns, r);
  for (int i = 0; i < n; i++)
  {
    z1[i] = z2[i] = 1.;
    memcpy(p + fsz * i, r, sizeof(cplx) * fsz);
    if (n != 1) memset(out + fsz * i, 0, sizeof(cplx) * fsz);
    sflags[i] = 1;
  }
  unsigned short notconverged;
  do
  {
    apply_op(op, Mk, k);
    alpha = orc_prod_re(ns, k, Mk);
    oldomega = omega;
    omega = -delta / alpha;
    for (int i = 0; i < n; i++)
      if (sflags[i])
      {
        z3[i] = oldomega * z1[i] * z2[i] / (omega * gamma * (z1[i] - z2[i]) + z1[i] * oldomega * (1. + shift[i] * omega));
        orc_mul_add_assign(ns, out + fsz * i, -omega * z3[i] / z2[i], p + fsz * i);
      }
    orc_mul_add_assign(ns, r, omega, Mk);
    lambda = orc_sqnorm(ns, r);
    gamma = lambda / delta;
    delta = lambda;
    la_mul(ns, k, gamma, k);
    la_add_assign(ns, k, r);
    notconverged = 0;
    for (int i = 0; i < n; i++)
    {
      if (delta * z3[i] * z3[i] < err2 * innorm2) sflags[i] = 0;
      if (sflags[i])
      {
        notconverged++;
        la_mul(ns, p + fsz * i, gamma * z3[i] * z3[i] / (z2[i] * z2[i]), p + fsz * i);
        orc_mul_add_assign(ns, p + fsz * i, z3[i], r);
        z1[i] = z2[i];
        z2[i] = z3[i];
      }
    }
    ++cgiter;
  } while ((max_iter == 0 || cgiter < max_iter) && notconverged);
  for (int i = 0; i < n; i++)
  {
    apply_op(op, Mk, out + fsz * i);
    ++cgiter;
    orc_mul_add_assign(ns, Mk, -shift[i], out + fsz * i);
    la_sub(ns, Mk, Mk, in);
    double norm = orc_sqnorm(ns, Mk) / orc_sqnorm(ns, in);
    sflags[i] = (fabs(norm) > err2) ? 0 : 1;
  }
  free(p); free(z1); free(z2); free(z3);
  return cgiter;
}

int orc_cg_mshift(int op, int n, const double *shift, double err2, int max_iter, const cplx *in, cplx *out)
{
  short sflags[n > 0 ? n : 1];
  size_t fsz = (size_t)op_sites(op) * SPN;
  int cgiter = cg_mshift_core(sflags, op, n, shift, err2, max_iter, in, out);
  for (int i = 0; i < n; i++)
  {
    int rep = 0;
    while (sflags[i] == 0 && rep < 100)
    {
      cgiter += cg_mshift_core(sflags + i, op, 1, shift + i, err2, max_iter, in, out + fsz * i);
      rep++;
    }
  }
  return cgiter;
}

/* ------------------------------------------------------------------------- */
/* mixed precision: LibHR/Inverters/cg_mshift_flt.c:22-276                    */
/* inner FP32 multishift CG (relative target clamped at 1e-10), outer FP64    */
/* defect correction.  Only the Wilson operators have float versions in the   */
/* reference (Dphi_flt.c); the FP32 operator is the float twin of `op`.       */
/* ------------------------------------------------------------------------- */
static void apply_op_flt(int op, fcplx *out, const fcplx *in)
{
  switch (op)
  {
  case ORC_OP_G5DPHI_SQ: orc_g5Dphi_sq_flt(static_mass_, out, in); break;
  default: orc_g5Dphi_eopre_sq_flt(static_mass_, out, in); break;
  }
}

static int cg_mshift_flt_core(const short *sflags, int op, int n, const double *shift, double err2, int max_iter,
                              const fcplx *in, fcplx *out)
{
  int ns = op_sites(op);
  size_t fsz = (size_t)ns * SPN;
  fcplx *p = malloc(sizeof(fcplx) * fsz * (n + 3));
  fcplx *k = p + fsz * n, *r = k + fsz, *Mk = r + fsz;
  double *z1 = malloc(sizeof(double) * n), *z2 = malloc(sizeof(double) * n), *z3 = malloc(sizeof(double) * n);
  int cgiter = 0;
  double omega = 1., oldomega, gamma = 0., alpha, lambda, delta;
  double innorm2 = la_sqnorm_flt(ns, in);
  if (n == 1)
  {
    apply_op_flt(op, Mk, out);
    ++cgiter;
    la_mul_add_assign_flt(ns, Mk, (float)(-shift[0]), out);
    for (size_t q = 0; q < fsz; q++) r[q] = in[q] - Mk[q];
  }
  else
    memcpy(r, in, sizeof(fcplx) * fsz);
  memcpy(k, r, sizeof(fcplx) * fsz);
  delta = la_sqnorm_flt(ns, r);
  for (int i = 0; i < n; i++)
  {
    z1[i] = z2[i] = 1.;
    z3[i] = 0.;
    memcpy(p + fsz * i, r, sizeof(fcplx) * fsz);
    if (n != 1) memset(out + fsz * i, 0, sizeof(fcplx) * fsz);
  }
  int notconverged;
  do
  {
    apply_op_flt(op, Mk, k);
    alpha = la_prod_re_flt(ns, k, Mk);
    oldomega = omega;
    omega = -delta / alpha;
    for (int i = 0; i < n; i++)
      if (sflags[i])
      {
        z3[i] = oldomega * z1[i] * z2[i] / (omega * gamma * (z1[i] - z2[i]) + z1[i] * oldomega * (1. + shift[i] * omega));
        la_mul_add_assign_flt(ns, out + fsz * i, (float)(-omega * z3[i] / z2[i]), p + fsz * i);
      }
    la_mul_add_assign_flt(ns, r, (float)omega, Mk);
    lambda = la_sqnorm_flt(ns, r);
    gamma = lambda / delta;
    delta = lambda;
    la_mul_flt(ns, k, (float)gamma, k);
    for (size_t q = 0; q < fsz; q++) k[q] += r[q];
    notconverged = 0;
    for (int i = 0; i < n; i++)
    {
      if (delta * z3[i] * z3[i] > err2 * innorm2) ++notconverged;
      if (sflags[i])
      {
        la_mul_flt(ns, p + fsz * i, (float)(gamma * z3[i] * z3[i] / (z2[i] * z2[i])), p + fsz * i);
        la_mul_add_assign_flt(ns, p + fsz * i, (float)z3[i], r);
        z1[i] = z2[i];
        z2[i] = z3[i];
      }
    }
    ++cgiter;
  } while ((max_iter == 0 || cgiter < max_iter) && notconverged != 0);
  free(p); free(z1); free(z2); free(z3);
  return cgiter;
}

int orc_cg_mshift_flt(int op, int n, const double *shift, double err2, int max_iter, const cplx *in, cplx *out)
{
  if (op == ORC_OP_G5CPHI_EOPRE_SQ || op == ORC_OP_G5CPHI_SQ) return -1; /* no float clover in the reference */
  int ns = op_sites(op);
  size_t fsz = (size_t)ns * SPN;
  int siter = 0, diter = 0;
  short sflags[n], loc_flags[n];
  double norm[n];
  fcplx *res_flt = malloc(sizeof(fcplx) * fsz * (1 + n)), *out_flt = res_flt + fsz;
  cplx *res = malloc(sizeof(cplx) * fsz * 3), *res2 = res + fsz, *tmp = res2 + fsz;
  double local_err2 = err2;
  for (int i = 0; i < n; i++)
  {
    sflags[i] = 1;
    if (n != 1) memset(out + fsz * i, 0, sizeof(cplx) * fsz);
  }
  double innorm2 = orc_sqnorm(ns, in);
  int notconverged, guard = 0;
  do
  {
    int first = 1;
    notconverged = 0;
    for (int i = 0; i < n; i++)
    {
      if (sflags[i] == 0) continue;
      apply_op(op, tmp, out + fsz * i);
      ++diter;
      la_sub(ns, res2, in, tmp);
      orc_mul_add_assign(ns, res2, shift[i], out + fsz * i);
      norm[i] = orc_sqnorm(ns, res2);
      if (norm[i] < innorm2 * err2)
      {
        sflags[i] = 0;
        norm[i] /= innorm2;
      }
      else
      {
        ++notconverged;
        if (first)
        {
          first = 0;
          local_err2 = norm[i] / innorm2;
          norm[i] = sqrt(norm[i]);
          la_mul(ns, res, 1. / norm[i], res2);
        }
        else
          norm[i] = orc_prod_re(ns, res, res2);
      }
    }
    if (notconverged)
    {
      for (size_t q = 0; q < fsz; q++) res_flt[q] = (fcplx)res[q];
      local_err2 = err2 / local_err2 * 0.9;
      if (local_err2 < 1.e-10) local_err2 = 1.e-10;
      for (int i = 0; i < n; i++) loc_flags[i] = sflags[i];
      siter += cg_mshift_flt_core(loc_flags, op, n, shift, local_err2, max_iter, res_flt, out_flt);
      for (int i = 0; i < n; i++)
        if (sflags[i] != 0)
        {
          for (size_t q = 0; q < fsz; q++) res2[q] = (cplx)out_flt[fsz * i + q];
          orc_mul_add_assign(ns, out + fsz * i, norm[i], res2);
        }
    }
  } while (notconverged && ++guard < 1000);
  free(res_flt);
  free(res);
  return siter + diter;
}

/* ------------------------------------------------------------------------- */
/* g5QMR for gamma_5-hermitian operators: LibHR/Inverters/g5QMR_mshift.c      */
/* ------------------------------------------------------------------------- */
static double g5_prod_re_n(int ns, const cplx *a, const cplx *b) { return orc_g5_prod_re(ns, a, b); }

/* plane rotation (c, s) with [c s; -s c] (a, b)^T = (1/r, 0)^T   (g5QMR_mshift.c:30-37) */
static void givens(double *r, double *c, double *s, double a, double b)
{
  if (fabs(a) < 1.e-15)
  {
    *r = 1. / b;
    *c = 0.;
    *s = 1.;
  }
  else
  {
    double t = b / a;
    *c = 1. / sqrt(1. + t * t);
    *s = t * (*c);
    *r = 1. / ((*c) * a + (*s) * b);
  }
}

/* g5QMR_mshift_core (g5QMR_mshift.c:83-279): valid[i] = 1 if |M x_i - shift_i x_i - in|^2 <= err2 |in|^2.
 * Returns the MVM count, or -1 when the gamma_5 norm of the start vector vanishes (HiRep stops there). */
static int g5qmr_core(short *valid, int op, int n, const double *shift, double err2, int max_iter, const cplx *in,
                      cplx *out)
{
  const int ns = op_sites(op);
  const size_t fsz = (size_t)ns * SPN;
  cplx *pool = calloc(fsz * (2 * n + 3), sizeof(cplx));
  cplx **q1 = malloc(sizeof(cplx *) * n), **q2 = malloc(sizeof(cplx *) * n);
  for (int i = 0; i < n; i++)
  {
    q1[i] = pool + fsz * i;
    q2[i] = pool + fsz * (n + i);
  }
  cplx *p1 = pool + fsz * 2 * n, *p2 = p1 + fsz, *Mp = p2 + fsz, *tmp;
  double *r = malloc(sizeof(double) * 5 * n), *s1 = r + n, *s2 = s1 + n, *c1 = s2 + n, *c2 = c1 + n;
  short *flags = malloc(sizeof(short) * n);
  int cgiter = 0, notconverged = n;
  memcpy(p2, in, sizeof(cplx) * fsz);
  const double innorm2 = orc_sqnorm(ns, in);
  if (n == 1) /* out[0] is the start vector */
  {
    apply_op(op, Mp, out);
    orc_mul_add_assign(ns, Mp, -shift[0], out);
    la_sub(ns, p2, p2, Mp);
  }
  double rho = sqrt(orc_sqnorm(ns, p2));
  la_mul(ns, p2, 1. / rho, p2);
  memset(p1, 0, sizeof(cplx) * fsz);
  for (int i = 0; i < n; i++)
  {
    r[i] = rho;
    c2[i] = c1[i] = 1.;
    s1[i] = s2[i] = 0.;
    if (n != 1) memset(out + fsz * i, 0, sizeof(cplx) * fsz);
    flags[i] = 1;
  }
  double delta = g5_prod_re_n(ns, p2, p2);
  if (fabs(delta) < 1.e-28)
  {
    free(pool); free(q1); free(q2); free(r); free(flags);
    return -1;
  }
  double beta = delta;
  do
  {
    ++cgiter;
    apply_op(op, Mp, p2);
    orc_mul_add_assign(ns, Mp, -shift[0], p2);
    const double alpha = g5_prod_re_n(ns, p2, Mp) / delta;
    orc_mul_add_assign(ns, Mp, -beta, p1);
    orc_mul_add_assign(ns, Mp, -alpha, p2);
    tmp = p1; p1 = p2; p2 = Mp; Mp = tmp;
    rho = sqrt(orc_sqnorm(ns, p2));
    double maxm = 1.e-10;
    for (int i = 0; i < n; i++)
    {
      if (!flags[i]) continue;
      const double a = alpha - shift[i] + shift[0];
      const double t = s1[i] * beta;
      const double e = c2[i] * c1[i] * beta + s2[i] * a;
      const double m = c2[i] * a - s2[i] * c1[i] * beta;
      double d;
      s1[i] = s2[i];
      c1[i] = c2[i];
      givens(&d, &c2[i], &s2[i], m, rho);
      if (fabs(m) > maxm) maxm = fabs(m);
      /* new direction q = d (p1 - t q1 - e q2), then the rotation q1 <- q2 <- q */
      for (size_t k = 0; k < fsz; k++) Mp[k] = -t * d * q1[i][k] - e * d * q2[i][k];
      orc_mul_add_assign(ns, Mp, d, p1);
      tmp = q1[i]; q1[i] = q2[i]; q2[i] = Mp; Mp = tmp;
      orc_mul_add_assign(ns, out + fsz * i, c2[i] * r[i], q2[i]);
      r[i] *= -s2[i];
      if (fabs(r[i] * r[i]) * (double)(1 + cgiter) < err2 * innorm2)
      {
        flags[i] = 0;
        --notconverged;
      }
    }
    if (fabs(rho) > 1.e-13)
    {
      la_mul(ns, p2, 1. / rho, p2);
      const double olddelta = delta;
      delta = g5_prod_re_n(ns, p2, p2);
      if (fabs(delta) < 1.e-6 || maxm < 1.e-3) notconverged = 0; /* the method has failed */
      beta = rho * delta / olddelta;
    }
    else
      notconverged = 0; /* converged */
  } while ((max_iter == 0 || cgiter < max_iter) && notconverged);
  for (int i = 0; i < n; i++)
  {
    apply_op(op, Mp, out + fsz * i);
    ++cgiter;
    if (shift[i] != 0.) orc_mul_add_assign(ns, Mp, -shift[i], out + fsz * i);
    la_sub(ns, Mp, Mp, in);
    valid[i] = (fabs(orc_sqnorm(ns, Mp) / innorm2) > err2) ? 0 : 1;
  }
  if (n == 1) ++cgiter;
  free(pool); free(q1); free(q2); free(r); free(flags);
  return cgiter;
}

/* MINRES for a hermitian operator (LibHR/Inverters/MINRES.c:24-158).  The operator
 * is g5 (M - sh) with M = op, the form g5QMR_mshift falls back to (g5QMR_mshift.c:466-474). */
static int herm_op_, herm_g5_;
static double herm_sh_;
static void herm_apply(cplx *out, const cplx *in)
{
  const int ns = op_sites(herm_op_);
  apply_op(herm_op_, out, in);
  if (herm_sh_ != 0.) orc_mul_add_assign(ns, out, -herm_sh_, in);
  if (herm_g5_) orc_g5(ns, out, out);
}

static int minres_core(short *valid, double err2, int max_iter, const cplx *in, cplx *out, const cplx *trial)
{
  const int ns = op_sites(herm_op_);
  const size_t fsz = (size_t)ns * SPN;
  cplx *pool = calloc(fsz * 5, sizeof(cplx));
  cplx *q1 = pool, *q2 = q1 + fsz, *p1 = q2 + fsz, *p2 = p1 + fsz, *Mp = p2 + fsz, *tmp;
  int cgiter = 0, notconverged = 1;
  memcpy(p2, in, sizeof(cplx) * fsz);
  if (trial)
  {
    herm_apply(p1, trial);
    ++cgiter;
    for (size_t k = 0; k < fsz; k++) p2[k] -= p1[k];
    if (out != trial) memcpy(out, trial, sizeof(cplx) * fsz);
  }
  else
    memset(out, 0, sizeof(cplx) * fsz);
  const double innorm2 = orc_sqnorm(ns, in);
  double beta = sqrt(orc_sqnorm(ns, p2));
  la_mul(ns, p2, 1. / beta, p2);
  memset(p1, 0, sizeof(cplx) * fsz);
  double r = beta, rho2 = beta, rho1 = 1., c2 = -1., rp = 0., s1 = 0., s2 = 0., c1 = 0.;
  do
  {
    ++cgiter;
    herm_apply(Mp, p2);
    const double alpha = orc_prod_re(ns, Mp, p2);
    orc_mul_add_assign(ns, Mp, -beta, p1);
    orc_mul_add_assign(ns, Mp, -alpha, p2);
    tmp = p1; p1 = p2; p2 = Mp; Mp = tmp;
    const double oldbeta = beta;
    beta = sqrt(orc_sqnorm(ns, p2));
    la_mul(ns, p2, 1. / beta, p2);
    const double d = (alpha - rp * c1) * s2;
    const double h = oldbeta * s1;
    rp = -oldbeta * c1 * s2 - alpha * c2;
    const double k = sqrt(rp * rp + beta * beta);
    c1 = c2;
    c2 = rp / k;
    s1 = s2;
    s2 = beta / k;
    for (size_t q = 0; q < fsz; q++) Mp[q] = -h / rho1 * q1[q] - d / rho2 * q2[q];
    tmp = q1; q1 = q2; q2 = tmp;
    for (size_t q = 0; q < fsz; q++) q2[q] = p1[q] + Mp[q];
    rho1 = rho2;
    rho2 = k;
    orc_mul_add_assign(ns, out, r * c2 / k, q2);
    r *= s2;
    if (r * r < err2 * innorm2) notconverged = 0;
  } while ((max_iter == 0 || cgiter < max_iter) && notconverged);
  herm_apply(Mp, out);
  ++cgiter;
  la_sub(ns, Mp, Mp, in);
  *valid = (fabs(orc_sqnorm(ns, Mp) / innorm2) > err2) ? 0 : 1;
  free(pool);
  return cgiter;
}

/* MINRES (MINRES.c:160-172): repeated from the last solution until valid (bounded here) */
int orc_MINRES(int op, int g5, double sh, double err2, int max_iter, const cplx *in, cplx *out, const cplx *trial)
{
  herm_op_ = op;
  herm_g5_ = g5;
  herm_sh_ = sh;
  short valid;
  int iter = minres_core(&valid, err2, max_iter, in, out, trial), rep = 0;
  while (!valid && (max_iter == 0 || iter < max_iter) && ++rep < 100) iter += minres_core(&valid, err2, max_iter, in, out, out);
  return iter;
}

/* g5QMR_mshift (g5QMR_mshift.c:481-542): unconverged shifts are solved again one at a
 * time from their current solution, then with MINRES on g5 (M - shift). */
int orc_g5QMR_mshift(int op, int n, const double *shift, double err2, int max_iter, const cplx *in, cplx *out)
{
  const int ns = op_sites(op);
  const size_t fsz = (size_t)ns * SPN;
  short valid[n > 0 ? n : 1];
  int cgiter = g5qmr_core(valid, op, n, shift, err2, max_iter, in, out);
  if (cgiter < 0) return -1;
  for (int i = 0; i < n; i++)
  {
    if (valid[i]) continue;
    int it = g5qmr_core(valid + i, op, 1, shift + i, err2, 0, in, out + fsz * i);
    if (it < 0) return -1;
    cgiter += it;
    if (!valid[i])
    {
      cplx *g5in = malloc(sizeof(cplx) * fsz);
      orc_g5(ns, g5in, in);
      cgiter += orc_MINRES(op, 1, shift[i], err2, 0, g5in, out + fsz * i, out + fsz * (i == 0 ? 0 : i - 1));
      free(g5in);
    }
  }
  return cgiter;
}

/* ------------------------------------------------------------------------- */
/* chronological initial guess (MRE): LibHR/Update/mre.c                      */
/* ------------------------------------------------------------------------- */
/* in-place LU with partial pivoting of A (max x max, row-major) and solution of
 * A x = conj(b) (mre.c:56-143) */
static int mre_lu_solve(int max, cplx *A, const cplx *b, cplx *x)
{
  int mutate[64];
  cplx y[64];
  for (int i = 0; i < max; i++) mutate[i] = i;
  for (int i = 0; i < max; i++)
  {
    for (int j = 0; j <= i; j++)
      for (int k = 0; k < j; k++) A[j * max + i] -= A[j * max + k] * A[k * max + i];
    double big = cabs(A[i * max + i]);
    int row = i;
    for (int j = i + 1; j < max; j++)
    {
      for (int k = 0; k < i; k++) A[j * max + i] -= A[j * max + k] * A[k * max + i];
      if (cabs(A[j * max + i]) > big)
      {
        big = cabs(A[j * max + i]);
        row = j;
      }
    }
    if (big < 1.0e-14) return -1; /* singular: HiRep keeps the previous x */
    if (row != i)
    {
      for (int k = 0; k < max; k++)
      {
        cplx t = A[row * max + k];
        A[row * max + k] = A[i * max + k];
        A[i * max + k] = t;
      }
      int t = mutate[row];
      mutate[row] = mutate[i];
      mutate[i] = t;
    }
    for (int k = i + 1; k < max; k++) A[k * max + i] = A[k * max + i] / A[i * max + i];
  }
  for (int i = 0; i < max; i++)
  {
    y[i] = conj(b[mutate[i]]);
    for (int k = 0; k < i; k++) y[i] -= A[i * max + k] * y[k];
  }
  for (int i = max - 1; i >= 0; i--)
  {
    x[i] = y[i];
    for (int k = i + 1; k < max; k++) x[i] -= A[i * max + k] * x[k];
    x[i] = x[i] / A[i * max + i];
  }
  return 0;
}

/* mre_guess (mre.c:230-268): s holds the `max` most recent solutions (newest
 * first); out = sum_i x_i v_i over their Gram-Schmidt basis v_i, with
 * A[j][i] = <DD v_i, v_j>, b_i = <v_i, pf> */
void orc_mre_guess(int op, int max, const cplx *s, cplx *out, const cplx *pf)
{
  const int ns = op_sites(op);
  const size_t fsz = (size_t)ns * SPN;
  memset(out, 0, sizeof(cplx) * fsz);
  if (max <= 0) return;
  cplx *v = malloc(sizeof(cplx) * fsz * (max + 1)), *Dv = v + fsz * max;
  memcpy(v, s, sizeof(cplx) * fsz * max);
  for (int i = 0; i < max; i++) /* gram_schmidt (mre.c:30-48) */
  {
    cplx *vi = v + fsz * i;
    la_mul(ns, vi, 1.0 / sqrt(orc_sqnorm(ns, vi)), vi);
    for (int j = i + 1; j < max; j++)
    {
      cplx *vj = v + fsz * j;
      cplx rij = orc_prod_re(ns, vi, vj) + I * orc_prod_im(ns, vi, vj);
      for (size_t q = 0; q < fsz; q++) vj[q] -= rij * vi[q];
    }
  }
  cplx A[64 * 64], b[64], x[64];
  for (int i = 0; i < max; i++)
  {
    apply_op(op, Dv, v + fsz * i);
    for (int j = 0; j < max; j++) A[j * max + i] = orc_prod_re(ns, Dv, v + fsz * j) + I * orc_prod_im(ns, Dv, v + fsz * j);
    b[i] = orc_prod_re(ns, v + fsz * i, pf) + I * orc_prod_im(ns, v + fsz * i, pf);
  }
  if (mre_lu_solve(max, A, b, x) == 0)
    for (int i = 0; i < max; i++)
      for (size_t q = 0; q < fsz; q++) out[q] += x[i] * v[fsz * i + q];
  free(v);
}

/* ------------------------------------------------------------------------- */
/* pseudofermion force: LibHR/Update/force_fermion_core.c                     */
/* ------------------------------------------------------------------------- */
void orc_fermion_force_begin(void)
{
  free(force_sum_);
  force_sum_ = calloc((size_t)V_ * 4 * DIMG_, sizeof(double));
  if (cl_force_) memset(cl_force_, 0, sizeof(cplx) * V_ * 6 * NF_ * NF_);
}

/* _suNf_FMAT accumulation (write_suN_headers.pl:3001-3090):
 * s1 += p0 (x) p2^+ + p1 (x) p3^+, real part only for real representations */
static void fmat(cplx *s1, const cplx *p0, const cplx *p1, const cplx *p2, const cplx *p3)
{
  int F = NF_;
  for (int i = 0; i < F; i++)
    for (int j = 0; j < F; j++)
    {
      cplx v = p0[i] * conj(p2[j]) + p1[i] * conj(p3[j]);
      if (REAL_) s1[i * F + j] += creal(p0[i] * conj(p2[j])) + creal(p1[i] * conj(p3[j]));
      else s1[i * F + j] += v;
    }
}

/* _F_DIR0.._F_DIR3 (force_fermion_core.c:72-114) */
static void f_dir(cplx *s1, int ix, int mu, const cplx *c1, const cplx *c2)
{
  int F = NF_;
  cplx pt[64], pt2[64], p0[64], p1[64], p2[64], p3[64];
  const cplx *a0 = c2, *a1 = c2 + F, *a2 = c2 + 2 * F, *a3 = c2 + 3 * F;
  const cplx *b0 = c1, *b1 = c1 + F, *b2 = c1 + 2 * F, *b3 = c1 + 3 * F;
  for (int i = 0; i < F; i++)
  {
    switch (mu)
    {
    case 0:
      pt[i] = a0[i] + a2[i]; pt2[i] = a1[i] + a3[i];
      p2[i] = b0[i] - b2[i]; p3[i] = b1[i] - b3[i];
      break;
    case 1:
      pt[i] = a0[i] + I * a3[i]; pt2[i] = a1[i] + I * a2[i];
      p2[i] = b0[i] - I * b3[i]; p3[i] = b1[i] - I * b2[i];
      break;
    case 2:
      pt[i] = a0[i] + a3[i]; pt2[i] = a1[i] - a2[i];
      p2[i] = b0[i] - b3[i]; p3[i] = b1[i] + b2[i];
      break;
    default:
      pt[i] = a0[i] + I * a2[i]; pt2[i] = a1[i] - I * a3[i];
      p2[i] = b0[i] - I * b2[i]; p3[i] = b1[i] + I * b3[i];
      break;
    }
  }
  link_mul(p0, ix, mu, pt);
  link_mul(p1, ix, mu, pt2);
  fmat(s1, p0, p1, p2, p3);
}

/* g5_sigma (force_fermion_core.c:123-250): s = g5 sigma_{mu nu} u */
static void g5_sigma(cplx *s, const cplx *u, int mu, int nu)
{
  int F = NF_;
  int src[4];
  cplx f[4];
  int a = mu < nu ? mu : nu, b = mu < nu ? nu : mu;
  double sg = (mu < nu) ? 1.0 : -1.0;
  if (a == 0 && b == 1) { int s_[4] = {1, 0, 3, 2}; cplx f_[4] = {-I, -I, -I, -I}; memcpy(src, s_, sizeof src); memcpy(f, f_, sizeof f); }
  else if (a == 0 && b == 2) { int s_[4] = {1, 0, 3, 2}; cplx f_[4] = {-1, 1, -1, 1}; memcpy(src, s_, sizeof src); memcpy(f, f_, sizeof f); }
  else if (a == 0 && b == 3) { int s_[4] = {0, 1, 2, 3}; cplx f_[4] = {-I, I, -I, I}; memcpy(src, s_, sizeof src); memcpy(f, f_, sizeof f); }
  else if (a == 1 && b == 2) { int s_[4] = {0, 1, 2, 3}; cplx f_[4] = {I, -I, -I, I}; memcpy(src, s_, sizeof src); memcpy(f, f_, sizeof f); }
  else if (a == 1 && b == 3) { int s_[4] = {1, 0, 3, 2}; cplx f_[4] = {-1, 1, 1, -1}; memcpy(src, s_, sizeof src); memcpy(f, f_, sizeof f); }
  else { int s_[4] = {1, 0, 3, 2}; cplx f_[4] = {I, I, -I, -I}; memcpy(src, s_, sizeof src); memcpy(f, f_, sizeof f); }
  for (int c = 0; c < 4; c++)
    for (int i = 0; i < F; i++) s[c * F + i] = sg * f[c] * u[src[c] * F + i];
}

/* fmat_create (force_fermion_core.c:252-280) */
static void fmat_create(cplx *fm, const cplx *al, const cplx *ar, const cplx *bl, const cplx *br)
{
  int F = NF_;
  for (int i = 0; i < F; i++)
    for (int j = 0; j < F; j++)
    {
      cplx s = 0;
      for (int k = 0; k < 4; k++)
        s += al[k * F + i] * conj(ar[k * F + j]) + bl[k * F + i] * conj(br[k * F + j]);
      fm[i * F + j] = REAL_ ? creal(s) : s;
    }
}

/* force_clover_fermion (force_fermion_core.c:384-454) */
static void force_clover_fermion(const cplx *Xs, const cplx *Ys, double residue)
{
  int F2 = NF_ * NF_;
  static const int mn[6][2] = {{0, 1}, {0, 2}, {1, 2}, {0, 3}, {1, 3}, {2, 3}};
#pragma omp parallel for
  for (int ix = 0; ix < V_; ix++)
  {
    cplx tl[4 * 64], tr[4 * 64], fm[F2];
    const cplx *rhs = Xs + (size_t)ix * SPN, *lhs = Ys + (size_t)ix * SPN;
    for (int q = 0; q < 6; q++)
    {
      g5_sigma(tr, rhs, mn[q][0], mn[q][1]);
      g5_sigma(tl, lhs, mn[q][0], mn[q][1]);
      fmat_create(fm, tl, rhs, tr, lhs);
      cplx *cf = cl_force_ + ((size_t)ix * 6 + q) * F2;
      for (int k = 0; k < F2; k++) cf[k] += residue * fm[k];
    }
  }
}

/* the truncation order of the exponential clover's Taylor forms, from csw and
 * the mass as evaluate_sw_order chooses it (clover_exp.c:70-100): the smallest n
 * with c^(n+1) e^c < eps (n+1)!, c = 3 csw/(4+m); the series then runs to n+2 */
static int sw_exp_order(double mass)
{
  const double c = 3.0 * csw_ / (4.0 + mass);
  double a = c * exp(c), b = 2.220446049250313e-16;
  for (int n = 1; n < 100; n++)
  {
    a *= c;
    b *= (double)(n + 1);
    if (a < b) return n + 2;
  }
  return 101; /* the reference stops here with "SW parameters are out of range" */
}

/* the exponential clover's force matrices (force_clover_fermion_taylor,
 * force_fermion_core.c:631-772): with A the clover block over 4+m,
 * rhs_k = A^k X, xi_l = A^l Y, lhs_k = sum_l C_kl xi_l, C_kl = 1/(k+l+1)! for
 * k+l <= n (factorialCoef, clover_exp.c:566-592), and the same sigma insertions
 * as the linear term for every k.  The reference takes the Cayley-Hamilton
 * coefficients (doublehorner, clover_exp.c:398-563) for NF = 2, 3: the same
 * derivative of the exponential, to rounding. */
static void force_expclover_fermion(const cplx *Xs, const cplx *Ys, double residue)
{
  const int F = NF_, n2 = 2 * NF_, F2 = NF_ * NF_;
  const int nexp = sw_exp_order(static_mass_);
  const double inv = 1.0 / (4.0 + static_mass_);
  static const int mn[6][2] = {{0, 1}, {0, 2}, {1, 2}, {0, 3}, {1, 3}, {2, 3}};
  double *fact = malloc(sizeof(double) * (2 * nexp + 2));
  fact[0] = 1.0;
  for (int k = 1; k < 2 * nexp + 2; k++) fact[k] = fact[k - 1] / k;
#pragma omp parallel for
  for (int ix = 0; ix < V_; ix++)
  {
    cplx a[2][n2 * n2];
    cplx *xi = malloc(sizeof(cplx) * (size_t)nexp * SPN);
    cplx rhs[4 * 64], lhs[4 * 64], tl[4 * 64], tr[4 * 64], fm[F2];
    for (int b = 0; b < 2; b++)
    {
      clover_block(a[b], ix, b);
      for (int k = 0; k < n2 * n2; k++) a[b][k] *= inv;
    }
    /* spinor <- A spinor, block by block */
#define APPLY_A(out, in)                                                          \
  for (int b = 0; b < 2; b++)                                                     \
    for (int i = 0; i < n2; i++)                                                  \
    {                                                                             \
      cplx v = 0;                                                                 \
      for (int j = 0; j < n2; j++) v += a[b][i * n2 + j] * (in)[2 * b * F + j];   \
      (out)[2 * b * F + i] = v;                                                   \
    }
    memcpy(xi, Ys + (size_t)ix * SPN, sizeof(cplx) * SPN);
    for (int k = 0; k + 1 < nexp; k++) { APPLY_A(xi + (size_t)(k + 1) * SPN, xi + (size_t)k * SPN) }
    memcpy(rhs, Xs + (size_t)ix * SPN, sizeof(cplx) * SPN);
    for (int k = 0; k < nexp; k++)
    {
      if (k > 0)
      {
        cplx t[4 * 64];
        APPLY_A(t, rhs)
        memcpy(rhs, t, sizeof(cplx) * SPN);
      }
      for (int c = 0; c < SPN; c++) lhs[c] = 0;
      for (int l = 0; l < nexp && k + l <= nexp; l++)
        for (int c = 0; c < SPN; c++) lhs[c] += fact[k + l + 1] * xi[(size_t)l * SPN + c];
      for (int q = 0; q < 6; q++)
      {
        g5_sigma(tr, rhs, mn[q][0], mn[q][1]);
        g5_sigma(tl, lhs, mn[q][0], mn[q][1]);
        fmat_create(fm, tl, rhs, tr, lhs);
        cplx *cf = cl_force_ + ((size_t)ix * 6 + q) * F2;
        for (int e = 0; e < F2; e++) cf[e] += residue * fm[e];
      }
    }
#undef APPLY_A
    free(xi);
  }
  free(fact);
}

static void av_mul_add(double *f, double c, const double *h)
{
  for (int A = 0; A < DIMG_; A++) f[A] += c * h[A];
}

/* force_clover_core (force_fermion_core.c:282-379) */
static void force_clover_core(double dt)
{
  int F2 = NF_ * NF_;
  double coeff = dt * (repr_norm2_ / fund_norm2_) * (1. / 8.) * csw_;
#pragma omp parallel for
  for (int ix = 0; ix < V_; ix++)
  {
    cplx W[9][F2], s1[F2], s2[F2], s3[F2], fm[F2], a[F2];
    double f[DIMG_], mr[F2];
    for (int mu = 0; mu < 4; mu++)
      for (int nu = 0; nu < 4; nu++)
      {
        if (mu == nu) continue;
        int o1 = iup_[4 * ix + mu], o2 = iup_[4 * ix + nu], o3 = idn_[4 * ix + nu];
        int o4 = iup_[4 * o3 + mu], o5 = iup_[4 * o2 + mu];
        int num, sign;
        if (mu < nu) { num = nu * (nu - 1) / 2 + mu; sign = +1; }
        else { num = mu * (mu - 1) / 2 + nu; sign = -1; }
        const cplx *Z0 = cl_force_ + ((size_t)ix * 6 + num) * F2;
        const cplx *Z1 = cl_force_ + ((size_t)o1 * 6 + num) * F2;
        const cplx *Z2 = cl_force_ + ((size_t)o3 * 6 + num) * F2;
        const cplx *Z3 = cl_force_ + ((size_t)o4 * 6 + num) * F2;
        const cplx *Z4 = cl_force_ + ((size_t)o5 * 6 + num) * F2;
        const cplx *Z5 = cl_force_ + ((size_t)o2 * 6 + num) * F2;
        get_link(a, o3, mu); dagger(W[0], a);
        get_link(W[1], o3, nu);
        get_link(W[2], o1, nu);
        get_link(a, o2, mu); dagger(W[3], a);
        get_link(a, ix, nu); dagger(W[4], a);
        get_link(a, o4, nu); dagger(W[5], a);
        mm(W[6], W[0], W[1]);
        mm(W[7], W[2], W[3]);
        mm(s1, W[5], W[6]);
        mm(W[8], W[7], W[4]);
        for (int k = 0; k < F2; k++) W[8][k] -= s1[k];
        mm(fm, W[8], Z0);
        mm(s1, Z1, W[8]);
        for (int k = 0; k < F2; k++) fm[k] += s1[k];
        mm(s1, W[0], Z2);
        mm(s2, s1, W[1]);
        mm(s3, Z3, W[6]);
        for (int k = 0; k < F2; k++) s2[k] += s3[k];
        mm(s1, W[5], s2);
        for (int k = 0; k < F2; k++) fm[k] -= s1[k];
        mm(s1, W[2], Z4);
        mm(s2, s1, W[3]);
        mm(s3, W[7], Z5);
        for (int k = 0; k < F2; k++) s2[k] += s3[k];
        mm(s1, s2, W[4]);
        for (int k = 0; k < F2; k++) fm[k] += s1[k];
        get_link(a, ix, mu);
        mm(s1, a, fm);
        if (REAL_)
        {
          for (int k = 0; k < F2; k++) mr[k] = creal(s1[k]);
          orc_algebra_project(f, mr);
        }
        else
          orc_algebra_project(f, s1);
        av_mul_add(force_sum_ + ((size_t)ix * 4 + mu) * DIMG_, sign * coeff, f);
      }
  }
}

/* force_fermion_core (force_fermion_core.c:788-928), UPDATE_EO build */
void orc_force_fermion_core(cplx *Xs, cplx *Ys, int auto_fill_odd, double dt, double residue)
{
  int F2 = NF_ * NF_;
  double coeff = residue * dt * (repr_norm2_ / fund_norm2_);
  if (auto_fill_odd)
  {
    orc_Dphi_(Xs + (size_t)VH_ * SPN, ORC_ODD, Xs, ORC_EVEN);
    orc_Dphi_(Ys + (size_t)VH_ * SPN, ORC_ODD, Ys, ORC_EVEN);
    if (cl_term_)
    {
      orc_Cphi_diag_inv(static_mass_, Xs + (size_t)VH_ * SPN, Xs + (size_t)VH_ * SPN, ORC_ODD);
      orc_Cphi_diag_inv(static_mass_, Ys + (size_t)VH_ * SPN, Ys + (size_t)VH_ * SPN, ORC_ODD);
    }
  }
  coeff = -coeff;
  if (cl_term_)
  {
    if (expclover_) force_expclover_fermion(Xs, Ys, residue);
    else force_clover_fermion(Xs, Ys, residue);
  }
#pragma omp parallel for
  for (int ix = 0; ix < V_; ix++)
  {
    cplx s1[F2];
    double f[DIMG_], mr[F2];
    for (int mu = 0; mu < 4; mu++)
    {
      int iy = iup_[4 * ix + mu];
      for (int k = 0; k < F2; k++) s1[k] = 0;
      f_dir(s1, ix, mu, Xs + (size_t)ix * SPN, Ys + (size_t)iy * SPN);
      f_dir(s1, ix, mu, Ys + (size_t)ix * SPN, Xs + (size_t)iy * SPN);
      if (REAL_)
      {
        for (int k = 0; k < F2; k++) mr[k] = creal(s1[k]);
        orc_algebra_project(f, mr);
      }
      else
        orc_algebra_project(f, s1);
      av_mul_add(force_sum_ + ((size_t)ix * 4 + mu) * DIMG_, coeff, f);
    }
  }
}

/* clover_la_logdet (clover_tools.c:312-331): la[id] -= nf log(prod of the LDL
 * diagonals of both blocks) on the odd sites, la in HiRep's site order */
void orc_clover_la_logdet(double nf, double mass, double *la)
{
  orc_compute_ldl_decomp(4.0 + mass);
  for (int id = VH_; id < V_; id++)
  {
    const cplx *A = cl_ldl_ + (size_t)id * 2 * LDLN, *B = A + LDLN;
    double prod = 1;
    for (int n = 0; n < 2 * NF_; n++) prod *= creal(CPX(A, n, n)) * creal(CPX(B, n, n));
    la[id] -= nf * log(prod);
  }
}

/* _compute_clover_force + compute_force_logdet (clover_tools.c:208-310) */
void orc_force_clover_logdet(double mass, double coeff)
{
  /* the exponential clover blocks are traceless, det D_oo does not depend on
   * the links: no log-det force (force_clover_logdet exists for WITH_CLOVER only,
   * force_fermion_core.c:776-782) */
  if (expclover_) return;
  int F = NF_, N2 = 2 * NF_, F2 = NF_ * NF_;
  orc_compute_ldl_decomp(4.0 + mass);
#pragma omp parallel for
  for (int id = VH_; id < V_; id++)
  {
    cplx A[N2][N2], B[N2][N2];
    memset(A, 0, sizeof(A));
    memset(B, 0, sizeof(B));
    const cplx *U = cl_ldl_ + (size_t)id * 2 * LDLN, *L = U + LDLN;
    for (int n = 0; n < N2; n++)
    {
      A[n][n] = coeff;
      B[n][n] = coeff;
      for (int i = n; i < N2; i++)
        for (int k = 0; k < i; k++)
        {
          A[i][n] -= CPX(U, i, k) * A[k][n];
          B[i][n] -= CPX(L, i, k) * B[k][n];
        }
      for (int i = N2 - 1; i >= n; i--)
      {
        A[i][n] /= creal(CPX(U, i, i));
        B[i][n] /= creal(CPX(L, i, i));
        for (int k = i + 1; k < N2; k++)
        {
          A[i][n] -= conj(CPX(U, k, i)) * A[k][n];
          B[i][n] -= conj(CPX(L, k, i)) * B[k][n];
        }
      }
    }
    cplx *cf = cl_force_ + (size_t)id * 6 * F2;
    for (int i = 0; i < F; i++)
      for (int j = 0; j < F; j++)
      {
        int ij = i * F + j;
        cplx a11, a12, a21, a22, a33, a34, a43, a44;
        a21 = A[i + F][j];
        a12 = conj(A[j + F][i]);
        a43 = B[i + F][j];
        a34 = conj(B[j + F][i]);
        if (i < j)
        {
          a11 = conj(A[j][i]); a22 = conj(A[j + F][i + F]);
          a33 = conj(B[j][i]); a44 = conj(B[j + F][i + F]);
        }
        else
        {
          a11 = A[i][j]; a22 = A[i + F][j + F];
          a33 = B[i][j]; a44 = B[i + F][j + F];
        }
        if (REAL_)
        {
          cf[0 * F2 + ij] += cimag(a12) + cimag(a21) - cimag(a34) - cimag(a43);
          cf[1 * F2 + ij] += creal(a12) - creal(a21) + creal(a43) - creal(a34);
          cf[2 * F2 + ij] += cimag(a22) - cimag(a11) + cimag(a44) - cimag(a33);
          cf[3 * F2 + ij] += cimag(a11) - cimag(a22) + cimag(a44) - cimag(a33);
          cf[4 * F2 + ij] += creal(a12) - creal(a21) + creal(a34) - creal(a43);
          cf[5 * F2 + ij] -= cimag(a12) + cimag(a21) + cimag(a34) + cimag(a43);
        }
        else
        {
          cf[0 * F2 + ij] -= I * (a12 + a21 - a34 - a43);
          cf[1 * F2 + ij] += a12 - a21 + a43 - a34;
          cf[2 * F2 + ij] -= I * (a22 - a11 + a44 - a33);
          cf[3 * F2 + ij] -= I * (a11 - a22 + a44 - a33);
          cf[4 * F2 + ij] += a12 - a21 + a34 - a43;
          cf[5 * F2 + ij] += I * (a12 + a21 + a34 + a43);
        }
      }
  }
}

/* fermion_force_end (force_fermion_core.c:964-993), periodic/antiperiodic BCs */
void orc_fermion_force_end(double dt, double *force)
{
  if (cl_term_) force_clover_core(dt);
  size_t m = (size_t)V_ * 4 * DIMG_;
  for (size_t k = 0; k < m; k++) force[k] += force_sum_[k];
}

void orc_get_force_sum(double *f) { memcpy(f, force_sum_, sizeof(double) * V_ * 4 * DIMG_); }
void orc_get_clover_force(cplx *cf) { memcpy(cf, cl_force_, sizeof(cplx) * V_ * 6 * NF_ * NF_); }

/* ------------------------------------------------------------------------- */
/* average plaquette (LibHR/Observables/avr_plaquette.c:29-53,92)            */
/* fundamental links u[4*ix+mu] NG x NG                                       */
/* ------------------------------------------------------------------------- */
/* ------------------------------------------------------------------------- */
/* HMC pieces: gauge force (LibHR/Update/force0.c:22-99, staples.c:22-70),    */
/* link update (field_update.c:18-66, ExpX in suN_exp_group.c:358-378),       */
/* reunitarisation (suN_utils.c:76-150), local action (local_action.c:19-90,  */
/* mon_pg.c:36-43).  Fundamental links u[V][4][NG*NG], momenta [V][4][DIMG].  */
/* ------------------------------------------------------------------------- */
static void mat_mul_dag(int n, cplx *c, const cplx *a, const cplx *b) /* c = a b^+ */
{
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
    {
      cplx t = 0;
      for (int k = 0; k < n; k++) t += a[i * n + k] * conj(b[j * n + k]);
      c[i * n + j] = t;
    }
}
static void mat_dag_mul(int n, cplx *c, const cplx *a, const cplx *b) /* c = a^+ b */
{
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
    {
      cplx t = 0;
      for (int k = 0; k < n; k++) t += conj(a[k * n + i]) * b[k * n + j];
      c[i * n + j] = t;
    }
}

/* sum of the six staples around link (ix, mu) (staples.c:22-70) */
static void staple_sum(cplx *v, const cplx *u, int ix, int mu)
{
  const int N = NG_, N2 = NG_ * NG_;
  cplx t1[N2], t2[N2];
  for (int k = 0; k < N2; k++) v[k] = 0;
  const int ixpmu = iup_[4 * ix + mu];
  for (int i = 1; i < 4; i++)
  {
    const int nu = (mu + i) & 3;
    const int ixpnu = iup_[4 * ix + nu], ixmnu = idn_[4 * ix + nu], ixpmumnu = idn_[4 * ixpmu + nu];
#define UL(x, m) (u + ((size_t)(x) * 4 + (m)) * N2)
    /* up: U(x,nu) U(x+nu,mu) U(x+mu,nu)^+ */
    mat_mul(N, t2, UL(ix, nu), UL(ixpnu, mu));
    mat_mul_dag(N, t1, t2, UL(ixpmu, nu));
    for (int k = 0; k < N2; k++) v[k] += t1[k];
    /* down: U(x-nu,nu)^+ U(x-nu,mu) U(x+mu-nu,nu) */
    mat_mul(N, t2, UL(ixmnu, mu), UL(ixpmumnu, nu));
    mat_dag_mul(N, t1, UL(ixmnu, nu), t2);
    for (int k = 0; k < N2; k++) v[k] += t1[k];
#undef UL
  }
}

/* force0: mom(x,mu) += (-dt beta / NG) proj(U(x,mu) S(x,mu)^+) */
void orc_force0(double dt, double beta, const cplx *u, double *mom)
{
  const int N = NG_, N2 = NG_ * NG_;
  const double coeff = -dt * beta / N;
#pragma omp parallel for
  for (int ix = 0; ix < V_; ix++)
  {
    cplx st[N2], w[N2];
    double f[DIMG_];
    for (int mu = 0; mu < 4; mu++)
    {
      staple_sum(st, u, ix, mu);
      mat_mul_dag(N, w, u + ((size_t)ix * 4 + mu) * N2, st);
      orc_fund_algebra_project(f, w);
      for (int A = 0; A < DIMG_; A++) mom[((size_t)ix * 4 + mu) * DIMG_ + A] += coeff * f[A];
    }
  }
}

/* e = exp(x) for an NG x NG matrix with small norm: scaling and squaring of
 * the Taylor series (the reference's suNg_Exp is exact to rounding as well) */
static void mat_exp(int n, cplx *e, const cplx *x)
{
  const int n2 = n * n;
  double nrm = 0;
  for (int k = 0; k < n2; k++) nrm += creal(x[k] * conj(x[k]));
  nrm = sqrt(nrm);
  int sq = 0;
  while (nrm > 0.25)
  {
    nrm *= 0.5;
    sq++;
  }
  const double scale = ldexp(1.0, -sq);
  cplx a[n2], term[n2], tmp[n2];
  for (int k = 0; k < n2; k++)
  {
    a[k] = x[k] * scale;
    e[k] = (k % (n + 1) == 0) ? 1.0 : 0.0;
    term[k] = e[k];
  }
  for (int j = 1; j <= 20; j++)
  {
    mat_mul(n, tmp, term, a);
    for (int k = 0; k < n2; k++)
    {
      term[k] = tmp[k] / j;
      e[k] += term[k];
    }
  }
  for (int q = 0; q < sq; q++)
  {
    mat_mul(n, tmp, e, e);
    memcpy(e, tmp, sizeof(cplx) * n2);
  }
}

/* U(x,mu) <- exp(dt X(mom(x,mu))) U(x,mu), X = sum_A mom_A iT_A (ExpX) */
void orc_update_gauge_field(double dt, cplx *u, const double *mom)
{
  const int N = NG_, N2 = NG_ * NG_;
#pragma omp parallel for
  for (int l = 0; l < 4 * V_; l++)
  {
    cplx x[N2], e[N2], t[N2];
    orc_fund_algebra_represent(x, mom + (size_t)l * DIMG_);
    for (int k = 0; k < N2; k++) x[k] *= dt;
    mat_exp(N, e, x);
    mat_mul(N, t, e, u + (size_t)l * N2);
    memcpy(u + (size_t)l * N2, t, sizeof(cplx) * N2);
  }
}

/* project_to_suNg (suN_utils.c:76-150): Gram-Schmidt of the rows, then the
 * determinant's phase removed with det^(-1/NG) (principal branch) */
static cplx mat_det(int n, const cplx *m)
{
  cplx a[n * n], d = 1;
  memcpy(a, m, sizeof(cplx) * n * n);
  for (int i = 0; i < n; i++)
  {
    int p = i;
    for (int r = i + 1; r < n; r++)
      if (cabs(a[r * n + i]) > cabs(a[p * n + i])) p = r;
    if (p != i)
    {
      for (int k = 0; k < n; k++)
      {
        cplx t = a[i * n + k];
        a[i * n + k] = a[p * n + k];
        a[p * n + k] = t;
      }
      d = -d;
    }
    if (a[i * n + i] == 0) return 0;
    d *= a[i * n + i];
    for (int r = i + 1; r < n; r++)
    {
      cplx f = a[r * n + i] / a[i * n + i];
      for (int k = i; k < n; k++) a[r * n + k] -= f * a[i * n + k];
    }
  }
  return d;
}

void orc_project_gauge_field(cplx *u)
{
  const int N = NG_, N2 = NG_ * NG_;
#pragma omp parallel for
  for (int l = 0; l < 4 * V_; l++)
  {
    cplx *m = u + (size_t)l * N2;
    double nrm = 0;
    for (int k = 0; k < N2; k++) nrm += creal(m[k] * conj(m[k]));
    if (nrm < 1.e-28) continue;
    for (int i = 0; i < N; i++)
    {
      cplx *vi = m + i * N;
      for (int j = 0; j < i; j++)
      {
        const cplx *vj = m + j * N;
        cplx z = 0;
        for (int k = 0; k < N; k++) z += conj(vj[k]) * vi[k];
        for (int k = 0; k < N; k++) vi[k] -= z * vj[k];
      }
      double q = 0;
      for (int k = 0; k < N; k++) q += creal(vi[k] * conj(vi[k]));
      q = 1.0 / sqrt(q);
      for (int k = 0; k < N; k++) vi[k] *= q;
    }
    cplx f = cpow(mat_det(N, m), -1.0 / N);
    for (int k = 0; k < N2; k++) m[k] *= f;
  }
}

/* local action per site (local_action.c:19-90, mon_pg.c:36-43):
 * 0.5 * C(F) * sum_mu |mom(x,mu)|^2 - beta/NG * (sum of the 6 plaquettes at x) */
void orc_local_hmc_action(double beta, const cplx *u, const double *mom, double *loc)
{
  const int N = NG_, N2 = NG_ * NG_;
#pragma omp parallel for
  for (int ix = 0; ix < V_; ix++)
  {
    double a = 0;
    for (int q = 0; q < 4 * DIMG_; q++) a += mom[(size_t)ix * 4 * DIMG_ + q] * mom[(size_t)ix * 4 * DIMG_ + q];
    a *= 0.5 * fund_norm2_;
    cplx w1[N2], w2[N2];
    double pl = 0;
    for (int mu = 1; mu < 4; mu++)
      for (int nu = 0; nu < mu; nu++)
      {
        mat_mul(N, w1, u + ((size_t)ix * 4 + mu) * N2, u + ((size_t)iup_[4 * ix + mu] * 4 + nu) * N2);
        mat_mul(N, w2, u + ((size_t)ix * 4 + nu) * N2, u + ((size_t)iup_[4 * ix + nu] * 4 + mu) * N2);
        for (int i = 0; i < N; i++)
          for (int k = 0; k < N; k++) pl += creal(w1[i * N + k] * conj(w2[i * N + k]));
      }
    loc[ix] = a - beta / N * pl;
  }
}

double orc_avr_plaquette(const cplx *u)
{
  int N = NG_;
  double pa = 0;
#pragma omp parallel for reduction(+ : pa)
  for (int ix = 0; ix < V_; ix++)
  {
    cplx w1[N * N], w2[N * N];
    for (int mu = 1; mu < 4; mu++)
      for (int nu = 0; nu < mu; nu++)
      {
        const cplx *v1 = u + (size_t)(4 * ix + mu) * N * N;
        const cplx *v2 = u + (size_t)(4 * iup_[4 * ix + mu] + nu) * N * N;
        const cplx *v3 = u + (size_t)(4 * iup_[4 * ix + nu] + mu) * N * N;
        const cplx *v4 = u + (size_t)(4 * ix + nu) * N * N;
        mat_mul(N, w1, v1, v2);
        mat_mul(N, w2, v4, v3);
        double p = 0;
        for (int i = 0; i < N; i++)
          for (int k = 0; k < N; k++) p += creal(w1[i * N + k] * conj(w2[i * N + k]));
        pa += p;
      }
  }
  return pa / (6.0 * N * V_);
}
