/*
 * hr_ref: a command server around HiRep's own library (libhr.a built from the
 * reference sources by oracle/ref/Makefile).  TEST INFRASTRUCTURE ONLY: the
 * tests, the smoke check and the CPU arm of bench.py run it as the checker and
 * as the reference CPU baseline; the GPU library never links or calls it.
 *
 * It runs HiRep's serial (no MPI) OpenMP build unchanged: setup_process /
 * setup_gauge_fields (LibHR/Geometry/process_init.c), the gauge-field read flow
 * of read_gauge_field (LibHR/IO/archive.c:230-243) on raw bytes, and then the
 * operators, inverters and force of the hot path as HiRep's programs call them.
 *
 * Protocol: one command per line on stdin, one reply line ("ok ..." or
 * "err ...") on the original stdout.  HiRep's logger writes to files in the
 * working directory (out_0, err_0); stdout itself is sent to hr_ref.log so
 * that nothing the library prints can interleave with the replies.  Bulk data
 * moves through files in HiRep's own host layout:
 *   spinor field   complex double [nsites][4][NF]   (nsites = V/2 or V)
 *   gauge field    complex double [V][4][NG][NG]     (site order = ipt)
 *   represented    [V][4][NF][NF] complex, or real for a real representation
 *   clover term    complex double [V][4][NF][NF]     (cl_term, clover_tools.c)
 *   clover LDL     complex double [V][2][NF(2NF+1)]  (ldl_t, spinor_field.h:31-35)
 *   force          double [V][4][NG*NG-1]            (suNg_av_field)
 *
 * Commands (slot = a block of n contiguous spinor fields of one geometry):
 *   alloc S e|o|f N          alloc_spinor_field_f(N, &glat_even/odd/glattice)
 *   load S K PATH            read field K of slot S from PATH
 *   save S K PATH            write field K of slot S to PATH
 *   gauge PATH               u_gauge <- PATH, BCs as read_gauge_field, represent_gauge_field()
 *   random_u                 random_u(u_gauge) (ranlux, rlx_seed of the input file), then as gauge
 *   gauge_save PATH          u_gauge (fundamental, with its BCs)
 *   gauge_f_save PATH        u_gauge_f (represented, with BCs)
 *   gaussian S K             gaussian_spinor_field(field K of slot S)
 *   geometry IPT IUP IDN     int32 ipt[V], iup[4V], idn[4V]
 *   csw C                    set_csw(C); compute_clover_term()
 *   clterm_save PATH         cl_term
 *   ldl_save M PATH          compute_ldl_decomp(4+M); cl_ldl
 *   op NAME M OUT IN         one operator application (names below)
 *   cg NAME M ERR2 MAXIT IN OUT N s1..sN      cg_mshift, reply "ok MVM"
 *   cgflt NAME M ERR2 MAXIT IN OUT N s1..sN   cg_mshift_flt with NAME's float form
 *   force M DT RES FILL X Y PATH              fermion_force_begin, force_fermion_core,
 *                                             fermion_force_end into a zero field
 *   clforce_save PATH        cl_force after the last force (clover builds)
 *   plaq                     avr_plaquette()
 *   sqnorm S K               spinor_field_sqnorm_f
 *   time NAME M OUT IN W R   W warm-up and R timed applications, reply
 *                            "ok MEDIAN_US MIN_US THREADS"
 *   timecg NAME M ERR2 IN OUT W R   the same for a single-shift cg_mshift
 *   g5qmr NAME M ERR2 MAXIT IN OUT N s1..sN   g5QMR_mshift, reply "ok MVM"
 *   minres NAME M ERR2 MAXIT IN OUT           MINRES (no trial), reply "ok MVM"
 *   mom_load PATH / mom_save PATH             the momenta field [V][4][NG*NG-1]
 *   force0 DT BETA           force0 (the plaquette action's force) into the momenta
 *   update_gauge DT          update_gauge_field: U <- exp(dt mom) U, represented
 *   gauge_write PATH / gauge_read PATH        write_gauge_field / read_gauge_field (+ represent)
 *   quit
 */
#define MAIN_PROGRAM

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <time.h>
#include <unistd.h>
#include <fcntl.h>
#include "io.h"
#include "random.h"
#include "error.h"
#include "geometry.h"
#include "memory.h"
#include "update.h"
#include "global.h"
#include "observables.h"
#include "suN.h"
#include "suN_types.h"
#include "dirac.h"
#include "linear_algebra.h"
#include "inverters.h"
#include "representation.h"
#include "utils.h"
#include "logger.h"
#include "setup.h"
#include "communications.h"
#include "clover_tools.h"
#ifdef _OPENMP
#include <omp.h>
#endif

#define NSLOT 64
static spinor_field *slot[NSLOT];
static suNg_av_field *g_mom = NULL;
static int slot_n[NSLOT];
static FILE *reply;

static void say(const char *fmt, ...) __attribute__((format(printf, 1, 2)));
#include <stdarg.h>
static void say(const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vfprintf(reply, fmt, ap);
  va_end(ap);
  fputc('\n', reply);
  fflush(reply);
}

static int rw(const char *path, void *buf, size_t bytes, int write)
{
  FILE *f = fopen(path, write ? "wb" : "rb");
  if (!f)
    return -1;
  size_t n = write ? fwrite(buf, 1, bytes, f) : fread(buf, 1, bytes, f);
  fclose(f);
  return n == bytes ? 0 : -1;
}

static size_t field_sites(spinor_field *s) { return (size_t)s->type->gsize_spinor; }

/* ---------------------------------------------------------------- operators */
typedef void (*mop_t)(double, spinor_field *, spinor_field *);
typedef void (*mop_flt_t)(double, spinor_field_flt *, spinor_field_flt *);

static void op_Dphi_massless(double m, spinor_field *out, spinor_field *in)
{
  (void)m;
  Dphi_(out, in);
}

static struct
{
  const char *name;
  mop_t f;
  mop_flt_t ff;
} ops[] = {
    {"Dphi_", op_Dphi_massless, NULL},
    {"Dphi", Dphi, Dphi_flt},
    {"g5Dphi", g5Dphi, g5Dphi_flt},
    {"g5Dphi_sq", g5Dphi_sq, g5Dphi_sq_flt},
    {"Dphi_eopre", Dphi_eopre, Dphi_eopre_flt},
    {"Dphi_oepre", Dphi_oepre, Dphi_oepre_flt},
    {"g5Dphi_eopre", g5Dphi_eopre, g5Dphi_eopre_flt},
    {"g5Dphi_eopre_sq", g5Dphi_eopre_sq, g5Dphi_eopre_sq_flt},
#if defined(WITH_CLOVER) || defined(WITH_EXPCLOVER)
    {"Cphi", Cphi, NULL},
    {"g5Cphi", g5Cphi, NULL},
    {"g5Cphi_sq", g5Cphi_sq, NULL},
    {"Cphi_eopre", Cphi_eopre, NULL},
    {"g5Cphi_eopre", g5Cphi_eopre, NULL},
    {"g5Cphi_eopre_sq", g5Cphi_eopre_sq, NULL},
    {"Cphi_diag", Cphi_diag, NULL},
    {"Cphi_diag_inv", Cphi_diag_inv, NULL},
#endif
};

static int find_op(const char *name)
{
  for (int i = 0; i < (int)(sizeof(ops) / sizeof(ops[0])); i++)
    if (strcmp(ops[i].name, name) == 0)
      return i;
  return -1;
}

/* the inverters take spinor_operator pointers; the mass rides in statics, as
 * in HiRep's own test programs (check_inverters_1.c) */
static mop_t cur_f;
static mop_flt_t cur_ff;
static double cur_m;
static void cur_op(spinor_field *out, spinor_field *in) { cur_f(cur_m, out, in); }
static void cur_op_flt(spinor_field_flt *out, spinor_field_flt *in) { cur_ff(cur_m, out, in); }

static double now_us(void)
{
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec * 1e6 + t.tv_nsec * 1e-3;
}

static int cmp_d(const void *a, const void *b)
{
  double x = *(const double *)a, y = *(const double *)b;
  return (x > y) - (x < y);
}

static int threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* the read flow of read_gauge_field (archive.c:230-243), then represent */
static void gauge_loaded(void)
{
  apply_BCs_on_fundamental_gauge_field();
#ifndef ALLOCATE_REPR_GAUGE_FIELD
  u_gauge_f = (suNf_field *)((void *)u_gauge);
  apply_BCs_on_represented_gauge_field();
#endif
  start_gf_sendrecv(u_gauge);
  represent_gauge_field();
}

static spinor_field *field_of(int s, int k)
{
  if (s < 0 || s >= NSLOT || slot[s] == NULL || k < 0 || k >= slot_n[s])
    return NULL;
  return slot[s] + k;
}

static void run(char *line)
{
  char cmd[64], a[512], b[512], c[512], d[64], e[64];
  int s, k, n;
  double m;
  if (sscanf(line, "%63s", cmd) != 1)
    return;
  if (strcmp(cmd, "alloc") == 0)
  {
    char par;
    if (sscanf(line, "%*s %d %c %d", &s, &par, &n) != 3 || s < 0 || s >= NSLOT || n < 1)
      return say("err alloc");
    geometry_descriptor *t = par == 'e' ? &glat_even : par == 'o' ? &glat_odd : &glattice;
    if (slot[s])
      free_spinor_field_f(slot[s]);
    slot[s] = alloc_spinor_field_f(n, t);
    slot_n[s] = n;
    for (int i = 0; i < n; i++)
      spinor_field_zero_f(slot[s] + i);
    return say("ok %d", (int)field_sites(slot[s]));
  }
  if (strcmp(cmd, "load") == 0 || strcmp(cmd, "save") == 0)
  {
    if (sscanf(line, "%*s %d %d %511s", &s, &k, a) != 3 || !field_of(s, k))
      return say("err %s", cmd);
    spinor_field *f = field_of(s, k);
    size_t bytes = field_sites(f) * sizeof(suNf_spinor);
    if (rw(a, f->ptr, bytes, cmd[0] == 's'))
      return say("err io %s", a);
    return say("ok");
  }
  if (strcmp(cmd, "gauge") == 0)
  {
    if (sscanf(line, "%*s %511s", a) != 1 || rw(a, u_gauge->ptr, 4 * (size_t)glattice.gsize_gauge * sizeof(suNg), 0))
      return say("err gauge");
    gauge_loaded();
    return say("ok");
  }
  if (strcmp(cmd, "random_u") == 0)
  {
    random_u(u_gauge);
    gauge_loaded();
    return say("ok");
  }
  if (strcmp(cmd, "gauge_save") == 0 || strcmp(cmd, "gauge_f_save") == 0)
  {
    if (sscanf(line, "%*s %511s", a) != 1)
      return say("err");
    int fund = strcmp(cmd, "gauge_save") == 0;
    void *p = fund ? (void *)u_gauge->ptr : (void *)u_gauge_f->ptr;
    size_t bytes = 4 * (size_t)glattice.gsize_gauge * (fund ? sizeof(suNg) : sizeof(suNf));
    return say(rw(a, p, bytes, 1) ? "err io" : "ok");
  }
  if (strcmp(cmd, "gaussian") == 0)
  {
    if (sscanf(line, "%*s %d %d", &s, &k) != 2 || !field_of(s, k))
      return say("err gaussian");
    gaussian_spinor_field(field_of(s, k));
    return say("ok");
  }
  if (strcmp(cmd, "geometry") == 0)
  {
    if (sscanf(line, "%*s %511s %511s %511s", a, b, c) != 3)
      return say("err geometry");
    size_t v = (size_t)GLB_T * GLB_X * GLB_Y * GLB_Z;
    if (rw(a, ipt, v * sizeof(int), 1) || rw(b, iup, 4 * v * sizeof(int), 1) || rw(c, idn, 4 * v * sizeof(int), 1))
      return say("err io");
    return say("ok %zu", v);
  }
  if (strcmp(cmd, "plaq") == 0)
    return say("ok %.17e", avr_plaquette());
  if (strcmp(cmd, "sqnorm") == 0)
  {
    if (sscanf(line, "%*s %d %d", &s, &k) != 2 || !field_of(s, k))
      return say("err sqnorm");
    return say("ok %.17e", spinor_field_sqnorm_f(field_of(s, k)));
  }
#if defined(WITH_CLOVER) || defined(WITH_EXPCLOVER)
  if (strcmp(cmd, "csw") == 0)
  {
    if (sscanf(line, "%*s %lf", &m) != 1)
      return say("err csw");
    set_csw(&m);
    compute_clover_term();
    return say("ok");
  }
  if (strcmp(cmd, "clterm_save") == 0)
  {
    if (sscanf(line, "%*s %511s", a) != 1)
      return say("err");
    return say(rw(a, cl_term->ptr, 4 * (size_t)glattice.gsize_gauge * sizeof(suNfc), 1) ? "err io" : "ok");
  }
  if (strcmp(cmd, "clforce_save") == 0)
  {
    if (sscanf(line, "%*s %511s", a) != 1)
      return say("err");
    return say(rw(a, cl_force->ptr, 6 * (size_t)glattice.gsize_gauge * sizeof(suNf), 1) ? "err io" : "ok");
  }
#endif
#if defined(WITH_CLOVER)
  if (strcmp(cmd, "ldl_save") == 0)
  {
    if (sscanf(line, "%*s %lf %511s", &m, a) != 2)
      return say("err");
    compute_ldl_decomp(4.0 + m);
    return say(rw(a, cl_ldl->ptr, (size_t)glattice.gsize_gauge * sizeof(ldl_t), 1) ? "err io" : "ok");
  }
#endif
  if (strcmp(cmd, "op") == 0 || strcmp(cmd, "time") == 0)
  {
    int o, i, w = 0, r = 1;
    int nread = sscanf(line, "%*s %63s %lf %d %d %d %d", d, &m, &o, &i, &w, &r);
    if (nread < 4 || (cmd[0] == 't' && nread != 6))
      return say("err %s args", cmd);
    int id = find_op(d);
    if (id < 0 || !field_of(o, 0) || !field_of(i, 0))
      return say("err %s operator or slot", cmd);
    if (cmd[0] == 'o')
    {
      ops[id].f(m, field_of(o, 0), field_of(i, 0));
      return say("ok");
    }
    if (r < 1)
      return say("err reps");
    double *t = malloc(sizeof(double) * r);
    for (int j = 0; j < w; j++)
      ops[id].f(m, field_of(o, 0), field_of(i, 0));
    for (int j = 0; j < r; j++)
    {
      double t0 = now_us();
      ops[id].f(m, field_of(o, 0), field_of(i, 0));
      t[j] = now_us() - t0;
    }
    qsort(t, r, sizeof(double), cmp_d);
    say("ok %.3f %.3f %d", t[r / 2], t[0], threads());
    free(t);
    return;
  }
  if (strcmp(cmd, "cg") == 0 || strcmp(cmd, "cgflt") == 0 || strcmp(cmd, "timecg") == 0)
  {
    double err2;
    int maxit = 0, in, out, off, w = 0, r = 1;
    int timed = cmd[0] == 't';
    if (timed)
    {
      if (sscanf(line, "%*s %63s %lf %lf %d %d %d %d", d, &m, &err2, &in, &out, &w, &r) != 7)
        return say("err timecg args");
      n = 1;
    }
    else if (sscanf(line, "%*s %63s %lf %lf %d %d %d %d%n", d, &m, &err2, &maxit, &in, &out, &n, &off) != 7)
      return say("err cg args");
    int id = find_op(d);
    if (id < 0 || n < 1 || n > 64 || !field_of(in, 0) || !field_of(out, n - 1))
      return say("err cg operator or slot");
    double sh[64] = {0};
    if (!timed)
    {
      char *p = line + off;
      for (int j = 0; j < n; j++)
      {
        int used;
        if (sscanf(p, "%lf%n", &sh[j], &used) != 1)
          return say("err cg shifts");
        p += used;
      }
    }
    mshift_par par;
    par.n = n;
    par.shift = sh;
    par.err2 = err2;
    par.max_iter = maxit;
    par.add_par = NULL;
    cur_f = ops[id].f;
    cur_ff = ops[id].ff;
    cur_m = m;
    int flt = strcmp(cmd, "cgflt") == 0;
    if (flt && (cur_ff == NULL || u_gauge_f_flt == NULL))
      return say("err no float operator");
    if (!timed)
    {
      int mvm = flt ? cg_mshift_flt(&par, cur_op, cur_op_flt, field_of(in, 0), field_of(out, 0))
                    : cg_mshift(&par, cur_op, field_of(in, 0), field_of(out, 0));
      return say("ok %d", mvm);
    }
    if (r < 1)
      return say("err reps");
    double *t = malloc(sizeof(double) * r);
    int mvm = 0;
    for (int j = 0; j < w + r; j++)
    {
      spinor_field_zero_f(field_of(out, 0));
      double t0 = now_us();
      mvm = cg_mshift(&par, cur_op, field_of(in, 0), field_of(out, 0));
      if (j >= w)
        t[j - w] = now_us() - t0;
    }
    qsort(t, r, sizeof(double), cmp_d);
    say("ok %.3f %.3f %d %d", t[r / 2], t[0], threads(), mvm);
    free(t);
    return;
  }
  if (strcmp(cmd, "g5qmr") == 0 || strcmp(cmd, "minres") == 0)
  {
    double err2;
    int maxit, in, out, off = 0;
    int qmr = cmd[0] == 'g';
    if (qmr)
    {
      if (sscanf(line, "%*s %63s %lf %lf %d %d %d %d%n", d, &m, &err2, &maxit, &in, &out, &n, &off) != 7)
        return say("err g5qmr args");
    }
    else
    {
      if (sscanf(line, "%*s %63s %lf %lf %d %d %d", d, &m, &err2, &maxit, &in, &out) != 6)
        return say("err minres args");
      n = 1;
    }
    int id = find_op(d);
    if (id < 0 || n < 1 || n > 64 || !field_of(in, 0) || !field_of(out, n - 1))
      return say("err %s operator or slot", cmd);
    cur_f = ops[id].f;
    cur_m = m;
    if (!qmr)
    {
      MINRES_par mp;
      mp.err2 = err2;
      mp.max_iter = maxit;
      return say("ok %d", MINRES(&mp, cur_op, field_of(in, 0), field_of(out, 0), NULL));
    }
    double sh[64] = {0};
    char *p = line + off;
    for (int j = 0; j < n; j++)
    {
      int used;
      if (sscanf(p, "%lf%n", &sh[j], &used) != 1)
        return say("err g5qmr shifts");
      p += used;
    }
    mshift_par par;
    par.n = n;
    par.shift = sh;
    par.err2 = err2;
    par.max_iter = maxit;
    par.add_par = NULL;
    return say("ok %d", g5QMR_mshift(&par, cur_op, field_of(in, 0), field_of(out, 0)));
  }
  if (strcmp(cmd, "mom_load") == 0 || strcmp(cmd, "mom_save") == 0)
  {
    if (sscanf(line, "%*s %511s", a) != 1)
      return say("err");
    if (!g_mom)
      g_mom = alloc_avfield(&glattice);
    return say(rw(a, g_mom->ptr, 4 * (size_t)glattice.gsize_gauge * sizeof(suNg_algebra_vector), cmd[4] == 's')
                   ? "err io"
                   : "ok");
  }
  if (strcmp(cmd, "force0") == 0)
  {
    double dt, beta;
    if (sscanf(line, "%*s %lf %lf", &dt, &beta) != 2 || !g_mom)
      return say("err force0");
    force_gauge_par fp;
    fp.beta = beta;
    fp.c0 = 1.0;
    fp.c1 = 0.0;
    fp.momenta = &g_mom;
    force0(dt, &fp);
    return say("ok");
  }
  if (strcmp(cmd, "update_gauge") == 0)
  {
    double dt;
    if (sscanf(line, "%*s %lf", &dt) != 1 || !g_mom)
      return say("err update_gauge");
    field_gauge_par gp;
    gp.field = &u_gauge;
    gp.momenta = &g_mom;
    update_gauge_field(dt, &gp);
    return say("ok");
  }
  if (strcmp(cmd, "gauge_write") == 0 || strcmp(cmd, "gauge_read") == 0)
  {
    if (sscanf(line, "%*s %511s", a) != 1)
      return say("err");
    if (cmd[6] == 'w')
      write_gauge_field(a);
    else
    {
      read_gauge_field(a);
      start_gf_sendrecv(u_gauge);
      represent_gauge_field();
    }
    return say("ok");
  }
  if (strcmp(cmd, "force") == 0)
  {
    double dt, res;
    int fill, xs, ys;
    if (sscanf(line, "%*s %lf %lf %lf %d %d %d %511s", &m, &dt, &res, &fill, &xs, &ys, a) != 7 ||
        !field_of(xs, 0) || !field_of(ys, 0))
      return say("err force args");
    set_dirac_mass(m);
    suNg_av_field *mom = alloc_avfield(&glattice);
    _MASTER_FOR(&glattice, ix)
    {
      for (int mu = 0; mu < 4; mu++)
      {
        _algebra_vector_zero_g(*_4FIELD_AT(mom, ix, mu));
      }
    }
    fermion_force_begin();
    force_fermion_core(field_of(xs, 0), field_of(ys, 0), fill, dt, res);
    fermion_force_end(dt, mom);
    int bad = rw(a, mom->ptr, 4 * (size_t)glattice.gsize_gauge * sizeof(suNg_algebra_vector), 1);
    free_avfield(mom);
    return say(bad ? "err io" : "ok");
  }
  (void)e;
  say("err unknown command %s", cmd);
}

int main(int argc, char *argv[])
{
  /* replies go to the original stdout; the library's own output to a file */
  int rfd = dup(1);
  reply = fdopen(rfd, "w");
  int lfd = open("hr_ref.log", O_WRONLY | O_CREAT | O_TRUNC, 0644);
  if (lfd >= 0)
  {
    dup2(lfd, 1);
    close(lfd);
  }

  logger_map("DEBUG", "debug");
  setup_process(&argc, &argv);
  setup_gauge_fields();
#ifdef DPHI_FLT
  /* setup_gauge_fields allocates the float links only under DPHI_FLT */
  if (u_gauge_f_flt == NULL)
    u_gauge_f_flt = alloc_gfield_f_flt(&glattice);
#endif
  say("ok ready NG=%d NF=%d V=%d threads=%d", NG, NF, GLB_T * GLB_X * GLB_Y * GLB_Z, threads());

  char *line = NULL;
  size_t cap = 0;
  while (getline(&line, &cap, stdin) > 0)
  {
    if (strncmp(line, "quit", 4) == 0)
      break;
    run(line);
  }
  free(line);
  say("ok bye");
  return 0;
}
