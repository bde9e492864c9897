/*
 * hrgpu_hirep.c -- HiRep's hot-path functions forwarded to libhrgpu, for a
 * HiRep program whose fields stay in host memory (no WITH_GPU build).
 *
 * This is the binding a HiRep maintainer adds on HiRep's side of the C ABI
 * (include/hrgpu.h).  It is compiled against HiRep's own headers (the ones its
 * generators write for the configuration) and linked into an unchanged HiRep
 * program with the linker's --wrap for every function it replaces, so HiRep's
 * sources stay untouched: a call to Dphi_eopre from the program or from the
 * rest of libhr (D_update.c's H2, the inverters, the force drivers) lands in
 * __wrap_Dphi_eopre here, and __real_X still names HiRep's own X.
 *
 * Each operator uploads its input field, runs on the GPU and downloads the
 * result (hrgpu_spinor_upload / _download convert HiRep's AoS layout and site
 * order exactly).  represent_gauge_field() keeps HiRep's own host computation
 * and then hands the represented links (boundary conditions applied) to the
 * GPU; a new clover term is rebuilt on the GPU at the next clover operator.
 * cg_mshift runs the device-resident solver for the operators HiRep's update
 * code passes (H2, H of D_update.c:41-74); for an operator the caller wrote
 * itself (check_inverters_1.c's M) the operator cannot be identified from its
 * address, so HiRep's own recursion runs on the host around it, each
 * application on the GPU through this file -- never a different operator.
 * Errors from the library go to HiRep's error() (fatal), except
 * HRGPU_E_NOCONV, which is logged like HiRep's own non-convergence
 * (cg_mshift.c:131-136).
 *
 * Threading: HiRep may call these from inside an OpenMP parallel region
 * (Dphi.c:210-225); the GPU work is issued once, by the master thread, and the
 * team waits at a barrier.
 */
#include <stdlib.h>
#include <cuda_runtime_api.h>

#include "global.h"
#include "dirac.h"
#include "inverters.h"
#include "update.h"
#include "memory.h"
#include "logger.h"
#include "error.h"
#include "representation.h"
#include "clover_tools.h"
#include "hr_omp.h"
#include "hrgpu.h"

#if defined(REPR_FUNDAMENTAL)
#define HRGPU_REPR HRGPU_FUND
#elif defined(REPR_ADJOINT)
#define HRGPU_REPR HRGPU_ADJ
#elif defined(REPR_SYMMETRIC)
#define HRGPU_REPR HRGPU_SYM
#else
#define HRGPU_REPR HRGPU_ASYM
#endif

#if defined(WITH_CLOVER) || defined(WITH_EXPCLOVER)
#define SHIM_CLOVER 1
#endif

#define HR(call)                                                                    \
  do                                                                                \
  {                                                                                 \
    int _rc = (call);                                                               \
    if (_rc)                                                                        \
      error(1, _rc, (char *)__func__, (char *)hrgpu_last_error());                  \
  } while (0)

/* the GPU work of one call, issued once inside a parallel region */
#define ONCE(...)                        \
  do                                     \
  {                                      \
    _OMP_PRAGMA(master) { __VA_ARGS__; } \
    _OMP_PRAGMA(barrier)                 \
  } while (0)

static int ready = 0;
#ifdef SHIM_CLOVER
static int clover_dirty = 1;
#endif

/* device fields: four of the full-lattice size (enough for any parity), plus
 * a pool for the solutions of a multi-shift solve */
#define NPOOL 64
static void *dev[4];
static void *pool[NPOOL];
static size_t full_bytes;

static void setup(void)
{
  if (ready)
    return;
  HR(hrgpu_init(0));
  HR(hrgpu_lattice_init(GLB_T, GLB_X, GLB_Y, GLB_Z, NG, HRGPU_REPR, ipt));
  full_bytes = hrgpu_spinor_bytes(HRGPU_FULL, HRGPU_DOUBLE);
  for (int i = 0; i < 4; i++)
    error(cudaMalloc(&dev[i], full_bytes) != cudaSuccess, 1, "hrgpu_hirep setup", "cudaMalloc failed");
  lprintf("HRGPU", 0, "hot path on the GPU (libhrgpu): %dx%dx%dx%d, NG=%d, NF=%d\n", GLB_T, GLB_X, GLB_Y, GLB_Z, NG,
          hrgpu_nf());
  ready = 1;
}

static void *pool_field(int i)
{
  error(i >= NPOOL, 1, "hrgpu_hirep", "more than 64 shifts");
  if (!pool[i])
    error(cudaMalloc(&pool[i], full_bytes) != cudaSuccess, 1, "hrgpu_hirep", "cudaMalloc failed");
  return pool[i];
}

static int par_of(geometry_descriptor *t)
{
  return t == &glat_even ? HRGPU_EVEN : t == &glat_odd ? HRGPU_ODD : HRGPU_FULL;
}

static void up(void *d, spinor_field *s) { HR(hrgpu_spinor_upload(d, s->ptr, par_of(s->type), HRGPU_DOUBLE)); }
static void down(spinor_field *s, void *d) { HR(hrgpu_spinor_download(s->ptr, d, par_of(s->type), HRGPU_DOUBLE)); }
static void up_f(void *d, spinor_field_flt *s) { HR(hrgpu_spinor_upload(d, s->ptr, par_of(s->type), HRGPU_FLOAT)); }
static void down_f(spinor_field_flt *s, void *d) { HR(hrgpu_spinor_download(s->ptr, d, par_of(s->type), HRGPU_FLOAT)); }

#ifdef SHIM_CLOVER
static void clover_sync(void)
{
  if (!clover_dirty)
    return;
#ifdef WITH_EXPCLOVER
  HR(hrgpu_expclover_init(get_csw()));
#else
  HR(hrgpu_clover_init(get_csw()));
#endif
  clover_dirty = 0;
}
#endif

/* ------------------------------------------------------------ gauge field -- */
void __real_represent_gauge_field(void);
/* representation.c:391-468: HiRep's host computation, then the links to the GPU */
void __wrap_represent_gauge_field(void)
{
  __real_represent_gauge_field();
  ONCE({
    setup();
    HR(hrgpu_gauge_set_f(u_gauge_f->ptr));
  });
#ifdef SHIM_CLOVER
  clover_dirty = 1;
#endif
}

#ifdef SHIM_CLOVER
void __real_compute_clover_term(void);
/* clover_tools.c:333-341: a new term (new links or csw) is rebuilt on the GPU when next used */
void __wrap_compute_clover_term(void)
{
  __real_compute_clover_term();
  clover_dirty = 1;
}
#endif

void __real_set_dirac_mass(double mass);
/* D_update.c:12-15 */
void __wrap_set_dirac_mass(double mass)
{
  __real_set_dirac_mass(mass);
  ONCE({
    setup();
    HR(hrgpu_set_dirac_mass(mass));
  });
}

/* Dphi.c:105-113 */
unsigned long int __wrap_getMVM(void)
{
  setup();
  return hrgpu_getMVM();
}

/* -------------------------------------------------------------- operators -- */
/* Dphi.c:193-374 */
void __wrap_Dphi_(spinor_field *out, spinor_field *in)
{
  ONCE({
    setup();
    up(dev[0], in);
    HR(hrgpu_Dphi_(dev[1], par_of(out->type), dev[0]));
    down(out, dev[1]);
  });
}

#define MASS_OP(name)                                            \
  void __wrap_##name(double m, spinor_field *out, spinor_field *in) \
  {                                                              \
    ONCE({                                                       \
      setup();                                                   \
      up(dev[0], in);                                            \
      HR(hrgpu_##name(m, dev[1], dev[0]));                       \
      down(out, dev[1]);                                         \
    });                                                          \
  }

MASS_OP(Dphi)             /* Dphi.c:703-783   */
MASS_OP(g5Dphi)           /* Dphi.c:785-867   */
MASS_OP(g5Dphi_sq)        /* Dphi.c:1001-1019 */
MASS_OP(Dphi_eopre)       /* Dphi.c:874-907   */
MASS_OP(Dphi_oepre)       /* Dphi.c:914-948   */
MASS_OP(g5Dphi_eopre)     /* Dphi.c:950-985   */
MASS_OP(g5Dphi_eopre_sq)  /* Dphi.c:988-998   */

#define MASS_OP_FLT(name)                                                \
  void __wrap_##name(double m, spinor_field_flt *out, spinor_field_flt *in) \
  {                                                                      \
    ONCE({                                                               \
      setup();                                                           \
      up_f(dev[0], in);                                                  \
      HR(hrgpu_##name(m, dev[1], dev[0]));                               \
      down_f(out, dev[1]);                                               \
    });                                                                  \
  }

/* Dphi_flt.c:162-593 (the library makes its FP32 links from the FP64 ones,
 * as assign_ud2u_f does on the host) */
void __wrap_Dphi_flt_(spinor_field_flt *out, spinor_field_flt *in)
{
  ONCE({
    setup();
    up_f(dev[0], in);
    HR(hrgpu_Dphi_flt_(dev[1], par_of(out->type), dev[0]));
    down_f(out, dev[1]);
  });
}
MASS_OP_FLT(Dphi_flt)
MASS_OP_FLT(g5Dphi_flt)
MASS_OP_FLT(g5Dphi_sq_flt)
MASS_OP_FLT(Dphi_eopre_flt)
MASS_OP_FLT(g5Dphi_eopre_flt)
MASS_OP_FLT(g5Dphi_eopre_sq_flt)

#ifdef SHIM_CLOVER
#define CLOVER_OP(name)                                          \
  void __wrap_##name(double m, spinor_field *out, spinor_field *in) \
  {                                                              \
    ONCE({                                                       \
      setup();                                                   \
      clover_sync();                                             \
      up(dev[0], in);                                            \
      HR(hrgpu_##name(m, dev[1], dev[0]));                       \
      down(out, dev[1]);                                         \
    });                                                          \
  }
CLOVER_OP(Cphi)             /* Dphi.c:1215-1221 */
CLOVER_OP(g5Cphi)           /* Dphi.c:1223-1227 */
CLOVER_OP(g5Cphi_sq)        /* Dphi.c:1229-1238 */
CLOVER_OP(Cphi_eopre)       /* Dphi.c:1240-1255 */
CLOVER_OP(g5Cphi_eopre)     /* Dphi.c:1257-1261 */
CLOVER_OP(g5Cphi_eopre_sq)  /* Dphi.c:1263-1272 */

/* Dphi.c:1274-1288 (out == in allowed: the copies go through separate device fields) */
void __wrap_Cphi_diag(double m, spinor_field *out, spinor_field *in)
{
  ONCE({
    setup();
    clover_sync();
    up(dev[0], in);
    HR(hrgpu_Cphi_diag(m, dev[1], dev[0], par_of(in->type)));
    down(out, dev[1]);
  });
}
void __wrap_Cphi_diag_inv(double m, spinor_field *out, spinor_field *in)
{
  ONCE({
    setup();
    clover_sync();
    up(dev[0], in);
    HR(hrgpu_Cphi_diag_inv(m, dev[1], dev[0], par_of(in->type)));
    down(out, dev[1]);
  });
}
#endif

/* -------------------------------------------------------------- inverters -- */
/* the device operator for the operators HiRep's own update code passes
 * (D_update.c:41-74), -1 for any other */
static int device_op(spinor_operator M)
{
#ifdef UPDATE_EO
#ifdef SHIM_CLOVER
  if (M == &H2)
    return HRGPU_OP_G5CPHI_EOPRE_SQ;
#else
  if (M == &H2)
    return HRGPU_OP_G5DPHI_EOPRE_SQ;
#endif
#else
#ifdef SHIM_CLOVER
  if (M == &H2)
    return HRGPU_OP_G5CPHI_SQ;
#else
  if (M == &H2)
    return HRGPU_OP_G5DPHI_SQ;
#endif
#endif
  return -1;
}

static int solve_status(int rc, int it, const char *who)
{
  if (rc == HRGPU_E_NOCONV)
    lprintf("INVERTER", 10, "%s: %s\n", who, hrgpu_last_error());
  else
    HR(rc);
  return it;
}

int __real_cg_mshift(mshift_par *par, spinor_operator M, spinor_field *in, spinor_field *out);
/* cg_mshift.c:147-195 */
int __wrap_cg_mshift(mshift_par *par, spinor_operator M, spinor_field *in, spinor_field *out)
{
  int op = device_op(M), it = 0;
  if (op < 0)
  {
    lprintf("HRGPU", 20, "cg_mshift: the caller's operator, HiRep's recursion around it\n");
    return __real_cg_mshift(par, M, in, out);
  }
  ONCE({
    setup();
#ifdef SHIM_CLOVER
    clover_sync();
#endif
    void *outs[NPOOL];
    up(dev[0], in);
    for (int i = 0; i < par->n; i++)
      outs[i] = pool_field(i);
    if (par->n == 1)
      up(outs[0], out); /* the initial guess */
    int rc = hrgpu_cg_mshift(op, get_dirac_mass(), par->n, par->shift, par->err2, par->max_iter, dev[0],
                             (void *const *)outs, &it);
    solve_status(rc, it, "cg_mshift");
    for (int i = 0; i < par->n; i++)
      down(out + i, outs[i]);
  });
  return it;
}

/* ------------------------------------------------------------------ force -- */
/* force_fermion_core.c:935-962 */
void __wrap_fermion_force_begin(void)
{
  ONCE({
    setup();
    HR(hrgpu_fermion_force_begin());
  });
}

/* force_fermion_core.c:788-928: Xs, Ys full-lattice; with auto_fill_odd their
 * odd halves are filled, as HiRep fills them in place */
void __wrap_force_fermion_core(spinor_field *Xs, spinor_field *Ys, int auto_fill_odd, double dt, double residue)
{
  ONCE({
    setup();
#ifdef SHIM_CLOVER
    clover_sync();
#endif
    spinor_field X = *Xs;
    spinor_field Y = *Ys;
    X.type = &glattice;
    Y.type = &glattice;
    up(dev[2], &X);
    up(dev[3], &Y);
    HR(hrgpu_force_fermion_core(dev[2], dev[3], auto_fill_odd, dt, residue));
    if (auto_fill_odd)
    {
      down(&X, dev[2]);
      down(&Y, dev[3]);
    }
  });
}

/* force_fermion_core.c:964-993: the accumulated force added to the host momenta */
void __wrap_fermion_force_end(double dt, suNg_av_field *force)
{
  ONCE({
    setup();
    HR(hrgpu_fermion_force_end(dt, (double *)force->ptr));
  });
}
