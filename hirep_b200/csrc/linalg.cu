// linalg.cu -- spinor-field linear algebra on the device
// (LibHR/Inverters/TMPL/linear_algebra.c.sdtmpl, instantiated for double and
// float like LibHR/Inverters/linear_algebra.c:20-59).
//
// Every operation is one streaming pass over the structure-of-arrays planes.
// Reductions use a fixed grid (<= RED_MAX_BLOCKS), a fixed per-thread order, a
// fixed block tree and a fixed fold, so results are bit-reproducible from run to
// run; they accumulate in double for both precisions.
#include "dirac.cuh"
#include "linalg.cuh"

namespace hrgpu {

// gamma matrices of Include/gamma_spinor.h:36-58: (g_mu s)_c = f[mu][c] * s_{src[mu][c]}
__constant__ int c_gsrc[4][4] = {{2, 3, 0, 1}, {3, 2, 1, 0}, {3, 2, 1, 0}, {2, 3, 0, 1}};
// factors as (re, im)
__constant__ double c_gfac[4][4][2] = {{{-1, 0}, {-1, 0}, {-1, 0}, {-1, 0}},
                                       {{0, -1}, {0, -1}, {0, 1}, {0, 1}},
                                       {{-1, 0}, {1, 0}, {1, 0}, {-1, 0}},
                                       {{0, -1}, {0, 1}, {0, 1}, {0, -1}}};

template <typename V>
__device__ __forceinline__ V cmulz(double2 c, V a) {
  V r;
  r.x = c.x * a.x - c.y * a.y;
  r.y = c.x * a.y + c.y * a.x;
  return r;
}

template <typename V>
__global__ void k_blas(int op, V *s1, const V *s2, const V *s3, double2 c1, double2 c2, long n, int ld, int nf) {
  long stride = (long)gridDim.x * blockDim.x;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    int comp = (int)((e / ld) % (4 * nf));
    int spin = comp / nf;
    double sg = spin < 2 ? 1.0 : -1.0;
    V a, b, r;
    switch (op) {
      case LA_MUL_ADD_ASSIGN: r = s1[e]; rmac(r, c1.x, s2[e]); s1[e] = r; break;
      case LA_MULC_ADD_ASSIGN: s1[e] = cadd(s1[e], cmulz(c1, s2[e])); break;
      case LA_G5_MULC_ADD_ASSIGN: s1[e] = cadd(s1[e], cmulz(make_double2(sg * c1.x, sg * c1.y), s2[e])); break;
      case LA_MUL: a = s2[e]; r.x = c1.x * a.x; r.y = c1.x * a.y; s1[e] = r; break;
      case LA_MULC: s1[e] = cmulz(c1, s2[e]); break;
      case LA_ADD: s1[e] = cadd(s2[e], s3[e]); break;
      case LA_SUB: s1[e] = csub(s2[e], s3[e]); break;
      case LA_ADD_ASSIGN: s1[e] = cadd(s1[e], s2[e]); break;
      case LA_SUB_ASSIGN: s1[e] = csub(s1[e], s2[e]); break;
      case LA_COPY: s1[e] = s2[e]; break;
      case LA_ZERO: r.x = 0; r.y = 0; s1[e] = r; break;
      case LA_MINUS: a = s2[e]; r.x = -a.x; r.y = -a.y; s1[e] = r; break;
      case LA_LC: a = s2[e]; b = s3[e]; r.x = c1.x * a.x; r.y = c1.x * a.y; rmac(r, c2.x, b); s1[e] = r; break;
      case LA_LC_ADD_ASSIGN: r = s1[e]; rmac(r, c1.x, s2[e]); rmac(r, c2.x, s3[e]); s1[e] = r; break;
      case LA_CLC: s1[e] = cadd(cmulz(c1, s2[e]), cmulz(c2, s3[e])); break;
      case LA_CLC_ADD_ASSIGN: s1[e] = cadd(s1[e], cadd(cmulz(c1, s2[e]), cmulz(c2, s3[e]))); break;
      case LA_G5: a = s2[e]; r.x = sg * a.x; r.y = sg * a.y; s1[e] = r; break;
      case LA_G5_ASSIGN: a = s1[e]; r.x = sg * a.x; r.y = sg * a.y; s1[e] = r; break;
      case LA_LC1: r = s1[e]; rmac(r, c1.x, s2[e]); s1[e] = r; break;
      case LA_LC2: a = s1[e]; r.x = c1.x * a.x; r.y = c1.x * a.y; rmac(r, c2.x, s2[e]); s1[e] = r; break;
      default: break;
    }
  }
}

// s1 = gamma_mu s2 (different components: one thread per element of s1)
template <typename V>
__global__ void k_gamma(int mu, V *s1, const V *s2, long n, int ld, int nf) {
  long stride = (long)gridDim.x * blockDim.x;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    long cb = e % ld;
    long q = e / ld;
    int comp = (int)(q % (4 * nf));
    long par = q / (4 * nf);
    int spin = comp / nf, col = comp % nf;
    int ss = c_gsrc[mu][spin];
    V a = s2[(par * 4 * nf + ss * nf + col) * ld + cb];
    double2 f = make_double2(c_gfac[mu][spin][0], c_gfac[mu][spin][1]);
    s1[e] = cmulz(f, a);
  }
}

template <typename V>
__global__ void k_lc3(V *s3, const V *s1, const V *s2, double c1, double c2, long n) {
  long stride = (long)gridDim.x * blockDim.x;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    V a = s3[e];
    rmac(a, -c1, s1[e]);
    rmac(a, -c2, s2[e]);
    a.x = -a.x;
    a.y = -a.y;
    s3[e] = a;
  }
}

// reductions: op 0 = <s1,s2> (re, im), 1 = <g5 s1, s2> (re, im), 2 = |s1|^2
template <typename V>
__global__ void __launch_bounds__(RED_THREADS) k_dot(int op, const V *s1, const V *s2, long n, int ld, int nf, double *partials) {
  double re = 0.0, im = 0.0;
  long stride = (long)gridDim.x * blockDim.x;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    V a = s1[e];
    if (op == 2) {
      re += (double)a.x * a.x + (double)a.y * a.y;
    } else {
      V b = s2[e];
      double sg = 1.0;
      if (op == 1) sg = ((int)((e / ld) % (4 * nf)) / nf) < 2 ? 1.0 : -1.0;
      re += sg * ((double)a.x * b.x + (double)a.y * b.y);
      im += sg * ((double)a.x * b.y - (double)a.y * b.x);
    }
  }
  re = block_sum(re);
  im = op == 2 ? 0.0 : block_sum(im);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = re;
    partials[2 * blockIdx.x + 1] = im;
  }
}

static unsigned grid_for(long n) {
  long b = (n + 255) / 256;
  return (unsigned)(b < RED_MAX_BLOCKS ? b : RED_MAX_BLOCKS);
}

int la_check(int par, int prec) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "linear algebra: lattice not initialised");
  HR_REQUIRE(par >= 0 && par <= 2 && (prec == HRGPU_DOUBLE || prec == HRGPU_FLOAT), HRGPU_E_ARG,
             "linear algebra: bad parity/precision");
  return 0;
}

int la_op(int op, int par, int prec, void *s1, const void *s2, const void *s3, double c1r, double c1i, double c2r,
          double c2i) {
  if (int rc = la_check(par, prec)) return rc;
  HR_REQUIRE(s1 != nullptr, HRGPU_E_ARG, "linear algebra: NULL field");
  long n = (long)spinor_elems(par);
  double2 c1 = make_double2(c1r, c1i), c2 = make_double2(c2r, c2i);
  if (prec == HRGPU_FLOAT) {
    // the float template rounds the coefficients to float (_REAL = float)
    c1 = make_double2((float)c1r, (float)c1i);
    c2 = make_double2((float)c2r, (float)c2i);
  }
  unsigned grid = grid_for(n);
  if (op >= LA_G0 && op <= LA_G3) {
    if (prec == HRGPU_DOUBLE)
      k_gamma<double2><<<grid, 256, 0, L.stream>>>(op - LA_G0, (double2 *)s1, (const double2 *)s2, n, L.ld, L.nf);
    else
      k_gamma<float2><<<grid, 256, 0, L.stream>>>(op - LA_G0, (float2 *)s1, (const float2 *)s2, n, L.ld, L.nf);
  } else if (op == LA_LC3) {
    if (prec == HRGPU_DOUBLE)
      k_lc3<double2><<<grid, 256, 0, L.stream>>>((double2 *)s1, (const double2 *)s2, (const double2 *)s3, c1r, c2r, n);
    else
      k_lc3<float2><<<grid, 256, 0, L.stream>>>((float2 *)s1, (const float2 *)s2, (const float2 *)s3, (float)c1r, (float)c2r, n);
  } else {
    if (prec == HRGPU_DOUBLE)
      k_blas<double2><<<grid, 256, 0, L.stream>>>(op, (double2 *)s1, (const double2 *)s2, (const double2 *)s3, c1, c2, n, L.ld, L.nf);
    else
      k_blas<float2><<<grid, 256, 0, L.stream>>>(op, (float2 *)s1, (const float2 *)s2, (const float2 *)s3, c1, c2, n, L.ld, L.nf);
  }
  HR_LAUNCH_CHECK();
  return 0;
}

int la_dot(int op, int par, int prec, const void *s1, const void *s2, double *res) {
  if (int rc = la_check(par, prec)) return rc;
  HR_REQUIRE(s1 && res && (op == 2 || s2), HRGPU_E_ARG, "linear algebra: NULL field");
  long n = (long)spinor_elems(par);
  unsigned grid = grid_for(n);
  if (prec == HRGPU_DOUBLE)
    k_dot<double2><<<grid, RED_THREADS, 0, L.stream>>>(op, (const double2 *)s1, (const double2 *)s2, n, L.ld, L.nf, L.partials);
  else
    k_dot<float2><<<grid, RED_THREADS, 0, L.stream>>>(op, (const float2 *)s1, (const float2 *)s2, n, L.ld, L.nf, L.partials);
  HR_LAUNCH_CHECK();
  double r[2];
  if (int rc = finish_reduction(grid, 2, r)) return rc;
  res[0] = r[0];
  if (op != 2) res[1] = r[1];  // |s1|^2 callers pass room for one value
  return 0;
}

}  // namespace hrgpu

using namespace hrgpu;

extern "C" {

int hrgpu_spinor_field_prod_re(int par, int prec, const void *s1, const void *s2, double *res) {
  double r[2];
  if (int rc = la_dot(0, par, prec, s1, s2, r)) return rc;
  *res = r[0];
  return 0;
}
int hrgpu_spinor_field_prod_im(int par, int prec, const void *s1, const void *s2, double *res) {
  double r[2];
  if (int rc = la_dot(0, par, prec, s1, s2, r)) return rc;
  *res = r[1];
  return 0;
}
int hrgpu_spinor_field_prod(int par, int prec, const void *s1, const void *s2, double *res) {
  return la_dot(0, par, prec, s1, s2, res);
}
int hrgpu_spinor_field_g5_prod_re(int par, int prec, const void *s1, const void *s2, double *res) {
  double r[2];
  if (int rc = la_dot(1, par, prec, s1, s2, r)) return rc;
  *res = r[0];
  return 0;
}
int hrgpu_spinor_field_g5_prod_im(int par, int prec, const void *s1, const void *s2, double *res) {
  double r[2];
  if (int rc = la_dot(1, par, prec, s1, s2, r)) return rc;
  *res = r[1];
  return 0;
}
int hrgpu_spinor_field_sqnorm(int par, int prec, const void *s1, double *res) {
  double r[2];
  if (int rc = la_dot(2, par, prec, s1, nullptr, r)) return rc;
  *res = r[0];
  return 0;
}
int hrgpu_spinor_field_mul_add_assign(int par, int prec, void *s1, double r, const void *s2) {
  return la_op(LA_MUL_ADD_ASSIGN, par, prec, s1, s2, nullptr, r, 0, 0, 0);
}
int hrgpu_spinor_field_mulc_add_assign(int par, int prec, void *s1, double cr, double ci, const void *s2) {
  return la_op(LA_MULC_ADD_ASSIGN, par, prec, s1, s2, nullptr, cr, ci, 0, 0);
}
int hrgpu_spinor_field_g5_mulc_add_assign(int par, int prec, void *s1, double cr, double ci, const void *s2) {
  return la_op(LA_G5_MULC_ADD_ASSIGN, par, prec, s1, s2, nullptr, cr, ci, 0, 0);
}
int hrgpu_spinor_field_mul(int par, int prec, void *s1, double r, const void *s2) {
  return la_op(LA_MUL, par, prec, s1, s2, nullptr, r, 0, 0, 0);
}
int hrgpu_spinor_field_mulc(int par, int prec, void *s1, double cr, double ci, const void *s2) {
  return la_op(LA_MULC, par, prec, s1, s2, nullptr, cr, ci, 0, 0);
}
int hrgpu_spinor_field_add(int par, int prec, void *r, const void *s1, const void *s2) {
  return la_op(LA_ADD, par, prec, r, s1, s2, 0, 0, 0, 0);
}
int hrgpu_spinor_field_sub(int par, int prec, void *r, const void *s1, const void *s2) {
  return la_op(LA_SUB, par, prec, r, s1, s2, 0, 0, 0, 0);
}
int hrgpu_spinor_field_add_assign(int par, int prec, void *s1, const void *s2) {
  return la_op(LA_ADD_ASSIGN, par, prec, s1, s2, nullptr, 0, 0, 0, 0);
}
int hrgpu_spinor_field_sub_assign(int par, int prec, void *s1, const void *s2) {
  return la_op(LA_SUB_ASSIGN, par, prec, s1, s2, nullptr, 0, 0, 0, 0);
}
int hrgpu_spinor_field_copy(int par, int prec, void *s1, const void *s2) {
  if (int rc = la_check(par, prec)) return rc;
  HR_CUDA(cudaMemcpyAsync(s1, s2, spinor_bytes(par, prec), cudaMemcpyDeviceToDevice, L.stream));
  return 0;
}
int hrgpu_spinor_field_zero(int par, int prec, void *s1) {
  if (int rc = la_check(par, prec)) return rc;
  HR_CUDA(cudaMemsetAsync(s1, 0, spinor_bytes(par, prec), L.stream));
  return 0;
}
int hrgpu_spinor_field_minus(int par, int prec, void *s1, const void *s2) {
  return la_op(LA_MINUS, par, prec, s1, s2, nullptr, 0, 0, 0, 0);
}
int hrgpu_spinor_field_lc(int par, int prec, void *s1, double r1, const void *s2, double r2, const void *s3) {
  return la_op(LA_LC, par, prec, s1, s2, s3, r1, 0, r2, 0);
}
int hrgpu_spinor_field_lc_add_assign(int par, int prec, void *s1, double r1, const void *s2, double r2, const void *s3) {
  return la_op(LA_LC_ADD_ASSIGN, par, prec, s1, s2, s3, r1, 0, r2, 0);
}
int hrgpu_spinor_field_clc(int par, int prec, void *s1, double c1r, double c1i, const void *s2, double c2r, double c2i,
                           const void *s3) {
  return la_op(LA_CLC, par, prec, s1, s2, s3, c1r, c1i, c2r, c2i);
}
int hrgpu_spinor_field_clc_add_assign(int par, int prec, void *s1, double c1r, double c1i, const void *s2, double c2r,
                                      double c2i, const void *s3) {
  return la_op(LA_CLC_ADD_ASSIGN, par, prec, s1, s2, s3, c1r, c1i, c2r, c2i);
}
int hrgpu_spinor_field_g5(int par, int prec, void *s1, const void *s2) {
  return la_op(LA_G5, par, prec, s1, s2, nullptr, 0, 0, 0, 0);
}
int hrgpu_spinor_field_g5_assign(int par, int prec, void *s1) {
  return la_op(LA_G5_ASSIGN, par, prec, s1, nullptr, nullptr, 0, 0, 0, 0);
}
int hrgpu_spinor_field_g0(int par, int prec, void *s1, const void *s2) { return la_op(LA_G0, par, prec, s1, s2, nullptr, 0, 0, 0, 0); }
int hrgpu_spinor_field_g1(int par, int prec, void *s1, const void *s2) { return la_op(LA_G1, par, prec, s1, s2, nullptr, 0, 0, 0, 0); }
int hrgpu_spinor_field_g2(int par, int prec, void *s1, const void *s2) { return la_op(LA_G2, par, prec, s1, s2, nullptr, 0, 0, 0, 0); }
int hrgpu_spinor_field_g3(int par, int prec, void *s1, const void *s2) { return la_op(LA_G3, par, prec, s1, s2, nullptr, 0, 0, 0, 0); }
int hrgpu_spinor_field_lc1(int par, int prec, double c1, void *s1, const void *s2) {
  return la_op(LA_LC1, par, prec, s1, s2, nullptr, c1, 0, 0, 0);
}
int hrgpu_spinor_field_lc2(int par, int prec, double c1, double c2, void *s1, const void *s2) {
  return la_op(LA_LC2, par, prec, s1, s2, nullptr, c1, 0, c2, 0);
}
int hrgpu_spinor_field_lc3(int par, int prec, double c1, double c2, const void *s1, const void *s2, void *s3) {
  return la_op(LA_LC3, par, prec, s3, s1, s2, c1, 0, c2, 0);
}

}  // extern "C"
