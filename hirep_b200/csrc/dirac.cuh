// dirac.cuh -- internal interfaces between the operator, clover, inverter and
// force translation units.
#pragma once
#include "hop.cuh"

namespace hrgpu {

template <typename R>
int launch_hop(int ep, HopArgs<R> &a);

template <typename R>
int hop(int outp, void *out, const void *in, int ep, double cacc, const void *aux, double caux, int g5, double *red,
        const R *cdg, const typename C2<R>::T *cod, int cb0 = 0, int cb1 = -1);

int check_gauge(int prec);
template <typename R>
int eo_stage(int clover, double mass, int stage, int outp, void *out, const void *in, int g5, double *red, int cb0,
             int cb1);
template <typename R>
int Dphi_eo(double m0, void *out, const void *in, int outp, int g5, double *red);
template <typename R>
int Cphi_eo(double mass, void *out, const void *in, int g5, double *red);
int apply_op(int op, int prec, double mass, void *out, const void *in);
int apply_op_sqnorm(int op, int prec, double mass, void *out, const void *in, double *red, int *nblocks);
int op_parity(int op);
double static_mass();
void add_mvm(unsigned long n);  // hops done outside hop(), e.g. replayed CUDA graphs
unsigned long mvm_count();      // the raw hop counter (captures read and restore it)
void mvm_restore(unsigned long n);
void batch_release();           // batch.cu: workspaces and captured graphs
void qmr_release();             // qmr.cu: the g5QMR / MINRES work fields
void hmc_release();             // hmc.cu: generators, local action
int fermion_force_finish(double dt);  // force.cu: clover part of fermion_force_end

// clover: make sure the packed (4+m)+A blocks and their inverse exist for this
// mass in this precision (the LDL cache of clover_tools.c:343-358)
int clover_prepare(double mass, int prec);
template <typename R>
void clover_blocks(const R **ddg, const typename C2<R>::T **dod, const R **idg, const typename C2<R>::T **iod);
int clover_apply(int which, double mass, void *out, const void *in, int par);

// dispatch helper for kernels templated on NF and on real/complex links
#define HR_NF_DISPATCH(REAL, NF, CALL)                                                     \
  do {                                                                                     \
    if (!(REAL)) {                                                                         \
      switch (NF) {                                                                        \
        case 2: { constexpr int N_ = 2; constexpr bool R_ = false; CALL; } break;           \
        case 3: { constexpr int N_ = 3; constexpr bool R_ = false; CALL; } break;           \
        case 4: { constexpr int N_ = 4; constexpr bool R_ = false; CALL; } break;           \
        case 5: { constexpr int N_ = 5; constexpr bool R_ = false; CALL; } break;           \
        case 6: { constexpr int N_ = 6; constexpr bool R_ = false; CALL; } break;           \
        case 10: { constexpr int N_ = 10; constexpr bool R_ = false; CALL; } break;         \
        default: set_error("no kernel instantiated for complex NF=%d", (int)(NF)); return HRGPU_E_NF; \
      }                                                                                    \
    } else {                                                                               \
      switch (NF) {                                                                        \
        case 3: { constexpr int N_ = 3; constexpr bool R_ = true; CALL; } break;            \
        case 8: { constexpr int N_ = 8; constexpr bool R_ = true; CALL; } break;            \
        case 15: { constexpr int N_ = 15; constexpr bool R_ = true; CALL; } break;          \
        default: set_error("no kernel instantiated for real NF=%d", (int)(NF)); return HRGPU_E_NF; \
      }                                                                                    \
    }                                                                                      \
  } while (0)

// dispatch over every NF of the lists above, complex data (clover blocks exist
// as complex matrices for real representations too)
#define HR_NFC_DISPATCH(NF, CALL)                                                          \
  do {                                                                                     \
    switch (NF) {                                                                          \
      case 2: { constexpr int N_ = 2; CALL; } break;                                        \
      case 3: { constexpr int N_ = 3; CALL; } break;                                        \
      case 4: { constexpr int N_ = 4; CALL; } break;                                        \
      case 5: { constexpr int N_ = 5; CALL; } break;                                        \
      case 6: { constexpr int N_ = 6; CALL; } break;                                        \
      case 8: { constexpr int N_ = 8; CALL; } break;                                        \
      case 10: { constexpr int N_ = 10; CALL; } break;                                      \
      case 15: { constexpr int N_ = 15; CALL; } break;                                      \
      default: set_error("no kernel instantiated for NF=%d", (int)(NF)); return HRGPU_E_NF; \
    }                                                                                      \
  } while (0)

// device index of the neighbour of (t,x,y,z) in direction mu (dir=+1/-1)
__device__ __forceinline__ int nbr_index(const Geo &g, int t, int x, int y, int z, int mu, int dir) {
  if (mu == 0) t = (t + dir + g.T) % g.T;
  if (mu == 1) x = (x + dir + g.X) % g.X;
  if (mu == 2) y = (y + dir + g.Y) % g.Y;
  if (mu == 3) z = (z + dir + g.Z) % g.Z;
  return ((t + x + y + z) & 1) * g.ld + coords_to_cb(g, t, x, y, z);
}

__device__ __forceinline__ void dev_coords(const Geo &g, int d, int &t, int &x, int &y, int &z) {
  int p = d >= g.ld ? 1 : 0;
  cb_to_coords(g, d - p * g.ld, p, t, x, y, z);
}

// small dense complex matrices in registers/local memory (row-major N x N)
template <int N>
struct CMat {
  double2 c[N * N];
};

template <int N, bool REAL>
__device__ __forceinline__ void mload(CMat<N> &m, const void *U, int mu, long d, long lplane) {
  if (REAL) {
    const double *u = (const double *)U + (long)mu * N * N * lplane + d;
#pragma unroll (N <= 3 ? N * N : 1)
    for (int k = 0; k < N * N; k++) m.c[k] = make_double2(__ldg(u + (long)k * lplane), 0.0);
  } else {
    const double2 *u = (const double2 *)U + (long)mu * N * N * lplane + d;
#pragma unroll (N <= 3 ? N * N : 1)
    for (int k = 0; k < N * N; k++) m.c[k] = __ldg(u + (long)k * lplane);
  }
}

// C = op(A) op(B), with op = identity or dagger
template <int N> struct SmallUnroll { static constexpr int v = N <= 3 ? N : 1; };

template <int N, bool DA, bool DB>
__device__ __forceinline__ void mmul(CMat<N> &C, const CMat<N> &A, const CMat<N> &B) {
#pragma unroll (SmallUnroll<N>::v)
  for (int i = 0; i < N; i++)
#pragma unroll (SmallUnroll<N>::v)
    for (int j = 0; j < N; j++) {
      double2 s = make_double2(0.0, 0.0);
#pragma unroll (SmallUnroll<N>::v)
      for (int k = 0; k < N; k++) {
        double2 a = DA ? make_double2(A.c[k * N + i].x, -A.c[k * N + i].y) : A.c[i * N + k];
        double2 b = DB ? make_double2(B.c[j * N + k].x, -B.c[j * N + k].y) : B.c[k * N + j];
        cmac(s, a, b);
      }
      C.c[i * N + j] = s;
    }
}

template <int N>
__device__ __forceinline__ void madd(CMat<N> &A, const CMat<N> &B) {
#pragma unroll (SmallUnroll<N * N>::v)
  for (int k = 0; k < N * N; k++) A.c[k] = cadd(A.c[k], B.c[k]);
}

// Hermitian clover block b (0: s0,s1; 1: s2,s3) of the clover term in its
// device planes [4][NF*NF][2ld], plus sigma on the diagonal, element (i,j), i >= j
template <int N>
__device__ __forceinline__ double2 hblock(const double2 *cl, int b, int i, int j, long lp, long d, double sigma) {
  const int N2 = N * N;
  const double2 *sa = cl + (long)(2 * b) * N2 * lp + d, *sb = cl + (long)(2 * b + 1) * N2 * lp + d;
  double2 v;
  if (i < N) {
    v = __ldg(sa + (long)(i * N + j) * lp);
  } else if (j < N) {
    double2 s = __ldg(sb + (long)(j * N + (i - N)) * lp);
    v = make_double2(s.x, -s.y);
  } else {
    double2 s = __ldg(sa + (long)((i - N) * N + (j - N)) * lp);
    v = make_double2(-s.x, -s.y);
  }
  if (i == j) v.x += sigma;
  return v;
}

// e = exp(x) of an N x N complex matrix: scaling and squaring of the Taylor
// series to order 20 (the norm is scaled below 1/4 first), exact to rounding
template <int N>
__device__ void mexp_sq(CMat<N> &e, const CMat<N> &x) {
  double nrm = 0;
  for (int k = 0; k < N * N; k++) nrm += x.c[k].x * x.c[k].x + x.c[k].y * x.c[k].y;
  nrm = sqrt(nrm);
  int sq = 0;
  while (nrm > 0.25 && sq < 60) {
    nrm *= 0.5;
    sq++;
  }
  const double scale = ldexp(1.0, -sq);
  CMat<N> a, term, tmp;
  for (int k = 0; k < N * N; k++) {
    a.c[k] = make_double2(x.c[k].x * scale, x.c[k].y * scale);
    e.c[k] = make_double2((k % (N + 1) == 0) ? 1.0 : 0.0, 0.0);
    term.c[k] = e.c[k];
  }
  for (int j = 1; j <= 20; j++) {
    mmul<N, false, false>(tmp, term, a);
    const double inv = 1.0 / j;
    for (int k = 0; k < N * N; k++) {
      term.c[k] = make_double2(tmp.c[k].x * inv, tmp.c[k].y * inv);
      e.c[k] = cadd(e.c[k], term.c[k]);
    }
  }
  for (int q = 0; q < sq; q++) {
    mmul<N, false, false>(tmp, e, e);
    e = tmp;
  }
}

}  // namespace hrgpu
