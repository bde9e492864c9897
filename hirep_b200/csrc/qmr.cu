// qmr.cu -- g5QMR_mshift (LibHR/Inverters/g5QMR_mshift.c), MINRES
// (LibHR/Inverters/MINRES.c) and the chronological initial guess MRE
// (LibHR/Update/mre.c) on the device.
//
// The recursions are HiRep's.  g5QMR keeps every scalar on the device (alpha,
// rho, delta, beta and the Givens rotations of every shift live in a state
// struct; one-block folds update them from the partial sums of the fused
// vector kernels), so an iteration is the operator plus five kernels and the
// host reads the state once per chunk of iterations, as the CG does (cg.cu).
// MINRES and MRE keep their few scalars on the host.  These solvers are
// HiRep's choice for the non-hermitian D (force_hmc.c:122-155,
// calc_prop.c:210-289) and the fallbacks around it.
#include <math.h>
#include <string.h>

#include <complex>
#include <vector>

#include "dirac.cuh"
#include "linalg.cuh"

namespace hrgpu {

#define QTRY(x)                  \
  do {                           \
    if (int rc_ = (x)) return rc_; \
  } while (0)

// device fields for the solvers, cached between calls
struct QPool {
  std::vector<void *> f;
  size_t bytes = 0;
};
static QPool QP;

static int qpool(int n, size_t bytes) {
  if (QP.bytes != bytes) {
    for (void *p : QP.f) cudaFree(p);
    QP.f.clear();
    QP.bytes = bytes;
  }
  while ((int)QP.f.size() < n) {
    void *p = nullptr;
    HR_CUDA(cudaMalloc(&p, bytes));
    HR_CUDA(cudaMemsetAsync(p, 0, bytes, L.stream));  // padding sites stay zero
    QP.f.push_back(p);
  }
  return 0;
}

static void qmr_release_state();

void qmr_release() {
  for (void *p : QP.f) cudaFree(p);
  QP = QPool();
  qmr_release_state();
}

// small wrappers over the linear algebra (FP64, parity par)
struct QLA {
  int par;
  int sqnorm(const void *a, double *r) const { return la_dot(2, par, HRGPU_DOUBLE, a, nullptr, r); }
  int g5re(const void *a, const void *b, double *r) const {
    double v[2];
    QTRY(la_dot(1, par, HRGPU_DOUBLE, a, b, v));
    *r = v[0];
    return 0;
  }
  int prod(const void *a, const void *b, std::complex<double> *r) const {
    double v[2];
    QTRY(la_dot(0, par, HRGPU_DOUBLE, a, b, v));
    *r = std::complex<double>(v[0], v[1]);
    return 0;
  }
  int op(int o, void *s1, const void *s2 = nullptr, const void *s3 = nullptr, double c1 = 0, double c2 = 0) const {
    return la_op(o, par, HRGPU_DOUBLE, s1, s2, s3, c1, 0, c2, 0);
  }
  int mulc_add(void *s1, std::complex<double> c, const void *s2) const {
    return la_op(LA_MULC_ADD_ASSIGN, par, HRGPU_DOUBLE, s1, s2, nullptr, c.real(), c.imag(), 0, 0);
  }
};

// ---------------------------------------------------------------------------
// g5QMR_mshift_core (g5QMR_mshift.c:83-279) with the scalars on the device.
// One iteration (p1, p2, Mp the three rotating directions, q1/q2 per shift):
//   Mp = M p2 - s_0 p2                      operator + k_q_alpha (<g5 p2, Mp> partials)
//   alpha = <g5 p2, Mp> / delta              k_q_fold_alpha
//   Mp -= beta p1 + alpha p2                 k_q_p (|Mp|^2 and <g5 Mp, Mp> partials)
//   rho, the Givens step of every shift,     k_q_fold_rho (one thread, HiRep's order;
//   delta = <g5 Mp, Mp>/rho^2, beta, flags    the convergence and failure tests)
//   per shift: q_new = d (p1 - t q1 - e q2),  k_q_shift (q_new overwrites q1 in place
//   out += c2 r q_new; p2 = Mp / rho           and the two q buffers swap roles)
// ---------------------------------------------------------------------------
constexpr int QMAX = 64;
constexpr int QMR_CHUNK = 4;  // iterations launched between two reads of the state

struct QMRState {
  double alpha, beta, delta, rho, scale, innorm2, err2;
  int n, iter, max_iter, state, notconv;
  double shift[QMAX], r[QMAX], s1[QMAX], s2[QMAX], c1[QMAX], c2[QMAX];
  double t[QMAX], e[QMAX], d[QMAX], cout[QMAX];  // this iteration's coefficients per shift
  int flag[QMAX], act[QMAX], qsel[QMAX], qpar[QMAX];
};

__device__ double q_fold(const double *partials, int nblocks, int stride, int off) {
  double v = 0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v += partials[(long)b * stride + off];
  return block_sum(v);
}

__device__ __forceinline__ double q_g5(long e, int ld, int nf) {
  return ((int)((e / ld) % (4 * nf)) / nf) < 2 ? 1.0 : -1.0;
}

// Mp -= s_0 p2 (the shift of the first system, g5QMR_mshift.c:128); partials of
// <g5 p2, Mp>.  SHIFT false: s_0 = 0 (the host knows the shifts), Mp is only read.
template <bool SHIFT>
__global__ void __launch_bounds__(RED_THREADS) k_q_alpha(const QMRState *S, double2 *Mp, const double2 *p2, long n,
                                                         int ld, int nf, double *partials) {
  if (S->state != 0) return;
  const double s0 = S->shift[0];
  double acc = 0.0;
  const long stride = (long)gridDim.x * blockDim.x;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    const double2 a = p2[e];
    double2 v = Mp[e];
    if (SHIFT) {
      rmac(v, -s0, a);
      Mp[e] = v;
    }
    acc += q_g5(e, ld, nf) * (a.x * v.x + a.y * v.y);
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

__global__ void k_q_fold_alpha(QMRState *S, const double *partials, int nblocks) {
  if (S->state != 0) return;
  const double a = q_fold(partials, nblocks, 1, 0);
  if (threadIdx.x == 0) S->alpha = a / S->delta;
}

// Mp -= beta p1 + alpha p2 (g5QMR_mshift.c:131-132); partials of |Mp|^2 and <g5 Mp, Mp>
__global__ void __launch_bounds__(RED_THREADS) k_q_p(const QMRState *S, double2 *Mp, const double2 *p1,
                                                     const double2 *p2, long n, int ld, int nf, double *partials) {
  if (S->state != 0) return;
  const double beta = S->beta, alpha = S->alpha;
  double nrm = 0.0, g5n = 0.0;
  const long stride = (long)gridDim.x * blockDim.x;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    double2 v = Mp[e];
    rmac(v, -beta, p1[e]);
    rmac(v, -alpha, p2[e]);
    Mp[e] = v;
    const double q = v.x * v.x + v.y * v.y;
    nrm += q;
    g5n += q_g5(e, ld, nf) * q;
  }
  nrm = block_sum(nrm);
  g5n = block_sum(g5n);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = nrm;
    partials[2 * blockIdx.x + 1] = g5n;
  }
}

// rho, the Givens step of every shift, delta and beta, convergence (g5QMR_mshift.c:135-228)
__global__ void k_q_fold_rho(QMRState *S, const double *partials, int nblocks) {
  if (S->state != 0) return;
  const double nrm = q_fold(partials, nblocks, 2, 0);
  const double g5n = q_fold(partials, nblocks, 2, 1);
  if (threadIdx.x != 0) return;
  const int iter = ++S->iter;
  const double rho = sqrt(nrm), alpha = S->alpha;
  double beta = S->beta, maxm = 1.e-10;
  int notconv = S->notconv;
  S->rho = rho;
  for (int i = 0; i < S->n; i++) {
    S->act[i] = S->flag[i];
    if (!S->flag[i]) continue;
    const double a = alpha - S->shift[i] + S->shift[0];
    const double t = S->s1[i] * beta;
    const double e = S->c2[i] * S->c1[i] * beta + S->s2[i] * a;
    const double m = S->c2[i] * a - S->s2[i] * S->c1[i] * beta;
    S->s1[i] = S->s2[i];
    S->c1[i] = S->c2[i];
    double d, c, sn;
    if (fabs(m) < 1.e-15) {  // the plane rotation of g5QMR_mshift.c:30-37
      d = 1. / rho;
      c = 0.;
      sn = 1.;
    } else {
      const double tt = rho / m;
      c = 1. / sqrt(1. + tt * tt);
      sn = tt * c;
      d = 1. / (c * m + sn * rho);
    }
    S->c2[i] = c;
    S->s2[i] = sn;
    if (fabs(m) > maxm) maxm = fabs(m);
    S->t[i] = t;
    S->e[i] = e;
    S->d[i] = d;
    S->cout[i] = c * S->r[i];
    S->r[i] *= -sn;
    S->qsel[i] = S->qpar[i];
    S->qpar[i] ^= 1;
    if (fabs(S->r[i] * S->r[i]) * (double)(1 + iter) < S->err2 * S->innorm2) {
      S->flag[i] = 0;
      --notconv;
    }
  }
  S->scale = 0.0;
  if (fabs(rho) > 1.e-13) {
    S->scale = 1. / rho;
    const double olddelta = S->delta;
    S->delta = g5n / (rho * rho);
    if (fabs(S->delta) < 1.e-6 || maxm < 1.e-3) notconv = 0;  // the method has failed
    beta = rho * S->delta / olddelta;
  } else {
    notconv = 0;  // converged
  }
  S->beta = beta;
  S->notconv = notconv;
  if (notconv == 0 || (S->max_iter != 0 && iter >= S->max_iter)) S->state = 1;
}

// per shift: q_new = d (p1 - t q1 - e q2) into q1's buffer, out += c2 r q_new
// (g5QMR_mshift.c:152-170); then p2 = Mp / rho (:188)
__global__ void k_q_shift(const QMRState *S, double2 *const *out, double2 *const *qa, double2 *const *qb,
                          const double2 *p1, double2 *p2, long n) {
  if (S->state >= 2) return;
  const int ns = S->n;
  const double scale = S->scale;
  const long stride = (long)gridDim.x * blockDim.x;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    const double2 pv = p1[e];
    for (int i = 0; i < ns; i++) {
      if (!S->act[i]) continue;
      double2 *q1 = S->qsel[i] ? qb[i] : qa[i];
      const double2 *q2 = S->qsel[i] ? qa[i] : qb[i];
      const double d = S->d[i];
      double2 v;
      const double2 a = q1[e], b = q2[e];
      v.x = (-S->t[i] * d) * a.x;
      v.y = (-S->t[i] * d) * a.y;
      rmac(v, -S->e[i] * d, b);
      rmac(v, d, pv);
      q1[e] = v;
      double2 o = out[i][e];
      rmac(o, S->cout[i], v);
      out[i][e] = o;
    }
    if (scale != 0.0) {
      double2 v = p2[e];
      v.x *= scale;
      v.y *= scale;
      p2[e] = v;
    }
  }
}

__global__ void k_q_advance(QMRState *S) {
  if (S->state == 1) S->state = 2;
}

struct QMRWork {
  QMRState *S = nullptr, *hS = nullptr;
  void **d_ptrs = nullptr;  // out[QMAX], qa[QMAX], qb[QMAX]
};
static QMRWork QW;

static void qmr_release_state() {
  if (QW.S) cudaFree(QW.S);
  if (QW.hS) cudaFreeHost(QW.hS);
  if (QW.d_ptrs) cudaFree(QW.d_ptrs);
  QW = QMRWork();
}

// valid[i]: the true residual of shift i is below err2.  Returns the MVM count in *iters.
static int g5qmr_core(short *valid, int op, double mass, int n, const double *shift, double err2, int max_iter,
                      const void *in, void *const *out, int *iters) {
  const int par = op_parity(op);
  const QLA la{par};
  HR_REQUIRE(n >= 1 && n <= QMAX, HRGPU_E_ARG, "g5QMR: %d shifts (1..%d)", n, QMAX);
  QTRY(qpool(2 * n + 3, spinor_bytes(par, HRGPU_DOUBLE)));
  if (!QW.S) {
    HR_CUDA(cudaMalloc(&QW.S, sizeof(QMRState)));
    HR_CUDA(cudaMallocHost(&QW.hS, sizeof(QMRState)));
    HR_CUDA(cudaMalloc(&QW.d_ptrs, sizeof(void *) * 3 * QMAX));
  }
  void *P[3] = {QP.f[2 * n], QP.f[2 * n + 1], QP.f[2 * n + 2]};  // p1, p2, Mp
  int ip1 = 0, ip2 = 1, imp = 2;
  int cgiter = 0;
  double innorm2, rho, delta;
  QTRY(la.op(LA_COPY, P[ip2], in));
  QTRY(la.sqnorm(in, &innorm2));
  if (n == 1) {  // out[0] is the start vector
    QTRY(apply_op(op, HRGPU_DOUBLE, mass, P[imp], out[0]));
    QTRY(la.op(LA_MUL_ADD_ASSIGN, P[imp], out[0], nullptr, -shift[0]));
    QTRY(la.op(LA_SUB, P[ip2], P[ip2], P[imp]));
  }
  QTRY(la.sqnorm(P[ip2], &rho));
  rho = sqrt(rho);
  QTRY(la.op(LA_MUL, P[ip2], P[ip2], nullptr, 1. / rho));
  QTRY(la.op(LA_ZERO, P[ip1]));
  for (int i = 0; i < n; i++) {
    if (n != 1) QTRY(la.op(LA_ZERO, out[i]));
    QTRY(la.op(LA_ZERO, QP.f[i]));
    QTRY(la.op(LA_ZERO, QP.f[n + i]));
  }
  QTRY(la.g5re(P[ip2], P[ip2], &delta));
  HR_REQUIRE(fabs(delta) >= 1.e-28, HRGPU_E_ARG,
             "g5QMR: gamma_5 norm of the initial guess is zero, change the initial guess");
  QMRState &h = *QW.hS;
  memset(&h, 0, sizeof(QMRState));
  h.alpha = 0;
  h.beta = delta;
  h.delta = delta;
  h.innorm2 = innorm2;
  h.err2 = err2;
  h.n = n;
  h.max_iter = max_iter;
  h.notconv = n;
  for (int i = 0; i < n; i++) {
    h.shift[i] = shift[i];
    h.r[i] = rho;
    h.c1[i] = h.c2[i] = 1.;
    h.s1[i] = h.s2[i] = 0.;
    h.flag[i] = 1;
  }
  HR_CUDA(cudaMemcpyAsync(QW.S, &h, sizeof(QMRState), cudaMemcpyHostToDevice, L.stream));
  void *ptrs[3 * QMAX];
  for (int i = 0; i < n; i++) {
    ptrs[i] = out[i];
    ptrs[QMAX + i] = QP.f[i];
    ptrs[2 * QMAX + i] = QP.f[n + i];
  }
  HR_CUDA(cudaMemcpyAsync(QW.d_ptrs, ptrs, sizeof(void *) * 3 * QMAX, cudaMemcpyHostToDevice, L.stream));
  double2 *const *d_out = (double2 *const *)QW.d_ptrs;
  double2 *const *d_qa = (double2 *const *)(QW.d_ptrs + QMAX);
  double2 *const *d_qb = (double2 *const *)(QW.d_ptrs + 2 * QMAX);
  const long ne = (long)spinor_elems(par);
  long gb = (ne + RED_THREADS - 1) / RED_THREADS;
  const unsigned g = (unsigned)(gb < RED_MAX_BLOCKS ? gb : RED_MAX_BLOCKS);
  const unsigned long m0 = mvm_count();
  unsigned long per_it = 0;
  int rc = 0;
  L.cur_stop = &QW.S->state;
  for (;;) {
    for (int c = 0; c < QMR_CHUNK && !rc; c++) {
      const unsigned long mb = mvm_count();
      rc = apply_op(op, HRGPU_DOUBLE, mass, P[imp], P[ip2]);
      if (rc) break;
      per_it = mvm_count() - mb;
      if (shift[0] != 0.0)
        k_q_alpha<true><<<g, RED_THREADS, 0, L.stream>>>(QW.S, (double2 *)P[imp], (const double2 *)P[ip2], ne, L.ld,
                                                         L.nf, L.partials);
      else
        k_q_alpha<false><<<g, RED_THREADS, 0, L.stream>>>(QW.S, (double2 *)P[imp], (const double2 *)P[ip2], ne, L.ld,
                                                          L.nf, L.partials);
      k_q_fold_alpha<<<1, RED_THREADS, 0, L.stream>>>(QW.S, L.partials, g);
      k_q_p<<<g, RED_THREADS, 0, L.stream>>>(QW.S, (double2 *)P[imp], (const double2 *)P[ip1],
                                             (const double2 *)P[ip2], ne, L.ld, L.nf, L.partials);
      k_q_fold_rho<<<1, RED_THREADS, 0, L.stream>>>(QW.S, L.partials, g);
      // the three directions rotate: p1 <- p2, p2 <- Mp, Mp <- p1
      const int o1 = ip1;
      ip1 = ip2;
      ip2 = imp;
      imp = o1;
      k_q_shift<<<g, RED_THREADS, 0, L.stream>>>(QW.S, d_out, d_qa, d_qb, (const double2 *)P[ip1], (double2 *)P[ip2],
                                                 ne);
      k_q_advance<<<1, 1, 0, L.stream>>>(QW.S);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) rc = fail_cuda(e, "g5QMR iteration", __FILE__, __LINE__);
    }
    if (rc) break;
    cudaError_t e = cudaMemcpyAsync(&h, QW.S, sizeof(QMRState), cudaMemcpyDeviceToHost, L.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(L.stream);
    if (e != cudaSuccess) {
      rc = fail_cuda(e, "g5QMR state readback", __FILE__, __LINE__);
      break;
    }
    if (h.state != 0) break;
  }
  L.cur_stop = nullptr;
  if (rc) return rc;
  mvm_restore(m0 + (unsigned long)h.iter * per_it);  // the launches after convergence did nothing
  cgiter = h.iter;
  void *Mp = P[imp];
  for (int i = 0; i < n; i++) {
    QTRY(apply_op(op, HRGPU_DOUBLE, mass, Mp, out[i]));
    ++cgiter;
    if (shift[i] != 0.) QTRY(la.op(LA_MUL_ADD_ASSIGN, Mp, out[i], nullptr, -shift[i]));
    QTRY(la.op(LA_SUB, Mp, Mp, in));
    double nr;
    QTRY(la.sqnorm(Mp, &nr));
    valid[i] = (fabs(nr / innorm2) > err2) ? 0 : 1;
  }
  if (n == 1) ++cgiter;
  *iters = cgiter;
  return 0;
}

// MINRES_core (MINRES.c:24-158) on the hermitian operator g5^g5f (op - sh)
struct Herm {
  int op, g5;
  double mass, sh;
  int apply(void *out, const void *in) const {
    const QLA la{op_parity(op)};
    QTRY(apply_op(op, HRGPU_DOUBLE, mass, out, in));
    if (sh != 0.) QTRY(la.op(LA_MUL_ADD_ASSIGN, out, in, nullptr, -sh));
    if (g5) QTRY(la.op(LA_G5_ASSIGN, out));
    return 0;
  }
};

static int minres_core(short *valid, const Herm &H, double err2, int max_iter, const void *in, void *out,
                       const void *trial, int *iters) {
  const int par = op_parity(H.op);
  const QLA la{par};
  // QP.f[0..4] (the g5QMR fallback keeps its shift pool alive only between calls)
  QTRY(qpool(5, spinor_bytes(par, HRGPU_DOUBLE)));
  void *q1 = QP.f[0], *q2 = QP.f[1], *p1 = QP.f[2], *p2 = QP.f[3], *Mp = QP.f[4], *tmp;
  int cgiter = 0, notconverged = 1;
  QTRY(la.op(LA_COPY, p2, in));
  if (trial) {
    QTRY(H.apply(p1, trial));
    ++cgiter;
    QTRY(la.op(LA_SUB_ASSIGN, p2, p1));
    if (out != trial) QTRY(la.op(LA_COPY, out, trial));
  } else {
    QTRY(la.op(LA_ZERO, out));
  }
  double innorm2, beta;
  QTRY(la.sqnorm(in, &innorm2));
  QTRY(la.sqnorm(p2, &beta));
  beta = sqrt(beta);
  QTRY(la.op(LA_MUL, p2, p2, nullptr, 1. / beta));
  QTRY(la.op(LA_ZERO, p1));
  double r = beta, rho2 = beta, rho1 = 1., c2 = -1., rp = 0., s1 = 0., s2 = 0., c1 = 0.;
  QTRY(la.op(LA_ZERO, q1));
  QTRY(la.op(LA_ZERO, q2));
  do {
    ++cgiter;
    QTRY(H.apply(Mp, p2));
    double alpha;
    std::complex<double> z;
    QTRY(la.prod(Mp, p2, &z));
    alpha = z.real();
    QTRY(la.op(LA_MUL_ADD_ASSIGN, Mp, p1, nullptr, -beta));
    QTRY(la.op(LA_MUL_ADD_ASSIGN, Mp, p2, nullptr, -alpha));
    tmp = p1; p1 = p2; p2 = Mp; Mp = tmp;
    const double oldbeta = beta;
    QTRY(la.sqnorm(p2, &beta));
    beta = sqrt(beta);
    QTRY(la.op(LA_MUL, p2, p2, nullptr, 1. / beta));
    const double d = (alpha - rp * c1) * s2;
    const double h = oldbeta * s1;
    rp = -oldbeta * c1 * s2 - alpha * c2;
    const double k = sqrt(rp * rp + beta * beta);
    c1 = c2;
    c2 = rp / k;
    s1 = s2;
    s2 = beta / k;
    QTRY(la.op(LA_LC, Mp, q1, q2, -h / rho1, -d / rho2));
    tmp = q1; q1 = q2; q2 = tmp;
    QTRY(la.op(LA_ADD, q2, p1, Mp));
    rho1 = rho2;
    rho2 = k;
    QTRY(la.op(LA_MUL_ADD_ASSIGN, out, q2, nullptr, r * c2 / k));
    r *= s2;
    if (r * r < err2 * innorm2) notconverged = 0;
  } while ((max_iter == 0 || cgiter < max_iter) && notconverged);
  QTRY(H.apply(Mp, out));
  ++cgiter;
  QTRY(la.op(LA_SUB, Mp, Mp, in));
  double nr;
  QTRY(la.sqnorm(Mp, &nr));
  *valid = (fabs(nr / innorm2) > err2) ? 0 : 1;
  *iters = cgiter;
  return 0;
}

// MINRES (MINRES.c:160-172): repeated from the last solution until valid; bounded
static int minres(const Herm &H, double err2, int max_iter, const void *in, void *out, const void *trial, int *iters) {
  short valid = 0;
  int it = 0, total = 0, rep = 0;
  QTRY(minres_core(&valid, H, err2, max_iter, in, out, trial, &it));
  total = it;
  while (!valid && (max_iter == 0 || total < max_iter)) {
    if (++rep > 100) {
      *iters = total;
      set_error("MINRES: err2=%g not reached after %d restarts", err2, rep - 1);
      return HRGPU_E_NOCONV;
    }
    QTRY(minres_core(&valid, H, err2, max_iter, in, out, out, &it));
    total += it;
  }
  *iters = total;
  if (!valid) {
    set_error("MINRES: err2=%g not reached in %d iterations", err2, total);
    return HRGPU_E_NOCONV;
  }
  return 0;
}

static bool qmr_op_ok(int op) {
  return op == HRGPU_OP_DPHI_EOPRE || op == HRGPU_OP_CPHI_EOPRE || op == HRGPU_OP_DPHI || op == HRGPU_OP_CPHI;
}
static bool herm_op_ok(int op) {
  return op == HRGPU_OP_G5DPHI_EOPRE || op == HRGPU_OP_G5CPHI_EOPRE || op == HRGPU_OP_G5DPHI_EOPRE_SQ ||
         op == HRGPU_OP_G5CPHI_EOPRE_SQ || op == HRGPU_OP_G5DPHI_SQ || op == HRGPU_OP_G5CPHI_SQ;
}

// ---------------------------------------------------------------------------
// MRE (mre.c): the last `max` solutions of a sequence of solves, newest first
// ---------------------------------------------------------------------------
struct MRE {
  int max = 0, par = 0, num[2] = {0, 0};
  std::vector<void *> s[2];  // s[p][0] is the newest
  std::vector<void *> v;     // Gram-Schmidt basis (max) + D v (1)
};

// in-place LU with partial pivoting and the solution of A x = conj(b) (mre.c:56-143)
static int mre_lu_solve(int max, std::vector<std::complex<double>> &A, const std::vector<std::complex<double>> &b,
                        std::vector<std::complex<double>> &x) {
  typedef std::complex<double> C;
  std::vector<int> mutate(max);
  std::vector<C> y(max);
  for (int i = 0; i < max; i++) mutate[i] = i;
  auto a = [&](int i, int j) -> C & { return A[(size_t)i * max + j]; };
  for (int i = 0; i < max; i++) {
    for (int j = 0; j <= i; j++)
      for (int k = 0; k < j; k++) a(j, i) -= a(j, k) * a(k, i);
    double big = std::abs(a(i, i));
    int row = i;
    for (int j = i + 1; j < max; j++) {
      for (int k = 0; k < i; k++) a(j, i) -= a(j, k) * a(k, i);
      if (std::abs(a(j, i)) > big) {
        big = std::abs(a(j, i));
        row = j;
      }
    }
    if (big < 1.0e-14) return -1;  // singular: no guess
    if (row != i) {
      for (int k = 0; k < max; k++) std::swap(a(row, k), a(i, k));
      std::swap(mutate[row], mutate[i]);
    }
    for (int k = i + 1; k < max; k++) a(k, i) = a(k, i) / a(i, i);
  }
  for (int i = 0; i < max; i++) {
    y[i] = std::conj(b[mutate[i]]);
    for (int k = 0; k < i; k++) y[i] -= a(i, k) * y[k];
  }
  x.assign(max, C(0, 0));
  for (int i = max - 1; i >= 0; i--) {
    x[i] = y[i];
    for (int k = i + 1; k < max; k++) x[i] -= a(i, k) * x[k];
    x[i] = x[i] / a(i, i);
  }
  return 0;
}

}  // namespace hrgpu

using namespace hrgpu;

extern "C" {

int hrgpu_g5QMR_mshift(int op, double mass, int n, const double *shift, double err2, int max_iter, const void *in,
                       void *const *out, int *iters) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "g5QMR_mshift: lattice not initialised");
  HR_REQUIRE(qmr_op_ok(op), HRGPU_E_ARG, "g5QMR_mshift: operator %d is not a Dirac operator D (Dphi_eopre, Cphi_eopre, Dphi, Cphi)", op);
  HR_REQUIRE(n > 0 && n <= 64, HRGPU_E_ARG, "g5QMR_mshift: n = %d shifts (1..64 supported)", n);
  HR_REQUIRE(shift && in && out && iters, HRGPU_E_ARG, "g5QMR_mshift: NULL argument");
  for (int i = 0; i < n; i++) HR_REQUIRE(out[i] && out[i] != in, HRGPU_E_ARG, "g5QMR_mshift: bad output field %d", i);
  QTRY(check_gauge(HRGPU_DOUBLE));
  std::vector<short> valid(n, 0);
  int total = 0, it = 0;
  QTRY(g5qmr_core(valid.data(), op, mass, n, shift, err2, max_iter, in, out, &it));
  total = it;
  // unconverged shifts: again one at a time from their current solution, then
  // MINRES on g5 (D - shift) with g5 in (g5QMR_mshift.c:495-533)
  int status = 0;
  for (int i = 0; i < n; i++) {
    if (valid[i]) continue;
    void *o[1] = {out[i]};
    QTRY(g5qmr_core(&valid[i], op, mass, 1, shift + i, err2, 0, in, o, &it));
    total += it;
    if (!valid[i]) {
      const int par = op_parity(op);
      QTRY(qpool(6, spinor_bytes(par, HRGPU_DOUBLE)));
      void *g5in = QP.f[5];
      QTRY(la_op(LA_G5, par, HRGPU_DOUBLE, g5in, in, nullptr, 0, 0, 0, 0));
      Herm H{op, 1, mass, shift[i]};
      int rc = minres(H, err2, 0, g5in, out[i], out[i == 0 ? 0 : i - 1], &it);
      total += it;
      if (rc == HRGPU_E_NOCONV) status = rc;
      else if (rc) return rc;
    }
  }
  *iters = total;
  return status;
}

int hrgpu_MINRES(int op, double mass, double err2, int max_iter, const void *in, void *out, const void *trial,
                 int *iters) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "MINRES: lattice not initialised");
  HR_REQUIRE(herm_op_ok(op), HRGPU_E_ARG, "MINRES: operator %d is not hermitian", op);
  HR_REQUIRE(in && out && iters && out != in, HRGPU_E_ARG, "MINRES: bad arguments");
  QTRY(check_gauge(HRGPU_DOUBLE));
  Herm H{op, 0, mass, 0.0};
  return minres(H, err2, max_iter, in, out, trial, iters);
}

void *hrgpu_mre_init(int max, int par) {
  if (!L.ready || max <= 0 || par < 0 || par > 2) {
    set_error("mre_init: bad arguments (max = %d, par = %d) or lattice not initialised", max, par);
    return nullptr;
  }
  MRE *m = new MRE();
  m->max = max < 15 ? max : 15;  // mre.c:15 (MAX)
  m->par = par;
  const size_t bytes = spinor_bytes(par, HRGPU_DOUBLE);
  for (int p = 0; p < 2; p++)
    for (int i = 0; i < m->max; i++) {
      void *f = nullptr;
      if (cudaMalloc(&f, bytes) != cudaSuccess || cudaMemset(f, 0, bytes) != cudaSuccess) {
        set_error("mre_init: cudaMalloc of %zu bytes failed", bytes);
        for (int q = 0; q < 2; q++)
          for (void *g : m->s[q]) cudaFree(g);
        if (f) cudaFree(f);
        delete m;
        return nullptr;
      }
      m->s[p].push_back(f);
    }
  for (int i = 0; i < m->max + 1; i++) {
    void *f = nullptr;
    if (cudaMalloc(&f, bytes) != cudaSuccess || cudaMemset(f, 0, bytes) != cudaSuccess) {
      set_error("mre_init: cudaMalloc of %zu bytes failed", bytes);
      for (int q = 0; q < 2; q++)
        for (void *g : m->s[q]) cudaFree(g);
      for (void *g : m->v) cudaFree(g);
      if (f) cudaFree(f);
      delete m;
      return nullptr;
    }
    m->v.push_back(f);
  }
  return m;
}

int hrgpu_mre_free(void *mre) {
  MRE *m = (MRE *)mre;
  if (!m) return 0;
  for (int p = 0; p < 2; p++)
    for (void *f : m->s[p]) cudaFree(f);
  for (void *f : m->v) cudaFree(f);
  delete m;
  return 0;
}

// mre_store (mre.c:202-228): the newest solution goes to slot 0
int hrgpu_mre_store(void *mre, int p, const void *in) {
  MRE *m = (MRE *)mre;
  HR_REQUIRE(m && in && (p == 0 || p == 1), HRGPU_E_ARG, "mre_store: bad arguments (p = %d)", p);
  void *last = m->s[p][m->max - 1];
  for (int i = m->max - 1; i > 0; i--) m->s[p][i] = m->s[p][i - 1];
  m->s[p][0] = last;
  QTRY(la_op(LA_COPY, m->par, HRGPU_DOUBLE, last, in, nullptr, 0, 0, 0, 0));
  m->num[p]++;
  return 0;
}

// mre_guess (mre.c:230-268): out = sum_i x_i v_i, v the Gram-Schmidt basis of the
// stored solutions, A[j][i] = <DD v_i, v_j>, b_i = <v_i, pf>, A x = conj(b)
int hrgpu_mre_guess(void *mre, int p, void *out, int op, double mass, const void *pf) {
  MRE *m = (MRE *)mre;
  HR_REQUIRE(m && out && pf && (p == 0 || p == 1), HRGPU_E_ARG, "mre_guess: bad arguments (p = %d)", p);
  HR_REQUIRE(op_parity(op) == m->par, HRGPU_E_ARG, "mre_guess: operator %d acts on another parity", op);
  const QLA la{m->par};
  QTRY(la.op(LA_ZERO, out));
  const int max = m->num[p] > m->max ? m->max : m->num[p];
  if (max == 0) return 0;
  typedef std::complex<double> C;
  for (int i = 0; i < max; i++) QTRY(la.op(LA_COPY, m->v[i], m->s[p][i]));
  for (int i = 0; i < max; i++) {  // gram_schmidt (mre.c:30-48)
    double rii;
    QTRY(la.sqnorm(m->v[i], &rii));
    QTRY(la.op(LA_MUL, m->v[i], m->v[i], nullptr, 1.0 / sqrt(rii)));
    for (int j = i + 1; j < max; j++) {
      C rij;
      QTRY(la.prod(m->v[i], m->v[j], &rij));
      QTRY(la.mulc_add(m->v[j], -rij, m->v[i]));
    }
  }
  std::vector<C> A((size_t)max * max), b(max), x;
  void *Dv = m->v[m->max];
  for (int i = 0; i < max; i++) {
    QTRY(apply_op(op, HRGPU_DOUBLE, mass, Dv, m->v[i]));
    for (int j = 0; j < max; j++) QTRY(la.prod(Dv, m->v[j], &A[(size_t)j * max + i]));
    QTRY(la.prod(m->v[i], pf, &b[i]));
  }
  if (mre_lu_solve(max, A, b, x) != 0) return 0;  // singular: out stays zero, as in the reference
  for (int i = 0; i < max; i++) QTRY(la.mulc_add(out, x[i], m->v[i]));
  return 0;
}

}  // extern "C"
