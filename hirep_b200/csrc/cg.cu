// cg.cu -- multi-shift CG on the device (LibHR/Inverters/cg_mshift.c) and its
// mixed-precision defect-correction driver (LibHR/Inverters/cg_mshift_flt.c).
//
// The recursion is HiRep's, term for term, but every scalar (alpha, omega,
// gamma, delta and the per-shift z1/z2/z3 and flags) lives in device memory and
// is updated by one-block "fold" kernels, so an iteration never waits for the
// host.  One iteration is
//   M k (the fused hopping kernels) -> <k,Mk> partials -> fold_alpha ->
//   update1 (x_i += c_i p_i, r += omega Mk, |r|^2 partials) -> fold_lambda ->
//   update2 (k = gamma k + r, p_i = d_i p_i + z3_i r) -> advance
// The host launches several iterations at a time (a captured CUDA graph) and
// reads one state word between chunks.  When fold_lambda finds the stopping condition it marks the
// state; the remaining kernels of that iteration finish it exactly as HiRep's
// loop body would, and every kernel of later iterations returns at once, so the
// solution and the iteration count are those of HiRep's loop.
#include <vector>

#include "dirac.cuh"
#include "linalg.cuh"

namespace hrgpu {

constexpr int MAXS = 64;
constexpr int CG_CHUNK = 4;
constexpr int CG_HARD_LIMIT = 200000;  // iterations, when the caller sets no max_iter

struct CGState {
  double omega, oldomega, gamma, alpha, lambda, delta, innorm2, err2;
  int n, state, iter, max_iter, notconv, flt;
  double shift[MAXS], z1[MAXS], z2[MAXS], z3[MAXS], cx[MAXS], cp[MAXS];
  int flag[MAXS];
};

__device__ double fold_partials(const double *partials, int nblocks, int stride, int off) {
  double s = 0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partials[(long)b * stride + off];
  return block_sum(s);
}

// alpha = <k, Mk>; omega = -delta/alpha; z3 and the solution coefficients (cg_mshift.c:82-91)
__global__ void k_cg_fold_alpha(CGState *S, const double *partials, int nblocks, int stride) {
  if (S->state != 0) return;
  double alpha = fold_partials(partials, nblocks, stride, 0);
  if (threadIdx.x == 0) {
    S->alpha = alpha;
    if (!isfinite(alpha) || alpha == 0.0) {  // breakdown (non-positive operator or NaN input)
      S->state = 3;
      return;
    }
    S->oldomega = S->omega;
    S->omega = -S->delta / alpha;
    double omega = S->omega, oldomega = S->oldomega, gamma = S->gamma;
    for (int i = 0; i < S->n; i++) {
      if (S->flag[i]) {
        double z1 = S->z1[i], z2 = S->z2[i];
        double z3 = oldomega * z1 * z2 / (omega * gamma * (z1 - z2) + z1 * oldomega * (1. + S->shift[i] * omega));
        S->z3[i] = z3;
        S->cx[i] = -omega * z3 / z2;
      } else {
        S->cx[i] = 0.0;
      }
    }
  }
}

// lambda = |r|^2, gamma, convergence flags (cg_mshift.c:92-111; cg_mshift_flt.c:96-118)
__global__ void k_cg_fold_lambda(CGState *S, const double *partials, int nblocks) {
  if (S->state != 0) return;
  double lambda = fold_partials(partials, nblocks, 1, 0);
  if (threadIdx.x == 0) {
    S->lambda = lambda;
    S->gamma = lambda / S->delta;
    S->delta = lambda;
    double gamma = S->gamma, delta = S->delta;
    int notconv = 0;
    for (int i = 0; i < S->n; i++) {
      double z3 = S->z3[i];
      if (S->flt) {
        if (delta * z3 * z3 > S->err2 * S->innorm2) ++notconv;
      } else {
        if (delta * z3 * z3 < S->err2 * S->innorm2) S->flag[i] = 0;
        if (S->flag[i]) ++notconv;
      }
      if (S->flag[i]) {
        double z2 = S->z2[i];
        S->cp[i] = gamma * z3 * z3 / (z2 * z2);
        S->z1[i] = S->z2[i];
        S->z2[i] = z3;
      }
    }
    S->notconv = notconv;
    S->iter++;
    if (!isfinite(lambda)) S->state = 3;
    else if (notconv == 0 || (S->max_iter != 0 && S->iter >= S->max_iter)) S->state = 1;
  }
}

__global__ void k_cg_advance(CGState *S) {
  if (S->state == 1) S->state = 2;
}

template <typename V>
__global__ void __launch_bounds__(RED_THREADS) k_cg_update1(CGState *S, V *const *x, V *const *p, V *r, const V *Mk,
                                                            long n, double *partials) {
  if (S->state != 0) return;
  const double omega = S->omega;
  const int ns = S->n;
  double nrm = 0.0;
  long stride = (long)gridDim.x * blockDim.x;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    for (int i = 0; i < ns; i++) {
      if (!S->flag[i]) continue;
      V xv = x[i][e];
      rmac(xv, (decltype(xv.x))S->cx[i], p[i][e]);
      x[i][e] = xv;
    }
    V rv = r[e];
    rmac(rv, (decltype(rv.x))omega, Mk[e]);
    r[e] = rv;
    nrm += (double)rv.x * rv.x + (double)rv.y * rv.y;
  }
  nrm = block_sum(nrm);
  if (threadIdx.x == 0) partials[blockIdx.x] = nrm;
}

template <typename V>
__global__ void k_cg_update2(CGState *S, V *const *p, V *k, const V *r, long n) {
  if (S->state >= 2) return;
  typedef decltype(k[0].x) R;
  const R gamma = (R)S->gamma;
  const int ns = S->n;
  long stride = (long)gridDim.x * blockDim.x;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    V rv = r[e];
    V kv = k[e];
    kv.x = gamma * kv.x + rv.x;
    kv.y = gamma * kv.y + rv.y;
    k[e] = kv;
    for (int i = 0; i < ns; i++) {
      if (!S->flag[i]) continue;
      V pv = p[i][e];
      R cp = (R)S->cp[i], z3 = (R)S->z3[i];
      pv.x = cp * pv.x;
      pv.y = cp * pv.y;
      rmac(pv, z3, rv);
      p[i][e] = pv;
    }
  }
}

// <k, Mk> partials (re, im per block) for the fold; stops with the state
template <typename V>
__global__ void __launch_bounds__(RED_THREADS) k_cg_dot(const CGState *S, const V *a, const V *b, long n, double *partials) {
  if (S->state != 0) return;
  double re = 0.0;
  long stride = (long)gridDim.x * blockDim.x;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    V u = a[e], v = b[e];
    re += (double)u.x * v.x + (double)u.y * v.y;
  }
  re = block_sum(re);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = re;
    partials[2 * blockIdx.x + 1] = 0.0;
  }
}

// ---------------------------------------------------------------------------
// workspace (cached between calls, grown on demand)
// ---------------------------------------------------------------------------
struct CGWork {
  std::vector<void *> bufs;  // p[0..n-1], k, r, Mk
  size_t bytes = 0;
  CGState *S = nullptr;
  CGState *hS = nullptr;  // pinned host copy
  void **d_ptrs = nullptr;  // device arrays of pointers: x[MAXS], p[MAXS]
};
static CGWork W[2];  // [prec]

// work fields of the defect-correction driver: FP64 res, res2, tmp; FP32 res_flt, out_flt[n]
struct FltWork {
  void *dres = nullptr, *dres2 = nullptr, *dtmp = nullptr;
  std::vector<void *> fbuf;
  size_t bd = 0, bf = 0;
};
static FltWork FW;

static int cg_workspace(int prec, int nvec, size_t bytes) {
  CGWork &w = W[prec];
  if (w.bytes != bytes) {
    for (void *b : w.bufs) cudaFree(b);
    w.bufs.clear();
    w.bytes = bytes;
  }
  while ((int)w.bufs.size() < nvec) {
    void *b = nullptr;
    HR_CUDA(cudaMalloc(&b, bytes));
    w.bufs.push_back(b);
  }
  if (!w.S) {
    HR_CUDA(cudaMalloc(&w.S, sizeof(CGState)));
    HR_CUDA(cudaMallocHost(&w.hS, sizeof(CGState)));
    HR_CUDA(cudaMalloc(&w.d_ptrs, sizeof(void *) * 2 * MAXS));
  }
  return 0;
}

// The chunk of iterations as a CUDA graph, captured once per (operator, mass,
// work buffers, kernel variants, link storage) and replayed: ten launches per
// iteration, most of them small, cost more in launch gaps than in work.  The
// graph reads the links and clover blocks at replay; the clover blocks (for
// this mass) and the BF16 link copy are brought up to date before each replay.
// (Folding the partials in the last block of the kernel that wrote them, with
// an atomic ticket, instead of one-block fold kernels was measured slower: the
// per-block fence outweighs the launches it saves inside a graph.)
struct CGGraph {
  int op = -1;
  double mass = 0;
  const void *ptrs[10] = {};
  int v[3] = {-1, -1, -1}, force = -1, flt_links = -1, pdl = -1;
  unsigned long mvm = 0;  // hop launches in one replay (the MVM counter)
  cudaGraphExec_t exec = nullptr;
};
static CGGraph CGG[2];  // [prec]
static cudaStream_t cg_cap = nullptr;

static void drop_cg_graph(CGGraph &c) {
  if (c.exec) cudaGraphExecDestroy(c.exec);
  c = CGGraph();
}

void cg_release() {
  batch_release();
  qmr_release();
  hmc_release();
  hostop_release();
  cudaFree(FW.dres); cudaFree(FW.dres2); cudaFree(FW.dtmp);
  for (void *b : FW.fbuf) cudaFree(b);
  FW = FltWork();
  for (int q = 0; q < 2; q++) drop_cg_graph(CGG[q]);
  if (cg_cap) cudaStreamDestroy(cg_cap);
  cg_cap = nullptr;
  for (int q = 0; q < 2; q++) {
    for (void *b : W[q].bufs) cudaFree(b);
    W[q].bufs.clear();
    W[q].bytes = 0;
    if (W[q].S) cudaFree(W[q].S);
    if (W[q].hS) cudaFreeHost(W[q].hS);
    if (W[q].d_ptrs) cudaFree(W[q].d_ptrs);
    W[q].S = nullptr;
    W[q].hS = nullptr;
    W[q].d_ptrs = nullptr;
  }
}

static unsigned red_grid(long n) {
  long b = (n + RED_THREADS - 1) / RED_THREADS;
  return (unsigned)(b < RED_MAX_BLOCKS ? b : RED_MAX_BLOCKS);
}

// CG_CHUNK iterations, launched one kernel at a time
template <typename R>
static int cg_iterations(int op, int prec, double mass, CGWork &w, void *k, void *r, void *Mk, long ne, unsigned g) {
  typedef typename C2<R>::T V;
  V *const *dx = (V *const *)w.d_ptrs;
  V *const *dp = (V *const *)(w.d_ptrs + MAXS);
  for (int c = 0; c < CG_CHUNK; c++) {
    // alpha = <k, H^2 k> = |H k|^2 from the first H's partials where the
    // operator is the even-odd H^2, else from a dot-product pass
    int nb = 0;
    const int rc = apply_op_sqnorm(op, prec, mass, Mk, k, L.partials, &nb);
    if (rc > 0) return rc;
    if (rc == 0) {
      k_cg_fold_alpha<<<1, RED_THREADS, 0, L.stream>>>(w.S, L.partials, nb, 1);
    } else {
      if (int q = apply_op(op, prec, mass, Mk, k)) return q;
      k_cg_dot<V><<<g, RED_THREADS, 0, L.stream>>>(w.S, (const V *)k, (const V *)Mk, ne, L.partials);
      k_cg_fold_alpha<<<1, RED_THREADS, 0, L.stream>>>(w.S, L.partials, g, 2);
    }
    k_cg_update1<V><<<g, RED_THREADS, 0, L.stream>>>(w.S, dx, dp, (V *)r, (const V *)Mk, ne, L.partials);
    k_cg_fold_lambda<<<1, RED_THREADS, 0, L.stream>>>(w.S, L.partials, g);
    k_cg_update2<V><<<g, RED_THREADS, 0, L.stream>>>(w.S, dp, (V *)k, (const V *)r, ne);
    k_cg_advance<<<1, 1, 0, L.stream>>>(w.S);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "cg iteration", __FILE__, __LINE__);
  }
  return 0;
}
static bool op_is_clover(int op) {
  return op == HRGPU_OP_G5CPHI_EOPRE_SQ || op == HRGPU_OP_G5CPHI_SQ || op == HRGPU_OP_CPHI_EOPRE ||
         op == HRGPU_OP_G5CPHI_EOPRE || op == HRGPU_OP_CPHI;
}
template <typename R>
static int cg_chunk(int op, int prec, double mass, CGWork &w, void *k, void *r, void *Mk, long ne, unsigned g) {
  if (op_is_clover(op))
    if (int rc = clover_prepare(mass, prec)) return rc;
  if (prec == HRGPU_FLOAT && L.flt_links == HRGPU_LINKS_BF16)
    if (int rc = ensure_links_bf16()) return rc;
  const int pi = prec == HRGPU_DOUBLE ? 0 : (L.flt_links == HRGPU_LINKS_BF16 ? 2 : 1);
  const bool clover = op_is_clover(op);
  const bool settled = L.hop_force >= 0 || (clover ? (L.hop_variant[pi][EP_CLOV] >= 0 &&
                                                      (op == HRGPU_OP_G5CPHI_SQ || op == HRGPU_OP_CPHI ||
                                                       L.hop_variant[pi][EP_CLOV_INV] >= 0))
                                                   : L.hop_variant[pi][EP_AXPY] >= 0);
  if (!settled) return cg_iterations<R>(op, prec, mass, w, k, r, Mk, ne, g);  // tunes the hopping kernels
  const void *links = prec == HRGPU_DOUBLE ? (const void *)L.U
                                           : (L.flt_links == HRGPU_LINKS_BF16 ? (const void *)L.Ubf : (const void *)L.Uf);
  const void *ptrs[10] = {k, r, Mk, w.S, w.d_ptrs, L.partials, links, L.cur_stop,
                          prec == HRGPU_DOUBLE ? L.tmp_e : L.tmp_e_f, prec == HRGPU_DOUBLE ? L.tmp_o : L.tmp_o_f};
  CGGraph &c = CGG[prec];
  bool same = c.exec && c.op == op && c.mass == mass && c.force == L.hop_force && c.flt_links == L.flt_links &&
              c.pdl == (int)L.hop_pdl;
  for (int i = 0; i < 3 && same; i++) same = c.v[i] == L.hop_variant[pi][i];
  for (int i = 0; i < 10 && same; i++) same = c.ptrs[i] == ptrs[i];
  if (!same) {
    drop_cg_graph(c);
    if (!cg_cap) HR_CUDA(cudaStreamCreateWithFlags(&cg_cap, cudaStreamNonBlocking));
    const unsigned long m0 = mvm_count();
    cudaGraph_t graph = nullptr;
    cudaStream_t saved = L.stream;
    HR_CUDA(cudaStreamBeginCapture(cg_cap, cudaStreamCaptureModeRelaxed));
    L.stream = cg_cap;
    int rc = cg_iterations<R>(op, prec, mass, w, k, r, Mk, ne, g);
    L.stream = saved;
    cudaError_t e = cudaStreamEndCapture(cg_cap, &graph);
    const unsigned long dm = mvm_count() - m0;
    mvm_restore(m0);  // nothing ran yet
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (e != cudaSuccess) return fail_cuda(e, "cg capture", __FILE__, __LINE__);
    e = cudaGraphInstantiate(&c.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      c.exec = nullptr;
      return fail_cuda(e, "cg graph instantiate", __FILE__, __LINE__);
    }
    c.op = op;
    c.mass = mass;
    c.force = L.hop_force;
    c.flt_links = L.flt_links;
    c.pdl = (int)L.hop_pdl;
    for (int i = 0; i < 3; i++) c.v[i] = L.hop_variant[pi][i];
    for (int i = 0; i < 10; i++) c.ptrs[i] = ptrs[i];
    c.mvm = dm;
  }
  HR_CUDA(cudaGraphLaunch(c.exec, L.stream));
  add_mvm(c.mvm);
  return 0;
}

// cg_mshift_core (cg_mshift.c:24-145) / cg_mshift_flt_core (cg_mshift_flt.c:22-140).
// out[i] are fields of precision `prec`; flags[i] in/out (flt: read only).
// Returns the iteration count, or a negative status.
template <typename R>
static int cg_core(int op, double mass, int n, const double *shift, double err2, int max_iter, const void *in,
                   void *const *out, int *flags, int flt, int *iters) {
  typedef typename C2<R>::T V;
  const int prec = sizeof(R) == 8 ? HRGPU_DOUBLE : HRGPU_FLOAT;
  const int par = op_parity(op);
  const size_t bytes = spinor_bytes(par, prec);
  const long ne = (long)spinor_elems(par);
  if (int rc = cg_workspace(prec, n + 3, bytes)) return rc;
  CGWork &w = W[prec];
  void *k = w.bufs[n], *r = w.bufs[n + 1], *Mk = w.bufs[n + 2];
  int cgiter = 0;
  double innorm2;
  if (int rc = la_dot(2, par, prec, in, nullptr, &innorm2)) return rc;
  if (!isfinite(innorm2)) {
    *iters = 0;
    set_error("cg_mshift: the source norm is not finite (%g)", innorm2);
    return HRGPU_E_BREAKDOWN;
  }
  if (innorm2 == 0.0) {  // (M - s_i) x = 0: every solution is zero, nothing to iterate
    for (int i = 0; i < n; i++) HR_CUDA(cudaMemsetAsync(out[i], 0, bytes, L.stream));
    *iters = 0;
    return 0;
  }
  if (n == 1) {
    // out[0] is the initial guess
    if (int rc = apply_op(op, prec, mass, Mk, out[0])) return rc;
    ++cgiter;
    if (int rc = la_op(LA_MUL_ADD_ASSIGN, par, prec, Mk, out[0], nullptr, -shift[0], 0, 0, 0)) return rc;
    if (int rc = la_op(LA_SUB, par, prec, r, in, Mk, 0, 0, 0, 0)) return rc;
  } else {
    HR_CUDA(cudaMemcpyAsync(r, in, bytes, cudaMemcpyDeviceToDevice, L.stream));
  }
  HR_CUDA(cudaMemcpyAsync(k, r, bytes, cudaMemcpyDeviceToDevice, L.stream));
  double delta;
  if (int rc = la_dot(2, par, prec, r, nullptr, &delta)) return rc;
  for (int i = 0; i < n; i++) {
    HR_CUDA(cudaMemcpyAsync(w.bufs[i], r, bytes, cudaMemcpyDeviceToDevice, L.stream));
    if (n != 1) HR_CUDA(cudaMemsetAsync(out[i], 0, bytes, L.stream));
  }
  CGState &h = *w.hS;
  memset(&h, 0, sizeof(CGState));
  h.omega = 1.0;
  h.gamma = 0.0;
  h.delta = delta;
  h.innorm2 = innorm2;
  h.err2 = err2;
  h.n = n;
  h.state = 0;
  h.iter = 0;
  h.max_iter = max_iter == 0 ? CG_HARD_LIMIT : (max_iter > cgiter ? max_iter - cgiter : 1);
  h.flt = flt;
  for (int i = 0; i < n; i++) {
    h.shift[i] = shift[i];
    h.z1[i] = h.z2[i] = 1.0;
    h.z3[i] = 0.0;
    h.flag[i] = flt ? flags[i] : 1;
  }
  HR_CUDA(cudaMemcpyAsync(w.S, &h, sizeof(CGState), cudaMemcpyHostToDevice, L.stream));
  void *ptrs[2 * MAXS];
  for (int i = 0; i < n; i++) {
    ptrs[i] = out[i];
    ptrs[MAXS + i] = w.bufs[i];
  }
  HR_CUDA(cudaMemcpyAsync(w.d_ptrs, ptrs, sizeof(void *) * 2 * MAXS, cudaMemcpyHostToDevice, L.stream));
  const unsigned g = red_grid(ne);
  L.cur_stop = &w.S->state;
  int rc = 0;
  for (;;) {
    rc = cg_chunk<R>(op, prec, mass, w, k, r, Mk, ne, g);
    if (rc) break;
    cudaError_t e = cudaMemcpyAsync(&h, w.S, sizeof(CGState), cudaMemcpyDeviceToHost, L.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(L.stream);
    if (e != cudaSuccess) {
      rc = fail_cuda(e, "cg state readback", __FILE__, __LINE__);
      break;
    }
    if (h.state != 0) break;
  }
  L.cur_stop = nullptr;
  if (rc) return rc;
  cgiter += h.iter;
  if (h.state == 3) {
    *iters = cgiter;
    set_error("cg_mshift: breakdown at iteration %d (alpha=%g, |r|^2=%g)", cgiter, h.alpha, h.lambda);
    return HRGPU_E_BREAKDOWN;
  }
  if (!flt) {
    // true residual of every shift (cg_mshift.c:122-137)
    for (int i = 0; i < n; i++) {
      if (int q = apply_op(op, prec, mass, Mk, out[i])) return q;
      ++cgiter;
      if (int q = la_op(LA_MUL_ADD_ASSIGN, par, prec, Mk, out[i], nullptr, -shift[i], 0, 0, 0)) return q;
      if (int q = la_op(LA_SUB_ASSIGN, par, prec, Mk, in, nullptr, 0, 0, 0, 0)) return q;
      double nr;
      if (int q = la_dot(2, par, prec, Mk, nullptr, &nr)) return q;
      if (!isfinite(nr)) {
        *iters = cgiter;
        set_error("cg_mshift: the true residual of shift %d is not finite (%g)", i, nr);
        return HRGPU_E_BREAKDOWN;
      }
      flags[i] = (fabs(nr / innorm2) > err2) ? 0 : 1;
    }
  }
  *iters = cgiter;
  return 0;
}

static int cg_check(int op, int n, const double *shift, const void *in, void *const *out, int *iters) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "cg_mshift: lattice not initialised");
  HR_REQUIRE(op >= 0 && op <= 3, HRGPU_E_ARG, "cg_mshift: unknown operator %d", op);
  HR_REQUIRE(n > 0 && n <= MAXS, HRGPU_E_ARG, "cg_mshift: n = %d shifts (1..%d supported)", n, MAXS);
  HR_REQUIRE(shift && in && out && iters, HRGPU_E_ARG, "cg_mshift: NULL argument");
  for (int i = 0; i < n; i++) HR_REQUIRE(out[i] != nullptr && out[i] != in, HRGPU_E_ARG, "cg_mshift: bad output field");
  return 0;
}

}  // namespace hrgpu

using namespace hrgpu;

extern "C" {

int hrgpu_cg_mshift(int op, double mass, int n, const double *shift, double err2, int max_iter, const void *in,
                    void *const *out, int *iters) {
  if (int rc = cg_check(op, n, shift, in, out, iters)) return rc;
  std::vector<int> flags(n, 1);
  int total = 0, it = 0;
  if (int rc = cg_core<double>(op, mass, n, shift, err2, max_iter, in, out, flags.data(), 0, &it)) return rc;
  total += it;
  // unconverged shifts are solved again one at a time from their current solution
  // (cg_mshift.c:170-179); bounded here so a hopeless system returns instead of looping
  int status = 0;
  for (int i = 0; i < n; i++) {
    int rep = 0;
    while (flags[i] == 0) {
      if (++rep > 20) {
        status = HRGPU_E_NOCONV;
        set_error("cg_mshift: shift %d did not reach err2=%g after %d restarts", i, err2, rep - 1);
        break;
      }
      void *o[1] = {out[i]};
      if (int rc = cg_core<double>(op, mass, 1, shift + i, err2, max_iter, in, o, &flags[i], 0, &it)) return rc;
      total += it;
    }
  }
  *iters = total;
  return status;
}

// cg_mshift_flt (cg_mshift_flt.c:144-276)
int hrgpu_cg_mshift_flt(int op, double mass, int n, const double *shift, double err2, int max_iter, const void *in,
                        void *const *out, int *iters) {
  if (int rc = cg_check(op, n, shift, in, out, iters)) return rc;
  HR_REQUIRE(op != HRGPU_OP_G5CPHI_SQ, HRGPU_E_ARG, "cg_mshift_flt: no float version of g5Cphi_sq");
  const int par = op_parity(op);
  const size_t bd = spinor_bytes(par, HRGPU_DOUBLE), bf = spinor_bytes(par, HRGPU_FLOAT);
  if (FW.bd != bd) {
    cudaFree(FW.dres); cudaFree(FW.dres2); cudaFree(FW.dtmp);
    HR_CUDA(cudaMalloc(&FW.dres, bd));
    HR_CUDA(cudaMalloc(&FW.dres2, bd));
    HR_CUDA(cudaMalloc(&FW.dtmp, bd));
    FW.bd = bd;
  }
  if (FW.bf != bf) {
    for (void *b : FW.fbuf) cudaFree(b);
    FW.fbuf.clear();
    FW.bf = bf;
  }
  while ((int)FW.fbuf.size() < n + 1) {
    void *b;
    HR_CUDA(cudaMalloc(&b, bf));
    FW.fbuf.push_back(b);
  }
  void *dres = FW.dres, *dres2 = FW.dres2, *dtmp = FW.dtmp;
  std::vector<void *> &fbuf = FW.fbuf;
  void *res_flt = fbuf[0];
  std::vector<void *> out_flt(fbuf.begin() + 1, fbuf.begin() + 1 + n);
  std::vector<int> sflags(n, 1), loc(n);
  std::vector<double> norm(n, 0.0);
  for (int i = 0; i < n; i++)
    if (n != 1) HR_CUDA(cudaMemsetAsync(out[i], 0, bd, L.stream));
  double innorm2;
  if (int rc = la_dot(2, par, HRGPU_DOUBLE, in, nullptr, &innorm2)) return rc;
  if (!isfinite(innorm2)) {
    *iters = 0;
    set_error("cg_mshift_flt: the source norm is not finite (%g)", innorm2);
    return HRGPU_E_BREAKDOWN;
  }
  if (innorm2 == 0.0) {
    for (int i = 0; i < n; i++) HR_CUDA(cudaMemsetAsync(out[i], 0, bd, L.stream));
    *iters = 0;
    return 0;
  }
  int siter = 0, diter = 0, notconverged, rounds = 0;
  const double mass_d = mass;
  do {
    int first = 1;
    notconverged = 0;
    double local_err2 = err2;
    for (int i = 0; i < n; i++) {
      if (!sflags[i]) continue;
      if (int rc = apply_op(op, HRGPU_DOUBLE, mass_d, dtmp, out[i])) return rc;
      ++diter;
      if (int rc = la_op(LA_SUB, par, HRGPU_DOUBLE, dres2, in, dtmp, 0, 0, 0, 0)) return rc;
      if (int rc = la_op(LA_MUL_ADD_ASSIGN, par, HRGPU_DOUBLE, dres2, out[i], nullptr, shift[i], 0, 0, 0)) return rc;
      if (int rc = la_dot(2, par, HRGPU_DOUBLE, dres2, nullptr, &norm[i])) return rc;
      if (!isfinite(norm[i])) {
        *iters = siter + diter;
        set_error("cg_mshift_flt: the residual of shift %d is not finite (%g)", i, norm[i]);
        return HRGPU_E_BREAKDOWN;
      }
      if (norm[i] < innorm2 * err2) {
        sflags[i] = 0;
        norm[i] /= innorm2;
      } else {
        ++notconverged;
        if (first) {
          first = 0;
          local_err2 = norm[i] / innorm2;
          norm[i] = sqrt(norm[i]);
          if (int rc = la_op(LA_MUL, par, HRGPU_DOUBLE, dres, dres2, nullptr, 1. / norm[i], 0, 0, 0)) return rc;
        } else {
          double pr[2];
          if (int rc = la_dot(0, par, HRGPU_DOUBLE, dres, dres2, pr)) return rc;
          norm[i] = pr[0];
        }
      }
    }
    if (notconverged) {
      if (int rc = hrgpu_assign_sd2s(res_flt, dres, par)) return rc;
      local_err2 = err2 / local_err2 * 0.9;
      if (local_err2 < 1.e-10) local_err2 = 1.e-10;
      for (int i = 0; i < n; i++) loc[i] = sflags[i];
      // a single shift starts the inner solve from out_flt[0]: start from zero
      if (n == 1) HR_CUDA(cudaMemsetAsync(out_flt[0], 0, bf, L.stream));
      int it = 0;
      if (int rc = cg_core<float>(op, mass_d, n, shift, local_err2, max_iter, res_flt, out_flt.data(), loc.data(), 1, &it))
        return rc;
      siter += it;
      for (int i = 0; i < n; i++)
        if (sflags[i]) {
          if (int rc = hrgpu_assign_s2sd(dres2, out_flt[i], par)) return rc;
          if (int rc = la_op(LA_MUL_ADD_ASSIGN, par, HRGPU_DOUBLE, out[i], dres2, nullptr, norm[i], 0, 0, 0)) return rc;
        }
    }
    if (++rounds > 200) {
      *iters = siter + diter;
      set_error("cg_mshift_flt: no convergence to err2=%g after %d defect-correction rounds", err2, rounds);
      return HRGPU_E_NOCONV;
    }
  } while (notconverged);
  *iters = siter + diter;
  return 0;
}

}  // extern "C"
