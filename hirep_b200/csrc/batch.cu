// batch.cu -- many right-hand sides at once.
//
// A batch of nb even-parity fields is one buffer in the tiled layout of
// hop_tile.cuh: tiles of 4 fields, blocks of 8 sites, element (component c,
// site n, field f) at (((f/4) * ld/8 + n/8) * 4NF + c) * 32 + (n%8) * 4 + f%4.
// The linear algebra sees a tile as rows of 4 fields (row = position of a
// (site, component) pair in the tile) and is indifferent to the row order.
// The even-odd preconditioned operators act on a whole batch with k_hopt, which
// reads each link and clover block once for all the fields of a tile and
// addresses every component at a constant offset.  On top of it sits a batched
// multi-shift CG: several Krylov spaces (HiRep's cg_mshift recursion,
// LibHR/Inverters/cg_mshift.c:24-145, for each) with any number of shifts each,
// every scalar on the device, the iteration captured once as a CUDA graph and
// replayed.  HiRep's defect-correction driver (LibHR/Inverters/cg_mshift_flt.c:
// 144-276) runs around it: FP64 true residuals of all systems in one batched
// operator call, the FP32 inner solves of all sources in one batched CG.
#include <math.h>
#include <string.h>

#include <vector>

#include "dirac.cuh"
#include "hop_tile.cuh"
#include "linalg.cuh"

namespace hrgpu {

template <typename R, int EP>
int launch_batch(TileArgs<R> &a);  // hop_batch_launch.cuh, instantiated in dirac_b_*.cu

constexpr int BMAXB = 64;   // Krylov spaces per batch
constexpr int BMAXS = 64;   // systems (Krylov space, shift) per batch
constexpr int BCHUNK = 8;   // CG iterations per captured graph

static inline int ntiles(int nb) { return (nb + TILE_F - 1) / TILE_F; }
static inline size_t batch_bytes(int prec, int nb) { return (size_t)ntiles(nb) * TILE_F * spinor_bytes(HRGPU_EVEN, prec); }

// ---------------------------------------------------------------------------
// copies of the links and clover blocks in blocks of 8 sites (hop_tile.cuh)
// ---------------------------------------------------------------------------
struct TileCopies {
  void *U[2] = {nullptr, nullptr};
  unsigned long ugen[2] = {0, 0};
  bool uok[2] = {false, false};
  void *dg[2] = {nullptr, nullptr}, *od[2] = {nullptr, nullptr}, *idg[2] = {nullptr, nullptr}, *iod[2] = {nullptr, nullptr};
  unsigned long cgen[2] = {0, 0};
  bool cok[2] = {false, false};
};
static TileCopies TC;

static unsigned copy_grid(long n) {
  long b = (n + 255) / 256;
  return (unsigned)(b < 148L * 16 ? b : 148L * 16);
}

static int ensure_tile_links(int prec) {
  if (TC.uok[prec] && TC.ugen[prec] == L.gauge_gen) return 0;
  const int nel = L.nf * L.nf;
  const size_t esz = (L.real ? 1 : 2) * (prec == HRGPU_DOUBLE ? sizeof(double) : sizeof(float));
  const long n = 2L * L.ld * 4 * nel;
  if (!TC.U[prec]) HR_CUDA(cudaMalloc(&TC.U[prec], (size_t)n * esz));
  const void *src = prec == HRGPU_DOUBLE ? L.U : L.Uf;
  const unsigned g = copy_grid(n);
  if (prec == HRGPU_DOUBLE) {
    if (L.real) k_tile_links<double><<<g, 256, 0, L.stream>>>((double *)TC.U[prec], (const double *)src, nel, L.ld);
    else k_tile_links<double2><<<g, 256, 0, L.stream>>>((double2 *)TC.U[prec], (const double2 *)src, nel, L.ld);
  } else {
    if (L.real) k_tile_links<float><<<g, 256, 0, L.stream>>>((float *)TC.U[prec], (const float *)src, nel, L.ld);
    else k_tile_links<float2><<<g, 256, 0, L.stream>>>((float2 *)TC.U[prec], (const float2 *)src, nel, L.ld);
  }
  HR_LAUNCH_CHECK();
  TC.ugen[prec] = L.gauge_gen;
  TC.uok[prec] = true;
  return 0;
}

template <typename E>
static int tile_clover_one(void **dst, const E *src, int kn) {
  const long n = 2L * L.ld * 2 * kn;
  if (!*dst) HR_CUDA(cudaMalloc(dst, (size_t)n * sizeof(E)));
  k_tile_clover<E><<<copy_grid(n), 256, 0, L.stream>>>((E *)*dst, src, kn, L.ld);
  HR_LAUNCH_CHECK();
  return 0;
}

// after clover_prepare(mass, prec): copies of (4+m)+A and of its inverse
static int ensure_tile_clover(int prec) {
  if (TC.cok[prec] && TC.cgen[prec] == L.clover_gen[prec]) return 0;
  const int kd = 2 * L.nf, ko = L.nf * (2 * L.nf - 1);
  if (prec == HRGPU_DOUBLE) {
    if (int rc = tile_clover_one<double>(&TC.dg[0], L.cl_dg, kd)) return rc;
    if (int rc = tile_clover_one<double2>(&TC.od[0], L.cl_od, ko)) return rc;
    if (int rc = tile_clover_one<double>(&TC.idg[0], L.cl_idg, kd)) return rc;
    if (int rc = tile_clover_one<double2>(&TC.iod[0], L.cl_iod, ko)) return rc;
  } else {
    if (int rc = tile_clover_one<float>(&TC.dg[1], L.cl_dg_f, kd)) return rc;
    if (int rc = tile_clover_one<float2>(&TC.od[1], L.cl_od_f, ko)) return rc;
    if (int rc = tile_clover_one<float>(&TC.idg[1], L.cl_idg_f, kd)) return rc;
    if (int rc = tile_clover_one<float2>(&TC.iod[1], L.cl_iod_f, ko)) return rc;
  }
  TC.cgen[prec] = L.clover_gen[prec];
  TC.cok[prec] = true;
  return 0;
}

// ---------------------------------------------------------------------------
// batched even-odd operators
// ---------------------------------------------------------------------------
struct BatchTmp {
  void *odd[2] = {nullptr, nullptr}, *even[2] = {nullptr, nullptr};  // [prec]
  size_t bytes[2] = {0, 0};
};
static BatchTmp BT;

static int ensure_batch_buf(void **p, size_t *have, size_t bytes) {
  if (*p && *have >= bytes) return 0;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  HR_CUDA(cudaMalloc(p, bytes));
  // padding sites (cb >= VH) and padding fields are never written: keep them zero
  HR_CUDA(cudaMemsetAsync(*p, 0, bytes, L.stream));
  *have = bytes;
  return 0;
}

static int ensure_batch_tmp(int prec, int nb) {
  const size_t bytes = batch_bytes(prec, nb);
  if (BT.bytes[prec] >= bytes && BT.odd[prec] && BT.even[prec]) return 0;
  size_t h1 = 0, h2 = 0;
  if (BT.odd[prec]) cudaFree(BT.odd[prec]);
  if (BT.even[prec]) cudaFree(BT.even[prec]);
  BT.odd[prec] = BT.even[prec] = nullptr;
  if (int rc = ensure_batch_buf(&BT.odd[prec], &h1, bytes)) return rc;
  if (int rc = ensure_batch_buf(&BT.even[prec], &h2, bytes)) return rc;
  BT.bytes[prec] = bytes;
  return 0;
}

template <typename R>
static int hopb(int outp, void *out, const void *in, int nb, int ep, double cacc, const void *aux, double caux, int g5,
                bool inv, const int *stop) {
  const int prec = sizeof(R) == 8 ? HRGPU_DOUBLE : HRGPU_FLOAT;
  TileArgs<R> a;
  a.in = in;
  a.out = out;
  a.aux = aux;
  a.U = TC.U[prec];
  a.cdg = (const R *)(inv ? TC.idg[prec] : TC.dg[prec]);
  a.cod = (const typename C2<R>::T *)(inv ? TC.iod[prec] : TC.od[prec]);
  a.stop = stop;
  a.cacc = (R)cacc;
  a.caux = (R)caux;
  a.outp = outp;
  a.g5 = g5;
  a.nb = nb;
  if (ep == EP_AXPY) return launch_batch<R, EP_AXPY>(a);
  if (ep == EP_CLOV_INV) return launch_batch<R, EP_CLOV_INV>(a);
  return launch_batch<R, EP_CLOV>(a);
}

// out = (4+m)^2 in - D_eo D_oe in on the even sites of nb fields (Dphi.c:874-907)
template <typename R>
static int Dphi_eo_b(double m0, void *out, const void *in, int nb, int g5, const int *stop) {
  const int prec = sizeof(R) == 8 ? HRGPU_DOUBLE : HRGPU_FLOAT;
  if (int rc = ensure_batch_tmp(prec, nb)) return rc;
  if (int rc = ensure_tile_links(prec)) return rc;
  if (int rc = hopb<R>(HRGPU_ODD, BT.odd[prec], in, nb, EP_AXPY, -0.5, nullptr, 0.0, 0, false, stop)) return rc;
  double rho;
  if (sizeof(R) == 4) {
    float r = 4.f + (float)m0;
    rho = (double)(r * r);
  } else {
    rho = (4.0 + m0) * (4.0 + m0);
  }
  return hopb<R>(HRGPU_EVEN, out, BT.odd[prec], nb, EP_AXPY, 0.5, in, rho, g5, false, stop);
}

// out = D_ee in - D_eo D_oo^-1 D_oe in (Dphi.c:1240-1255)
template <typename R>
static int Cphi_eo_b(double mass, void *out, const void *in, int nb, int g5, const int *stop) {
  const int prec = sizeof(R) == 8 ? HRGPU_DOUBLE : HRGPU_FLOAT;
  HR_REQUIRE(L.clover, HRGPU_E_STATE, "Cphi_eopre: no clover term (hrgpu_clover_init)");
  if (int rc = clover_prepare(mass, prec)) return rc;
  if (int rc = ensure_tile_clover(prec)) return rc;
  if (int rc = ensure_tile_links(prec)) return rc;
  if (int rc = ensure_batch_tmp(prec, nb)) return rc;
  if (int rc = hopb<R>(HRGPU_ODD, BT.odd[prec], in, nb, EP_CLOV_INV, -0.5, nullptr, 0.0, 0, true, stop)) return rc;
  return hopb<R>(HRGPU_EVEN, out, BT.odd[prec], nb, EP_CLOV, 0.5, in, 0.0, g5, false, stop);
}

static bool batch_op_ok(int op) {
  return op == HRGPU_OP_G5DPHI_EOPRE_SQ || op == HRGPU_OP_G5CPHI_EOPRE_SQ || op == HRGPU_OP_G5DPHI_EOPRE ||
         op == HRGPU_OP_G5CPHI_EOPRE || op == HRGPU_OP_DPHI_EOPRE || op == HRGPU_OP_CPHI_EOPRE;
}
static bool batch_op_clover(int op) {
  return op == HRGPU_OP_G5CPHI_EOPRE_SQ || op == HRGPU_OP_G5CPHI_EOPRE || op == HRGPU_OP_CPHI_EOPRE;
}

// the operators of one batch; the squared ones go through the even temporary
static int apply_op_b(int op, int prec, double mass, void *out, const void *in, int nb, const int *stop) {
  if (int rc = check_gauge(prec)) return rc;
  const bool clov = batch_op_clover(op);
  const bool sq = op == HRGPU_OP_G5DPHI_EOPRE_SQ || op == HRGPU_OP_G5CPHI_EOPRE_SQ;
  const int g5 = (op == HRGPU_OP_DPHI_EOPRE || op == HRGPU_OP_CPHI_EOPRE) ? 0 : 1;
  auto one = [&](void *o, const void *i) -> int {
    if (prec == HRGPU_DOUBLE) return clov ? Cphi_eo_b<double>(mass, o, i, nb, g5, stop) : Dphi_eo_b<double>(mass, o, i, nb, g5, stop);
    return clov ? Cphi_eo_b<float>(mass, o, i, nb, g5, stop) : Dphi_eo_b<float>(mass, o, i, nb, g5, stop);
  };
  if (!sq) return one(out, in);
  if (int rc = ensure_batch_tmp(prec, nb)) return rc;
  if (int rc = one(BT.even[prec], in)) return rc;
  return one(out, BT.even[prec]);
}

// everything the operator reads, made up to date outside any graph capture
static int prepare_op_b(int op, int prec, double mass, int nb) {
  if (int rc = check_gauge(prec)) return rc;
  if (batch_op_clover(op)) {
    HR_REQUIRE(L.clover, HRGPU_E_STATE, "Cphi_eopre: no clover term (hrgpu_clover_init)");
    if (int rc = clover_prepare(mass, prec)) return rc;
    if (int rc = ensure_tile_clover(prec)) return rc;
  }
  if (int rc = ensure_tile_links(prec)) return rc;
  return ensure_batch_tmp(prec, nb);
}

// ---------------------------------------------------------------------------
// linear algebra on batches.  Block (x, y): tile y, rows of that tile strided
// over the x blocks; thread t works on field 4y + t%4 of rows t/4, t/4 +
// rows-per-grid, ... so a warp reads 8 rows x 4 fields contiguously and every
// thread keeps one field for the whole loop.
// ---------------------------------------------------------------------------
constexpr int BTHREADS = 256;

__device__ __forceinline__ long bix(long row, int f, long rows) {
  return ((long)(f / TILE_F) * rows + row) * TILE_F + (f % TILE_F);
}

struct BMap {
  int f;
  long row, stride;
  bool on;
};

__device__ __forceinline__ BMap bmap(int nb) {
  BMap m;
  m.f = blockIdx.y * TILE_F + (threadIdx.x % TILE_F);
  m.row = (long)blockIdx.x * (BTHREADS / TILE_F) + threadIdx.x / TILE_F;
  m.stride = (long)gridDim.x * (BTHREADS / TILE_F);
  m.on = m.f < nb;
  return m;
}

// part[blockIdx.x * 4*gridDim.y + f] = the block's sum of v for each of its 4 fields
__device__ __forceinline__ void bpartial(double v, double *part) {
  __shared__ double sh[BTHREADS];
  sh[threadIdx.x] = v;
  __syncthreads();
  if (threadIdx.x < TILE_F) {
    double s = 0.0;
    for (int k = 0; k < BTHREADS / TILE_F; k++) s += sh[k * TILE_F + threadIdx.x];
    part[(long)blockIdx.x * TILE_F * gridDim.y + blockIdx.y * TILE_F + threadIdx.x] = s;
  }
}

static dim3 bgrid(long rows, int nb) {
  const long per = BTHREADS / TILE_F;
  long b = (rows + per - 1) / per;
  b = b < RED_MAX_BLOCKS ? (b > 0 ? b : 1) : RED_MAX_BLOCKS;
  return dim3((unsigned)b, (unsigned)ntiles(nb));
}

// row of a tile holding component c of site n
__device__ __forceinline__ long tile_row(long n, long c, int ncomp) {
  return ((n / TILE_S) * ncomp + c) * TILE_S + (n % TILE_S);
}

// separate single-field arrays (element (c, n) at c*ld + n) into a batch, and
// back; threads run over the single-field order, whose runs of 8 sites are
// runs of 8 rows of the tile
template <typename V>
__global__ void k_bpack(V *dst, const V *const *src, long rows, int ld, int ncomp, int nb) {
  BMap m = bmap(nb);
  if (!m.on) return;
  const V *s = src[m.f];
  for (long i = m.row; i < rows; i += m.stride) {
    const long c = i / ld, n = i - c * ld;
    dst[bix(tile_row(n, c, ncomp), m.f, rows)] = s[i];
  }
}
template <typename V>
__global__ void k_bunpack(V *const *dst, const V *src, long rows, int ld, int ncomp, int nb) {
  BMap m = bmap(nb);
  if (!m.on) return;
  V *d = dst[m.f];
  for (long i = m.row; i < rows; i += m.stride) {
    const long c = i / ld, n = i - c * ld;
    d[i] = src[bix(tile_row(n, c, ncomp), m.f, rows)];
  }
}

// per-field Re <a_f, b_f> partials
template <typename V>
__global__ void __launch_bounds__(BTHREADS) k_bdot(const int *state, const V *a, const V *b, long rows, int nb,
                                                   double *part) {
  if (state && *state != 0) return;
  BMap m = bmap(nb);
  double s = 0.0;
  if (m.on)
    for (long r = m.row; r < rows; r += m.stride) {
      V u = a[bix(r, m.f, rows)], v = b[bix(r, m.f, rows)];
      s += (double)u.x * v.x + (double)u.y * v.y;
    }
  bpartial(s, part);
}

// sum over the nblk partial rows of field f (row stride nbp = 4 * tiles), fixed
// tree order (one block)
__device__ double bfold_one(const double *part, int nblk, int nbp, int f) {
  double s = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += part[(long)b * nbp + f];
  return block_sum(s);
}

__global__ void k_bfold(const double *part, int nblk, int nb, double *out) {
  const int nbp = ((nb + TILE_F - 1) / TILE_F) * TILE_F;
  for (int f = 0; f < nb; f++) {
    double v = bfold_one(part, nblk, nbp, f);
    if (threadIdx.x == 0) out[f] = v;
  }
}

// per-field sums of Re <a_f, b_f> (or |a_f|^2 with b = a) to the host
static int bdot_host(const void *a, const void *b, int prec, long rows, int nb, double *part, double *dres,
                     double *hres, double *out) {
  const dim3 g = bgrid(rows, nb);
  if (prec == HRGPU_DOUBLE)
    k_bdot<double2><<<g, BTHREADS, 0, L.stream>>>(nullptr, (const double2 *)a, (const double2 *)b, rows, nb, part);
  else
    k_bdot<float2><<<g, BTHREADS, 0, L.stream>>>(nullptr, (const float2 *)a, (const float2 *)b, rows, nb, part);
  k_bfold<<<1, BTHREADS, 0, L.stream>>>(part, g.x, nb, dres);
  HR_LAUNCH_CHECK();
  HR_CUDA(cudaMemcpyAsync(hres, dres, sizeof(double) * nb, cudaMemcpyDeviceToHost, L.stream));
  HR_CUDA(cudaStreamSynchronize(L.stream));
  for (int f = 0; f < nb; f++) out[f] = hres[f];
  return 0;
}

// ---------------------------------------------------------------------------
// batched multi-shift CG.  Per source s: HiRep's scalars; per system j (a
// source and one shift): z1, z2, z3, the solution and direction coefficients
// and the convergence flag.  Source states: 0 running, 1 stop after this
// iteration, 2 stopped, 3 breakdown.  The batch state follows the same codes
// and reaches 1 when no source is running; the hopping kernels read it and
// return at once after that, so replaying a captured chunk past the end does
// nothing.
// ---------------------------------------------------------------------------
struct BSrc {
  double omega, oldomega, gamma, alpha, lambda, delta, innorm2, err2;
  int state, iter, notconv, pad;
};
struct BState {
  int nb, nsys, max_iter, flt, state, iter;
  BSrc s[BMAXB];
  int src[BMAXS], flag[BMAXS];
  double shift[BMAXS], z1[BMAXS], z2[BMAXS], z3[BMAXS], cx[BMAXS], cp[BMAXS];
};

// alpha = <k, Mk> per source; omega, z3 and the solution coefficients (cg_mshift.c:82-91)
__global__ void k_bfold_alpha(BState *S, const double *part, int nblk) {
  if (S->state != 0) return;
  const int nb = S->nb;
  for (int f = 0; f < nb; f++) {
    double alpha = bfold_one(part, nblk, ((nb + TILE_F - 1) / TILE_F) * TILE_F, f);
    if (threadIdx.x != 0) continue;
    BSrc &q = S->s[f];
    if (q.state != 0) {
      for (int j = 0; j < S->nsys; j++)
        if (S->src[j] == f) S->cx[j] = 0.0;
      continue;
    }
    q.alpha = alpha;
    if (!isfinite(alpha) || alpha == 0.0) {  // breakdown: this source stops, the others go on
      q.state = 3;
      for (int j = 0; j < S->nsys; j++)
        if (S->src[j] == f) S->cx[j] = 0.0;
      continue;
    }
    q.oldomega = q.omega;
    q.omega = -q.delta / alpha;
    const double omega = q.omega, oldomega = q.oldomega, gamma = q.gamma;
    for (int j = 0; j < S->nsys; j++) {
      if (S->src[j] != f) continue;
      if (S->flag[j]) {
        const double z1 = S->z1[j], z2 = S->z2[j];
        const double z3 = oldomega * z1 * z2 / (omega * gamma * (z1 - z2) + z1 * oldomega * (1. + S->shift[j] * omega));
        S->z3[j] = z3;
        S->cx[j] = -omega * z3 / z2;
      } else {
        S->cx[j] = 0.0;
      }
    }
  }
}

// lambda = |r|^2 per source; gamma, flags, stopping (cg_mshift.c:92-111; cg_mshift_flt.c:96-118)
__global__ void k_bfold_lambda(BState *S, const double *part, int nblk) {
  if (S->state != 0) return;
  const int nb = S->nb;
  for (int f = 0; f < nb; f++) {
    double lambda = bfold_one(part, nblk, ((nb + TILE_F - 1) / TILE_F) * TILE_F, f);
    if (threadIdx.x != 0) continue;
    BSrc &q = S->s[f];
    if (q.state != 0) continue;
    q.lambda = lambda;
    q.gamma = lambda / q.delta;
    q.delta = lambda;
    const double gamma = q.gamma, delta = q.delta;
    int notconv = 0;
    for (int j = 0; j < S->nsys; j++) {
      if (S->src[j] != f) continue;
      const double z3 = S->z3[j];
      if (S->flt) {
        if (delta * z3 * z3 > q.err2 * q.innorm2) ++notconv;
      } else {
        if (delta * z3 * z3 < q.err2 * q.innorm2) S->flag[j] = 0;
        if (S->flag[j]) ++notconv;
      }
      if (S->flag[j]) {
        const double z2 = S->z2[j];
        S->cp[j] = gamma * z3 * z3 / (z2 * z2);
        S->z1[j] = S->z2[j];
        S->z2[j] = z3;
      }
    }
    q.notconv = notconv;
    q.iter++;
    if (!isfinite(lambda)) q.state = 3;
    else if (notconv == 0 || (S->max_iter != 0 && q.iter >= S->max_iter)) q.state = 1;
  }
  if (threadIdx.x == 0) {
    S->iter++;
    bool any = false;
    for (int f = 0; f < nb; f++) any = any || S->s[f].state == 0;
    if (!any) S->state = 1;
  }
}

__global__ void k_badvance(BState *S) {
  for (int f = 0; f < S->nb; f++)
    if (S->s[f].state == 1) S->s[f].state = 2;
  if (S->state == 1) S->state = 2;
}

// r += omega Mk per source, with |r|^2 partials
template <typename V>
__global__ void __launch_bounds__(BTHREADS) k_bupd_r(const BState *S, V *r, const V *Mk, long rows, double *part) {
  if (S->state != 0) return;
  const int nb = S->nb;
  BMap m = bmap(nb);
  double s = 0.0;
  if (m.on && S->s[m.f].state == 0) {
    typedef decltype(r[0].x) R;
    const R omega = (R)S->s[m.f].omega;
    for (long i = m.row; i < rows; i += m.stride) {
      const long e = bix(i, m.f, rows);
      V rv = r[e];
      rmac(rv, omega, Mk[e]);
      r[e] = rv;
      s += (double)rv.x * rv.x + (double)rv.y * rv.y;
    }
  }
  bpartial(s, part);
}

// x_j += cx_j p_j (the direction of this iteration), then p_j = cp_j p_j + z3_j r
template <typename V>
__global__ void __launch_bounds__(BTHREADS) k_bupd_xp(const BState *S, V *x, V *p, const V *r, long rows) {
  if (S->state >= 2) return;
  const int ns = S->nsys;
  BMap m = bmap(ns);
  if (!m.on) return;
  const int j = m.f, sj = S->src[j];
  if (S->s[sj].state >= 2) return;
  typedef decltype(r[0].x) R;
  const R cx = (R)S->cx[j], cp = (R)S->cp[j], z3 = (R)S->z3[j];
  const bool upd_p = S->flag[j] != 0;
  for (long i = m.row; i < rows; i += m.stride) {
    const long e = bix(i, j, rows);
    V pv = p[e];
    if (cx != (R)0) {
      V xv = x[e];
      rmac(xv, cx, pv);
      x[e] = xv;
    }
    if (upd_p) {
      pv.x = cp * pv.x;
      pv.y = cp * pv.y;
      rmac(pv, z3, r[bix(i, sj, rows)]);
      p[e] = pv;
    }
  }
}

// k = gamma k + r per source
template <typename V>
__global__ void __launch_bounds__(BTHREADS) k_bupd_k(const BState *S, V *k, const V *r, long rows) {
  if (S->state >= 2) return;
  const int nb = S->nb;
  BMap m = bmap(nb);
  if (!m.on || S->s[m.f].state >= 2) return;
  typedef decltype(r[0].x) R;
  const R gamma = (R)S->s[m.f].gamma;
  for (long i = m.row; i < rows; i += m.stride) {
    const long e = bix(i, m.f, rows);
    V kv = k[e], rv = r[e];
    kv.x = gamma * kv.x + rv.x;
    kv.y = gamma * kv.y + rv.y;
    k[e] = kv;
  }
}

// p_j = rhs of the source of j
template <typename V>
__global__ void k_bspread(V *p, const V *r, const int *src, long rows, int ns, int nb) {
  BMap m = bmap(ns);
  if (!m.on) return;
  const int sj = src[m.f];
  for (long i = m.row; i < rows; i += m.stride) p[bix(i, m.f, rows)] = r[bix(i, sj, rows)];
}

// ---------------------------------------------------------------------------
// FP64 defect-correction helpers (systems: an ns-field batch)
// ---------------------------------------------------------------------------
// res_j = b_src(j) - Mx_j + shift_j x_j (in place over Mx), |res_j|^2 partials
__global__ void __launch_bounds__(BTHREADS) k_bres(double2 *res, const double2 *b, const double2 *x, const int *src,
                                                   const double *shift, long rows, int ns, double *part) {
  BMap m = bmap(ns);
  double s = 0.0;
  if (m.on) {
    const int j = m.f, sj = src[j];
    const double sh = shift[j];
    for (long i = m.row; i < rows; i += m.stride) {
      const long e = bix(i, j, rows);
      double2 v = res[e], bb = b[bix(i, sj, rows)], xx = x[e];
      v.x = bb.x - v.x + sh * xx.x;
      v.y = bb.y - v.y + sh * xx.y;
      res[e] = v;
      s += v.x * v.x + v.y * v.y;
    }
  }
  bpartial(s, part);
}

// Re <res_first(j), res_j> partials
__global__ void __launch_bounds__(BTHREADS) k_bproj(const double2 *res, const int *first, long rows, int ns,
                                                    double *part) {
  BMap m = bmap(ns);
  double s = 0.0;
  if (m.on && first[m.f] >= 0) {
    const int j = m.f, fj = first[j];
    for (long i = m.row; i < rows; i += m.stride) {
      double2 u = res[bix(i, fj, rows)], v = res[bix(i, j, rows)];
      s += u.x * v.x + u.y * v.y;
    }
  }
  bpartial(s, part);
}

// inner right-hand sides: rhs_s = res_first(s) * scale_s in FP32 (zero for sources without work)
__global__ void k_brhs(float2 *rhs, const double2 *res, const int *first, const double *scale, long rows, int nb) {
  BMap m = bmap(nb);
  if (!m.on) return;
  const int fs = first[m.f];
  const double sc = scale[m.f];
  for (long i = m.row; i < rows; i += m.stride) {
    float2 o = make_float2(0.f, 0.f);
    if (fs >= 0) {
      double2 v = res[bix(i, fs, rows)];
      o = make_float2((float)(v.x * sc), (float)(v.y * sc));
    }
    rhs[bix(i, m.f, rows)] = o;
  }
}

// x_map(k) += c_k xf_k (FP64 += FP64 * FP32) for the nsi inner systems k, which
// correct the systems map[k] of the outer batch; c_k = 0: untouched
__global__ void k_bacc(double2 *x, const float2 *xf, const double *c, const int *map, long rows, int nsi) {
  BMap m = bmap(nsi);
  if (!m.on) return;
  const double ck = c[m.f];
  if (ck == 0.0) return;
  const int j = map[m.f];
  for (long i = m.row; i < rows; i += m.stride) {
    const long e = bix(i, j, rows);
    double2 v = x[e];
    float2 w = xf[bix(i, m.f, rows)];
    v.x += ck * (double)w.x;
    v.y += ck * (double)w.y;
    x[e] = v;
  }
}

// ---------------------------------------------------------------------------
// workspace: cached between calls, grown on demand; one per precision
// ---------------------------------------------------------------------------
struct BWork {
  void *r = nullptr, *k = nullptr, *Mk = nullptr, *p = nullptr;
  size_t hr = 0, hk = 0, hm = 0, hp = 0;
  BState *S = nullptr, *hS = nullptr;
  // captured chunk of iterations and what it was captured for
  cudaGraphExec_t exec = nullptr;
  int g_op = -1, g_nb = 0, g_ns = 0;
  double g_mass = 0.0;
  const void *g_key[12] = {};
};
static BWork BW[2];

// FP64 driver buffers and shared reduction scratch
struct BOuter {
  void *b = nullptr, *x = nullptr, *res = nullptr, *rhs = nullptr, *xf = nullptr;
  size_t hb = 0, hx = 0, hres = 0, hrhs = 0, hxf = 0;
  double *part = nullptr, *dres = nullptr, *hres_h = nullptr;
  int *d_src = nullptr, *d_first = nullptr, *d_map = nullptr;
  int *d_isrc = nullptr;  // source of each system of the inner (bcg_core) batch
  double *d_shift = nullptr, *d_scale = nullptr;
  void **d_ptrs = nullptr;
  cudaStream_t cap = nullptr;  // capture stream
};
static BOuter BO;

static int bouter_init() {
  if (BO.part) return 0;
  HR_CUDA(cudaMalloc(&BO.part, sizeof(double) * RED_MAX_BLOCKS * BMAXS));
  HR_CUDA(cudaMalloc(&BO.dres, sizeof(double) * BMAXS));
  HR_CUDA(cudaMallocHost(&BO.hres_h, sizeof(double) * BMAXS));
  HR_CUDA(cudaMalloc(&BO.d_src, sizeof(int) * BMAXS));
  HR_CUDA(cudaMalloc(&BO.d_first, sizeof(int) * BMAXS));
  HR_CUDA(cudaMalloc(&BO.d_map, sizeof(int) * BMAXS));
  HR_CUDA(cudaMalloc(&BO.d_isrc, sizeof(int) * BMAXS));
  HR_CUDA(cudaMalloc(&BO.d_shift, sizeof(double) * BMAXS));
  HR_CUDA(cudaMalloc(&BO.d_scale, sizeof(double) * BMAXS));
  HR_CUDA(cudaMalloc(&BO.d_ptrs, sizeof(void *) * BMAXS));
  HR_CUDA(cudaStreamCreateWithFlags(&BO.cap, cudaStreamNonBlocking));
  return 0;
}

static void drop_graph(BWork &w) {
  if (w.exec) cudaGraphExecDestroy(w.exec);
  w.exec = nullptr;
  w.g_op = -1;
}

void batch_release() {
  for (int q = 0; q < 2; q++) {
    BWork &w = BW[q];
    drop_graph(w);
    cudaFree(w.r); cudaFree(w.k); cudaFree(w.Mk); cudaFree(w.p);
    if (w.S) cudaFree(w.S);
    if (w.hS) cudaFreeHost(w.hS);
    w = BWork();
    cudaFree(BT.odd[q]);
    cudaFree(BT.even[q]);
  }
  BT = BatchTmp();
  for (int q = 0; q < 2; q++) {
    cudaFree(TC.U[q]); cudaFree(TC.dg[q]); cudaFree(TC.od[q]); cudaFree(TC.idg[q]); cudaFree(TC.iod[q]);
  }
  TC = TileCopies();
  cudaFree(BO.b); cudaFree(BO.x); cudaFree(BO.res); cudaFree(BO.rhs); cudaFree(BO.xf);
  cudaFree(BO.part); cudaFree(BO.dres); cudaFree(BO.d_src); cudaFree(BO.d_first); cudaFree(BO.d_map); cudaFree(BO.d_isrc);
  cudaFree(BO.d_shift); cudaFree(BO.d_scale); cudaFree(BO.d_ptrs);
  if (BO.hres_h) cudaFreeHost(BO.hres_h);
  if (BO.cap) cudaStreamDestroy(BO.cap);
  BO = BOuter();
}

// one batched CG iteration (the loop body of cg_mshift_core for every source)
template <typename R>
static int bcg_iteration(int op, double mass, int nb, int ns, long rows, BWork &w, void *x) {
  typedef typename C2<R>::T V;
  const int prec = sizeof(R) == 8 ? HRGPU_DOUBLE : HRGPU_FLOAT;
  const dim3 gb = bgrid(rows, nb), gs = bgrid(rows, ns);
  if (int rc = apply_op_b(op, prec, mass, w.Mk, w.k, nb, &w.S->state)) return rc;
  k_bdot<V><<<gb, BTHREADS, 0, L.stream>>>(&w.S->state, (const V *)w.k, (const V *)w.Mk, rows, nb, BO.part);
  k_bfold_alpha<<<1, BTHREADS, 0, L.stream>>>(w.S, BO.part, gb.x);
  k_bupd_r<V><<<gb, BTHREADS, 0, L.stream>>>(w.S, (V *)w.r, (const V *)w.Mk, rows, BO.part);
  k_bfold_lambda<<<1, BTHREADS, 0, L.stream>>>(w.S, BO.part, gb.x);
  k_bupd_xp<V><<<gs, BTHREADS, 0, L.stream>>>(w.S, (V *)x, (V *)w.p, (const V *)w.r, rows);
  k_bupd_k<V><<<gb, BTHREADS, 0, L.stream>>>(w.S, (V *)w.k, (const V *)w.r, rows);
  k_badvance<<<1, 1, 0, L.stream>>>(w.S);
  HR_LAUNCH_CHECK();
  return 0;
}

// capture BCHUNK iterations once for these buffers and arguments
// (the kernels of the graph hold these pointers: any change means a new capture)
template <typename R>
static void graph_key(BWork &w, void *x, const void **key) {
  const int prec = sizeof(R) == 8 ? HRGPU_DOUBLE : HRGPU_FLOAT;
  const void *k[12] = {w.r, w.k, w.Mk, w.p, x, BT.odd[prec], BT.even[prec], TC.U[prec],
                       TC.idg[prec], TC.dg[prec], BO.part, w.S};
  for (int i = 0; i < 12; i++) key[i] = k[i];
}

template <typename R>
static int bcg_graph(int op, double mass, int nb, int ns, long rows, BWork &w, void *x) {
  const void *key[12];
  graph_key<R>(w, x, key);
  bool same = w.exec && w.g_op == op && w.g_nb == nb && w.g_ns == ns && w.g_mass == mass;
  for (int i = 0; i < 12 && same; i++) same = key[i] == w.g_key[i];
  if (same) return 0;
  drop_graph(w);
  // tune the hopping kernels for this batch before the capture (Mk is scratch here)
  const int prec = sizeof(R) == 8 ? HRGPU_DOUBLE : HRGPU_FLOAT;
  if (int rc = apply_op_b(op, prec, mass, w.Mk, w.k, nb, nullptr)) return rc;
  cudaStream_t saved = L.stream;
  HR_CUDA(cudaStreamBeginCapture(BO.cap, cudaStreamCaptureModeRelaxed));
  L.stream = BO.cap;
  int rc = 0;
  for (int c = 0; c < BCHUNK && rc == 0; c++) rc = bcg_iteration<R>(op, mass, nb, ns, rows, w, x);
  L.stream = saved;
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(BO.cap, &graph);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess) return fail_cuda(e, "cudaStreamEndCapture", __FILE__, __LINE__);
  e = cudaGraphInstantiate(&w.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    w.exec = nullptr;
    return fail_cuda(e, "cudaGraphInstantiate", __FILE__, __LINE__);
  }
  w.g_op = op;
  w.g_nb = nb;
  w.g_ns = ns;
  w.g_mass = mass;
  for (int i = 0; i < 12; i++) w.g_key[i] = key[i];
  return 0;
}

// Batched multi-shift CG from x = 0 on nb sources (rhs, batch of precision R)
// for ns systems (src[j], shift[j]).  flt: HiRep's flt-core semantics (flags
// fixed, per-source err2[s]); otherwise flags are cleared as systems converge.
// iters[s] += iterations of source s.  Returns a status.
template <typename R>
static int bcg_core(int op, double mass, int nb, int ns, const int *src, const double *shift, int *flags,
                    const double *err2, int flt, int max_iter, const void *rhs, void *x, int *iters) {
  const int prec = sizeof(R) == 8 ? HRGPU_DOUBLE : HRGPU_FLOAT;
  BWork &w = BW[prec];
  const long rows = (long)4 * L.nf * L.ld;
  if (int rc = bouter_init()) return rc;
  if (int rc = ensure_batch_buf(&w.r, &w.hr, batch_bytes(prec, nb))) return rc;
  if (int rc = ensure_batch_buf(&w.k, &w.hk, batch_bytes(prec, nb))) return rc;
  if (int rc = ensure_batch_buf(&w.Mk, &w.hm, batch_bytes(prec, nb))) return rc;
  if (int rc = ensure_batch_buf(&w.p, &w.hp, batch_bytes(prec, ns))) return rc;
  if (!w.S) {
    HR_CUDA(cudaMalloc(&w.S, sizeof(BState)));
    HR_CUDA(cudaMallocHost(&w.hS, sizeof(BState)));
  }
  if (int rc = prepare_op_b(op, prec, mass, nb)) return rc;
  typedef typename C2<R>::T V;
  HR_CUDA(cudaMemcpyAsync(w.r, rhs, batch_bytes(prec, nb), cudaMemcpyDeviceToDevice, L.stream));
  HR_CUDA(cudaMemcpyAsync(w.k, rhs, batch_bytes(prec, nb), cudaMemcpyDeviceToDevice, L.stream));
  HR_CUDA(cudaMemsetAsync(x, 0, batch_bytes(prec, ns), L.stream));
  HR_CUDA(cudaMemcpyAsync(BO.d_isrc, src, sizeof(int) * ns, cudaMemcpyHostToDevice, L.stream));
  k_bspread<V><<<bgrid(rows, ns), BTHREADS, 0, L.stream>>>((V *)w.p, (const V *)w.r, BO.d_isrc, rows, ns, nb);
  HR_LAUNCH_CHECK();
  double nrm[BMAXB];
  if (int rc = bdot_host(w.r, w.r, prec, rows, nb, BO.part, BO.dres, BO.hres_h, nrm)) return rc;
  BState &h = *w.hS;
  memset(&h, 0, sizeof(BState));
  h.nb = nb;
  h.nsys = ns;
  h.max_iter = max_iter == 0 ? 200000 : max_iter;
  h.flt = flt;
  bool any = false;
  for (int s = 0; s < nb; s++) {
    BSrc &q = h.s[s];
    q.omega = 1.0;
    q.gamma = 0.0;
    q.delta = nrm[s];
    q.innorm2 = nrm[s];
    q.err2 = err2[s];
    bool work = false;
    for (int j = 0; j < ns; j++)
      if (src[j] == s && (!flt || flags[j])) work = true;
    q.state = (work && nrm[s] > 0.0) ? 0 : 2;  // a zero source is solved by x = 0
    any = any || q.state == 0;
  }
  for (int j = 0; j < ns; j++) {
    h.src[j] = src[j];
    h.shift[j] = shift[j];
    h.z1[j] = h.z2[j] = 1.0;
    h.flag[j] = flt ? flags[j] : (h.s[src[j]].state == 0 ? 1 : 0);
  }
  if (!any) return 0;
  HR_CUDA(cudaMemcpyAsync(w.S, &h, sizeof(BState), cudaMemcpyHostToDevice, L.stream));
  if (int rc = bcg_graph<R>(op, mass, nb, ns, rows, w, x)) return rc;
  for (;;) {
    HR_CUDA(cudaGraphLaunch(w.exec, L.stream));
    HR_CUDA(cudaMemcpyAsync(&h, w.S, sizeof(BState), cudaMemcpyDeviceToHost, L.stream));
    HR_CUDA(cudaStreamSynchronize(L.stream));
    if (h.state != 0) break;
  }
  unsigned long mvm = 0;
  int bad = -1;
  for (int s = 0; s < nb; s++) {
    iters[s] += h.s[s].iter;
    mvm += 4UL * h.s[s].iter;  // H^2: four hops
    if (h.s[s].state == 3) bad = s;
  }
  add_mvm(mvm);
  if (!flt)
    for (int j = 0; j < ns; j++) flags[j] = h.flag[j];
  if (bad >= 0) {
    set_error("cg_mshift_batch: breakdown of source %d at iteration %d (alpha=%g, |r|^2=%g)", bad, h.s[bad].iter,
              h.s[bad].alpha, h.s[bad].lambda);
    return HRGPU_E_BREAKDOWN;
  }
  return 0;
}

// res_j = b_src(j) - (M - shift_j) x_j for all systems (FP64), |res_j|^2 -> norm[j]
static int bresidual(int op, double mass, int nb, int ns, long rows, double *norm) {
  if (int rc = apply_op_b(op, HRGPU_DOUBLE, mass, BO.res, BO.x, ns, nullptr)) return rc;
  const dim3 g = bgrid(rows, ns);
  k_bres<<<g, BTHREADS, 0, L.stream>>>((double2 *)BO.res, (const double2 *)BO.b, (const double2 *)BO.x, BO.d_src,
                                       BO.d_shift, rows, ns, BO.part);
  k_bfold<<<1, BTHREADS, 0, L.stream>>>(BO.part, g.x, ns, BO.dres);
  HR_LAUNCH_CHECK();
  HR_CUDA(cudaMemcpyAsync(BO.hres_h, BO.dres, sizeof(double) * ns, cudaMemcpyDeviceToHost, L.stream));
  HR_CUDA(cudaStreamSynchronize(L.stream));
  for (int j = 0; j < ns; j++) norm[j] = BO.hres_h[j];
  add_mvm((unsigned long)ns * 4);
  return 0;
}

}  // namespace hrgpu

using namespace hrgpu;

extern "C" {

size_t hrgpu_batch_bytes(int prec, int nb) {
  if (!L.ready || nb <= 0 || (prec != HRGPU_DOUBLE && prec != HRGPU_FLOAT)) return 0;
  return batch_bytes(prec, nb);
}

int hrgpu_batch_pack(void *batch, const void *const *fields, int nb, int prec) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "batch_pack: lattice not initialised");
  HR_REQUIRE(batch && fields && nb > 0 && nb <= BMAXS && (prec == HRGPU_DOUBLE || prec == HRGPU_FLOAT), HRGPU_E_ARG,
             "batch_pack: bad arguments (nb = %d, 1..%d supported)", nb, BMAXS);
  for (int f = 0; f < nb; f++) HR_REQUIRE(fields[f] != nullptr, HRGPU_E_ARG, "batch_pack: field %d is NULL", f);
  if (int rc = bouter_init()) return rc;
  const long rows = (long)4 * L.nf * L.ld;
  HR_CUDA(cudaMemcpyAsync(BO.d_ptrs, fields, sizeof(void *) * nb, cudaMemcpyHostToDevice, L.stream));
  if (prec == HRGPU_DOUBLE)
    k_bpack<double2><<<bgrid(rows, nb), BTHREADS, 0, L.stream>>>((double2 *)batch, (const double2 *const *)BO.d_ptrs, rows, L.ld, 4 * L.nf, nb);
  else
    k_bpack<float2><<<bgrid(rows, nb), BTHREADS, 0, L.stream>>>((float2 *)batch, (const float2 *const *)BO.d_ptrs, rows, L.ld, 4 * L.nf, nb);
  HR_LAUNCH_CHECK();
  // the pointer array is reused by the next call: finish reading it first
  HR_CUDA(cudaStreamSynchronize(L.stream));
  return 0;
}

int hrgpu_batch_unpack(void *const *fields, const void *batch, int nb, int prec) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "batch_unpack: lattice not initialised");
  HR_REQUIRE(batch && fields && nb > 0 && nb <= BMAXS && (prec == HRGPU_DOUBLE || prec == HRGPU_FLOAT), HRGPU_E_ARG,
             "batch_unpack: bad arguments (nb = %d, 1..%d supported)", nb, BMAXS);
  for (int f = 0; f < nb; f++) HR_REQUIRE(fields[f] != nullptr, HRGPU_E_ARG, "batch_unpack: field %d is NULL", f);
  if (int rc = bouter_init()) return rc;
  const long rows = (long)4 * L.nf * L.ld;
  HR_CUDA(cudaMemcpyAsync(BO.d_ptrs, fields, sizeof(void *) * nb, cudaMemcpyHostToDevice, L.stream));
  if (prec == HRGPU_DOUBLE)
    k_bunpack<double2><<<bgrid(rows, nb), BTHREADS, 0, L.stream>>>((double2 *const *)BO.d_ptrs, (const double2 *)batch, rows, L.ld, 4 * L.nf, nb);
  else
    k_bunpack<float2><<<bgrid(rows, nb), BTHREADS, 0, L.stream>>>((float2 *const *)BO.d_ptrs, (const float2 *)batch, rows, L.ld, 4 * L.nf, nb);
  HR_LAUNCH_CHECK();
  HR_CUDA(cudaStreamSynchronize(L.stream));
  return 0;
}

int hrgpu_set_batch_variant(int variant) {
  HR_REQUIRE(variant >= -1 && variant < HOPB_VARIANTS, HRGPU_E_ARG, "set_batch_variant: variant must be -1..%d",
             HOPB_VARIANTS - 1);
  L.hopb_force = variant;
  return 0;
}

int hrgpu_batch_tuning(int prec, int epilogue, int nb, int *chosen, float *ms) {
  HR_REQUIRE(prec >= 0 && prec <= 1 && epilogue >= 0 && epilogue <= 2 && nb > 0 && nb <= HOPB_MAXNB && chosen && ms,
             HRGPU_E_ARG, "batch_tuning: bad arguments");
  *chosen = L.hopb_variant[prec][epilogue][nb] - 1;
  for (int v = 0; v < HOPB_VARIANTS; v++) ms[v] = L.hopb_tune_ms[prec][epilogue][nb][v];
  return 0;
}

int hrgpu_apply_op_batch(int op, int prec, double mass, void *out, const void *in, int nb) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "apply_op_batch: lattice not initialised");
  HR_REQUIRE(batch_op_ok(op), HRGPU_E_ARG, "apply_op_batch: operator %d has no batched form (even-odd operators only)", op);
  HR_REQUIRE(prec == HRGPU_DOUBLE || prec == HRGPU_FLOAT, HRGPU_E_ARG, "apply_op_batch: bad precision %d", prec);
  HR_REQUIRE(nb > 0 && nb <= BMAXS, HRGPU_E_ARG, "apply_op_batch: nb = %d (1..%d supported)", nb, BMAXS);
  HR_REQUIRE(out && in && out != in, HRGPU_E_ARG, "apply_op_batch: input and output batches must be different");
  const bool sq = op == HRGPU_OP_G5DPHI_EOPRE_SQ || op == HRGPU_OP_G5CPHI_EOPRE_SQ;
  if (int rc = apply_op_b(op, prec, mass, out, in, nb, nullptr)) return rc;
  add_mvm((unsigned long)nb * (sq ? 4 : 2));
  return 0;
}

// Batched cg_mshift / cg_mshift_flt.  Source s (in[s], FP64 even fields) is
// solved for the shifts shift[o_s .. o_s + nshift[s] - 1], o_s = nshift[0] +
// ... + nshift[s-1]: out[o_s + i] = (M - shift[o_s + i])^-1 in[s], all from a
// zero start.  flt = 1: FP32 inner solves inside FP64 defect correction.
int hrgpu_cg_mshift_batch(int op, double mass, int nsrc, const int *nshift, const double *shift, double err2,
                          int max_iter, const void *const *in, void *const *out, int flt, int *iters) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "cg_mshift_batch: lattice not initialised");
  HR_REQUIRE(op == HRGPU_OP_G5DPHI_EOPRE_SQ || op == HRGPU_OP_G5CPHI_EOPRE_SQ, HRGPU_E_ARG,
             "cg_mshift_batch: operator %d not supported (g5Dphi_eopre_sq, g5Cphi_eopre_sq)", op);
  HR_REQUIRE(nsrc > 0 && nsrc <= BMAXB, HRGPU_E_ARG, "cg_mshift_batch: nsrc = %d (1..%d supported)", nsrc, BMAXB);
  HR_REQUIRE(nshift && shift && in && out && iters, HRGPU_E_ARG, "cg_mshift_batch: NULL argument");
  HR_REQUIRE(err2 > 0.0, HRGPU_E_ARG, "cg_mshift_batch: err2 must be positive");
  int ns = 0;
  for (int s = 0; s < nsrc; s++) {
    HR_REQUIRE(nshift[s] > 0, HRGPU_E_ARG, "cg_mshift_batch: source %d has no shift", s);
    ns += nshift[s];
  }
  HR_REQUIRE(ns <= BMAXS, HRGPU_E_ARG, "cg_mshift_batch: %d systems (1..%d supported)", ns, BMAXS);
  for (int s = 0; s < nsrc; s++) HR_REQUIRE(in[s] != nullptr, HRGPU_E_ARG, "cg_mshift_batch: source %d is NULL", s);
  for (int j = 0; j < ns; j++) {
    HR_REQUIRE(out[j] != nullptr, HRGPU_E_ARG, "cg_mshift_batch: output %d is NULL", j);
    for (int s = 0; s < nsrc; s++) HR_REQUIRE(out[j] != in[s], HRGPU_E_ARG, "cg_mshift_batch: output %d aliases a source", j);
  }
  if (int rc = check_gauge(HRGPU_DOUBLE)) return rc;
  if (flt) {
    if (int rc = check_gauge(HRGPU_FLOAT)) return rc;
  }
  if (int rc = bouter_init()) return rc;
  std::vector<int> src(ns), flags(ns, 1);
  for (int s = 0, j = 0; s < nsrc; s++)
    for (int i = 0; i < nshift[s]; i++) src[j++] = s;
  for (int s = 0; s < nsrc; s++) iters[s] = 0;
  const long rows = (long)4 * L.nf * L.ld;
  if (int rc = ensure_batch_buf(&BO.b, &BO.hb, batch_bytes(HRGPU_DOUBLE, nsrc))) return rc;
  if (int rc = ensure_batch_buf(&BO.x, &BO.hx, batch_bytes(HRGPU_DOUBLE, ns))) return rc;
  if (int rc = ensure_batch_buf(&BO.res, &BO.hres, batch_bytes(HRGPU_DOUBLE, ns))) return rc;
  if (int rc = hrgpu_batch_pack(BO.b, in, nsrc, HRGPU_DOUBLE)) return rc;
  HR_CUDA(cudaMemcpyAsync(BO.d_src, src.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, L.stream));
  HR_CUDA(cudaMemcpyAsync(BO.d_shift, shift, sizeof(double) * ns, cudaMemcpyHostToDevice, L.stream));
  std::vector<double> innorm2(nsrc), norm(ns);
  if (int rc = bdot_host(BO.b, BO.b, HRGPU_DOUBLE, rows, nsrc, BO.part, BO.dres, BO.hres_h, innorm2.data())) return rc;
  for (int s = 0; s < nsrc; s++)
    HR_REQUIRE(isfinite(innorm2[s]), HRGPU_E_BREAKDOWN, "cg_mshift_batch: the norm of source %d is not finite (%g)", s,
               innorm2[s]);
  int status = 0;

  if (!flt) {
    // FP64 batch, then HiRep's check of every shift's true residual (cg_mshift.c:122-137)
    std::vector<double> e2(nsrc, err2);
    if (int rc = bcg_core<double>(op, mass, nsrc, ns, src.data(), shift, flags.data(), e2.data(), 0, max_iter, BO.b,
                                  BO.x, iters))
      return rc;
    if (int rc = bresidual(op, mass, nsrc, ns, rows, norm.data())) return rc;
    for (int j = 0; j < ns; j++)
      HR_REQUIRE(isfinite(norm[j]), HRGPU_E_BREAKDOWN, "cg_mshift_batch: the residual of system %d is not finite (%g)",
                 j, norm[j]);
    for (int j = 0; j < ns; j++) {
      iters[src[j]]++;
      flags[j] = (innorm2[src[j]] == 0.0 || norm[j] / innorm2[src[j]] <= err2) ? 1 : 0;
    }
    if (int rc = hrgpu_batch_unpack(out, BO.x, ns, HRGPU_DOUBLE)) return rc;
    // unconverged systems: HiRep's single-shift restart from the current solution (cg_mshift.c:170-179)
    for (int j = 0; j < ns; j++) {
      if (flags[j]) continue;
      int it = 0;
      int rc = hrgpu_cg_mshift(op, mass, 1, shift + j, err2, max_iter, in[src[j]], out + j, &it);
      iters[src[j]] += it;
      if (rc == HRGPU_E_NOCONV) status = rc;
      else if (rc) return rc;
    }
    return status;
  }

  // Defect correction (cg_mshift_flt.c:144-276).  The first correction pass
  // starts from x = 0, where the residuals of a source's shifts are all equal:
  // as in HiRep, one FP32 multi-shift solve per source corrects all its shifts.
  // After an FP32 inner solve the shifted residuals are collinear only to the
  // FP32 noise (about 1e-2 of their size at an inner tolerance of 1e-5), so
  // HiRep's projection onto the first residual gains two digits a pass for the
  // other shifts.  From the second pass on every unconverged system is
  // therefore corrected from its own residual: one single-shift Krylov space
  // each, all in one batch.
  if (int rc = ensure_batch_buf(&BO.rhs, &BO.hrhs, batch_bytes(HRGPU_FLOAT, ns))) return rc;
  if (int rc = ensure_batch_buf(&BO.xf, &BO.hxf, batch_bytes(HRGPU_FLOAT, ns))) return rc;
  HR_CUDA(cudaMemsetAsync(BO.x, 0, batch_bytes(HRGPU_DOUBLE, ns), L.stream));
  std::vector<int> sflag(ns, 1), first(ns, -1);
  int rounds = 0;
  for (;;) {
    if (int rc = bresidual(op, mass, nsrc, ns, rows, norm.data())) return rc;
    for (int j = 0; j < ns; j++)
      HR_REQUIRE(isfinite(norm[j]), HRGPU_E_BREAKDOWN, "cg_mshift_batch: the residual of system %d is not finite (%g)",
                 j, norm[j]);
    std::vector<int> todo;
    for (int j = 0; j < ns; j++) {
      const int s = src[j];
      iters[s]++;
      if (!sflag[j]) continue;
      if (innorm2[s] == 0.0 || norm[j] < innorm2[s] * err2) sflag[j] = 0;
      else todo.push_back(j);
    }
    if (todo.empty()) break;
    if (++rounds > 200) {
      if (int rc = hrgpu_batch_unpack(out, BO.x, ns, HRGPU_DOUBLE)) return rc;
      set_error("cg_mshift_batch: no convergence to err2=%g after %d defect-correction rounds", err2, rounds - 1);
      return HRGPU_E_NOCONV;
    }
    // the inner batch: Krylov spaces (isrc of each inner system, its shift),
    // right-hand side = res_firsts[k] * sscale[k], correction x_map[k] += c[k] xf_k
    std::vector<int> isrc, firsts, map, loc, owner;
    std::vector<double> ishift, sscale, c, e2;
    if (rounds == 1) {
      std::vector<int> firstj(nsrc, -1);
      bool need_proj = false;
      for (int j = 0; j < ns; j++) first[j] = -1;
      for (int j : todo) {
        const int s = src[j];
        if (firstj[s] < 0) firstj[s] = j;
        else {
          first[j] = firstj[s];
          need_proj = true;
        }
      }
      std::vector<int> slot(nsrc, -1);
      for (int s = 0; s < nsrc; s++) {
        if (firstj[s] < 0) continue;
        slot[s] = (int)firsts.size();
        firsts.push_back(firstj[s]);
        owner.push_back(s);
        sscale.push_back(1.0 / sqrt(norm[firstj[s]]));
        const double le = err2 / (norm[firstj[s]] / innorm2[s]) * 0.9;
        e2.push_back(le < 1.e-10 ? 1.e-10 : le);
      }
      std::vector<double> proj(ns, 0.0);
      if (need_proj) {
        // later shifts of a source: their residual along the normalised first
        // residual (cg_mshift_flt.c:205-208)
        HR_CUDA(cudaMemcpyAsync(BO.d_first, first.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, L.stream));
        const dim3 g = bgrid(rows, ns);
        k_bproj<<<g, BTHREADS, 0, L.stream>>>((const double2 *)BO.res, BO.d_first, rows, ns, BO.part);
        k_bfold<<<1, BTHREADS, 0, L.stream>>>(BO.part, g.x, ns, BO.dres);
        HR_LAUNCH_CHECK();
        HR_CUDA(cudaMemcpyAsync(BO.hres_h, BO.dres, sizeof(double) * ns, cudaMemcpyDeviceToHost, L.stream));
        HR_CUDA(cudaStreamSynchronize(L.stream));
        for (int j = 0; j < ns; j++) proj[j] = BO.hres_h[j];
      }
      for (int j = 0; j < ns; j++) {
        const int s = src[j];
        if (slot[s] < 0) continue;
        isrc.push_back(slot[s]);
        ishift.push_back(shift[j]);
        map.push_back(j);
        loc.push_back(sflag[j]);
        c.push_back(!sflag[j] ? 0.0 : first[j] < 0 ? sqrt(norm[j]) : proj[j] * sscale[slot[s]]);
      }
    } else {
      for (int j : todo) {
        const int k = (int)firsts.size();
        firsts.push_back(j);
        owner.push_back(src[j]);
        sscale.push_back(1.0 / sqrt(norm[j]));
        const double le = err2 / (norm[j] / innorm2[src[j]]) * 0.9;
        e2.push_back(le < 1.e-10 ? 1.e-10 : le);
        isrc.push_back(k);
        ishift.push_back(shift[j]);
        map.push_back(j);
        loc.push_back(1);
        c.push_back(sqrt(norm[j]));
      }
    }
    const int nbi = (int)firsts.size(), nsi = (int)isrc.size();
    HR_CUDA(cudaMemcpyAsync(BO.d_first, firsts.data(), sizeof(int) * nbi, cudaMemcpyHostToDevice, L.stream));
    HR_CUDA(cudaMemcpyAsync(BO.d_scale, sscale.data(), sizeof(double) * nbi, cudaMemcpyHostToDevice, L.stream));
    k_brhs<<<bgrid(rows, nbi), BTHREADS, 0, L.stream>>>((float2 *)BO.rhs, (const double2 *)BO.res, BO.d_first,
                                                        BO.d_scale, rows, nbi);
    HR_LAUNCH_CHECK();
    std::vector<int> it_in(nbi, 0);
    if (int rc = bcg_core<float>(op, mass, nbi, nsi, isrc.data(), ishift.data(), loc.data(), e2.data(), 1, max_iter,
                                 BO.rhs, BO.xf, it_in.data()))
      return rc;
    std::vector<int> it_src(nsrc, 0);
    for (int k = 0; k < nbi; k++) it_src[owner[k]] = it_src[owner[k]] > it_in[k] ? it_src[owner[k]] : it_in[k];
    for (int s = 0; s < nsrc; s++) iters[s] += it_src[s];
    HR_CUDA(cudaMemcpyAsync(BO.d_scale, c.data(), sizeof(double) * nsi, cudaMemcpyHostToDevice, L.stream));
    HR_CUDA(cudaMemcpyAsync(BO.d_map, map.data(), sizeof(int) * nsi, cudaMemcpyHostToDevice, L.stream));
    k_bacc<<<bgrid(rows, nsi), BTHREADS, 0, L.stream>>>((double2 *)BO.x, (const float2 *)BO.xf, BO.d_scale, BO.d_map,
                                                        rows, nsi);
    HR_LAUNCH_CHECK();
    // the host vectors above are read by the copies before the next round reuses the buffers
    HR_CUDA(cudaStreamSynchronize(L.stream));
  }
  return hrgpu_batch_unpack(out, BO.x, ns, HRGPU_DOUBLE);
}

}  // extern "C"
