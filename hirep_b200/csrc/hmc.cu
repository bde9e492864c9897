// hmc.cu -- the gauge-side pieces of an HMC step on the device, so that a
// molecular-dynamics step needs no host transfer of links or momenta:
//   momenta field            (suNg_av_field, suN_momenta)
//   force0 + staples         (LibHR/Update/force0.c:22-99, staples.c:22-70)
//   update_gauge_field       (LibHR/Update/field_update.c:18-66, ExpX in
//                             LibHR/Utils/suN_exp_group.c:358-378), with the
//                             reunitarisation of every 17th call
//                             (project_to_suNg, LibHR/Utils/suN_utils.c:76-150)
//                             and represent_gauge_field after it
//   local HMC action         (LibHR/Update/local_action.c:19-90, mon_pg.c:36-43,
//                             pf_local_action)
//   fermion_force_end into the device momenta.
// Fundamental links are L.Ug [4][NG*NG][2ld]; momenta [4][NG*NG-1][2ld].
#include <math.h>

#include "dirac.cuh"
#include "rng.cuh"

namespace hrgpu {

int launch_links_in(void *dev, const void *host_stage, int nel, int real, int ndir);  // lattice.cu
int links_out(void *host, const void *dev, int nel, int elem_bytes, int ndir);        // lattice.cu

static double2 *g_gT = nullptr;  // generators T_A [dimg][NG*NG] on the device
static double *g_loc = nullptr;  // local action [2ld]
static double *g_plaq = nullptr; // per-site plaquette sums [2ld] (avr_plaquette)
static int g_upd_count = 0;      // update_gauge_field's call counter (field_update.c:14-16)

void hmc_release() {
  cudaFree(g_gT);
  cudaFree(g_loc);
  cudaFree(g_plaq);
  g_gT = nullptr;
  g_loc = nullptr;
  g_plaq = nullptr;
  g_upd_count = 0;
}

static int hmc_setup() {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "lattice not initialised");
  if (!g_gT) {
    HR_CUDA(cudaMalloc(&g_gT, sizeof(double2) * L.dimg * L.ng * L.ng));
    HR_CUDA(cudaMemcpy(g_gT, L.h_gT, sizeof(double2) * L.dimg * L.ng * L.ng, cudaMemcpyHostToDevice));
  }
  if (!L.mom) {
    const size_t b = sizeof(double) * 4 * L.dimg * 2 * L.ld;
    HR_CUDA(cudaMalloc(&L.mom, b));
    HR_CUDA(cudaMemsetAsync(L.mom, 0, b, L.stream));
  }
  return 0;
}

// padding sites (cb >= VH) of a [.][2ld] array
__device__ __forceinline__ bool real_site(const Geo &g, long d) {
  return (d >= g.ld ? d - g.ld : d) < g.VH;
}

// f_A = Re Tr(conj(i T_A) w) / (1/2): the fundamental algebra projection
template <int N>
__device__ __forceinline__ double fund_project(const CMat<N> &w, const double2 *gT, int A) {
  double s = 0;
  const double2 *t = gT + (long)A * N * N;
#pragma unroll (SmallUnroll<N * N>::v)
  for (int k = 0; k < N * N; k++) {
    // conj(i t) = -i conj(t) = (-t.y) - i t.x; Re((a - i b)(c + i d)) = a c + b d
    s += -t[k].y * w.c[k].x + t[k].x * w.c[k].y;
  }
  return s * 2.0;
}

// force0: mom(x,mu) += coeff * proj(U(x,mu) S(x,mu)^+), S the six staples
template <int N>
__global__ void k_force0(double *mom, const double2 *Ug, const double2 *gT, Geo g, int dimg, double coeff) {
  const long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (d >= 2L * g.ld || !real_site(g, d)) return;
  const long lp = 2L * g.ld;
  int t, x, y, z;
  dev_coords(g, (int)d, t, x, y, z);
  const int xpmu = nbr_index(g, t, x, y, z, mu, 1);
  CMat<N> S, a, b, c;
#pragma unroll (SmallUnroll<N * N>::v)
  for (int k = 0; k < N * N; k++) S.c[k] = make_double2(0, 0);
  for (int i = 1; i < 4; i++) {
    const int nu = (mu + i) & 3;
    const int xpnu = nbr_index(g, t, x, y, z, nu, 1), xmnu = nbr_index(g, t, x, y, z, nu, -1);
    int t2, x2, y2, z2;
    dev_coords(g, xpmu, t2, x2, y2, z2);
    const int xpmumnu = nbr_index(g, t2, x2, y2, z2, nu, -1);
    // up: U(x,nu) U(x+nu,mu) U(x+mu,nu)^+
    mload<N, false>(a, Ug, nu, d, lp);
    mload<N, false>(b, Ug, mu, xpnu, lp);
    mmul<N, false, false>(c, a, b);
    mload<N, false>(a, Ug, nu, xpmu, lp);
    mmul<N, false, true>(b, c, a);
    madd<N>(S, b);
    // down: U(x-nu,nu)^+ U(x-nu,mu) U(x+mu-nu,nu)
    mload<N, false>(a, Ug, mu, xmnu, lp);
    mload<N, false>(b, Ug, nu, xpmumnu, lp);
    mmul<N, false, false>(c, a, b);
    mload<N, false>(a, Ug, nu, xmnu, lp);
    mmul<N, true, false>(b, a, c);
    madd<N>(S, b);
  }
  mload<N, false>(a, Ug, mu, d, lp);
  mmul<N, false, true>(b, a, S);
  for (int A = 0; A < dimg; A++) mom[((long)mu * dimg + A) * lp + d] += coeff * fund_project<N>(b, gT, A);
}

// U(x,mu) <- exp(dt sum_A mom_A iT_A) U(x,mu)   (ExpX)
template <int N>
__global__ void k_update_gauge(double2 *Ug, const double *mom, const double2 *gT, Geo g, int dimg, double dt) {
  const long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (d >= 2L * g.ld || !real_site(g, d)) return;
  const long lp = 2L * g.ld;
  CMat<N> X, E, U, R;
  for (int k = 0; k < N * N; k++) X.c[k] = make_double2(0, 0);
  for (int A = 0; A < dimg; A++) {
    const double h = dt * mom[((long)mu * dimg + A) * lp + d];
    const double2 *t = gT + (long)A * N * N;
    for (int k = 0; k < N * N; k++) {  // h * i t
      X.c[k].x -= h * t[k].y;
      X.c[k].y += h * t[k].x;
    }
  }
  mexp_sq<N>(E, X);  // the reference's suNg_Exp is exact to rounding as well
  mload<N, false>(U, Ug, mu, d, lp);
  mmul<N, false, false>(R, E, U);
  for (int k = 0; k < N * N; k++) Ug[((long)mu * N * N + k) * lp + d] = R.c[k];
}

// project_to_suNg: Gram-Schmidt of the rows, then times det^(-1/N) (principal branch)
template <int N>
__global__ void k_project_suNg(double2 *Ug, Geo g) {
  const long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (d >= 2L * g.ld || !real_site(g, d)) return;
  const long lp = 2L * g.ld;
  CMat<N> m;
  mload<N, false>(m, Ug, mu, d, lp);
  double nrm = 0;
  for (int k = 0; k < N * N; k++) nrm += m.c[k].x * m.c[k].x + m.c[k].y * m.c[k].y;
  if (nrm < 1.e-28) return;
  for (int i = 0; i < N; i++) {
    for (int j = 0; j < i; j++) {
      double2 zz = make_double2(0, 0);
      for (int k = 0; k < N; k++) cmacc(zz, m.c[j * N + k], m.c[i * N + k]);  // conj(v_j) . v_i
      for (int k = 0; k < N; k++) {
        const double2 vj = m.c[j * N + k];
        m.c[i * N + k].x -= zz.x * vj.x - zz.y * vj.y;
        m.c[i * N + k].y -= zz.x * vj.y + zz.y * vj.x;
      }
    }
    double q = 0;
    for (int k = 0; k < N; k++) q += m.c[i * N + k].x * m.c[i * N + k].x + m.c[i * N + k].y * m.c[i * N + k].y;
    q = 1.0 / sqrt(q);
    for (int k = 0; k < N; k++) m.c[i * N + k] = make_double2(m.c[i * N + k].x * q, m.c[i * N + k].y * q);
  }
  // determinant by elimination with partial pivoting
  CMat<N> a = m;
  double2 det = make_double2(1, 0);
  for (int i = 0; i < N; i++) {
    int p = i;
    double best = a.c[i * N + i].x * a.c[i * N + i].x + a.c[i * N + i].y * a.c[i * N + i].y;
    for (int r = i + 1; r < N; r++) {
      const double v = a.c[r * N + i].x * a.c[r * N + i].x + a.c[r * N + i].y * a.c[r * N + i].y;
      if (v > best) {
        best = v;
        p = r;
      }
    }
    if (p != i) {
      for (int k = 0; k < N; k++) {
        const double2 tmp = a.c[i * N + k];
        a.c[i * N + k] = a.c[p * N + k];
        a.c[p * N + k] = tmp;
      }
      det = make_double2(-det.x, -det.y);
    }
    const double2 piv = a.c[i * N + i];
    det = make_double2(det.x * piv.x - det.y * piv.y, det.x * piv.y + det.y * piv.x);
    const double pn = piv.x * piv.x + piv.y * piv.y;
    for (int r = i + 1; r < N; r++) {
      const double2 ar = a.c[r * N + i];
      const double2 f = make_double2((ar.x * piv.x + ar.y * piv.y) / pn, (ar.y * piv.x - ar.x * piv.y) / pn);
      for (int k = i; k < N; k++) {
        const double2 aik = a.c[i * N + k];
        a.c[r * N + k].x -= f.x * aik.x - f.y * aik.y;
        a.c[r * N + k].y -= f.x * aik.y + f.y * aik.x;
      }
    }
  }
  const double r = pow(sqrt(det.x * det.x + det.y * det.y), -1.0 / N);
  const double th = -atan2(det.y, det.x) / N;
  const double2 f = make_double2(r * cos(th), r * sin(th));
  for (int k = 0; k < N * N; k++) {
    const double2 v = m.c[k];
    Ug[((long)mu * N * N + k) * lp + d] = make_double2(v.x * f.x - v.y * f.y, v.x * f.y + v.y * f.x);
  }
}

// local action of the momenta (mom may be null) and the plaquette gauge
// action; mode 0 (NEW): loc = value, mode 1 (DELTA): loc = value - loc
template <int N>
__global__ void k_local_action(double *loc, const double *mom, const double2 *Ug, Geo g, int dimg, double beta,
                               double fund_norm2, int mode) {
  const long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= 2L * g.ld) return;
  if (!real_site(g, d)) {
    loc[d] = 0.0;
    return;
  }
  const long lp = 2L * g.ld;
  double a = 0;
  if (mom)
    for (int mu = 0; mu < 4; mu++)
      for (int A = 0; A < dimg; A++) {
        const double p = mom[((long)mu * dimg + A) * lp + d];
        a += p * p;
      }
  a *= 0.5 * fund_norm2;
  int t, x, y, z;
  dev_coords(g, (int)d, t, x, y, z);
  double pl = 0;
  CMat<N> u1, u2, w1, w2;
  for (int mu = 1; mu < 4; mu++)
    for (int nu = 0; nu < mu; nu++) {
      mload<N, false>(u1, Ug, mu, d, lp);
      mload<N, false>(u2, Ug, nu, nbr_index(g, t, x, y, z, mu, 1), lp);
      mmul<N, false, false>(w1, u1, u2);
      mload<N, false>(u1, Ug, nu, d, lp);
      mload<N, false>(u2, Ug, mu, nbr_index(g, t, x, y, z, nu, 1), lp);
      mmul<N, false, false>(w2, u1, u2);
      for (int k = 0; k < N * N; k++) pl += w1.c[k].x * w2.c[k].x + w1.c[k].y * w2.c[k].y;  // Re Tr(w1 w2^+)
    }
  const double v = a - beta / N * pl;
  loc[d] = mode ? v - loc[d] : v;
}

// loc(x) += |pf(x)|^2 for a parity (or full) field
__global__ void k_clover_la_logdet(double *loc, const double *ldet, double nf, Geo g) {
  const long cb = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (cb >= g.VH) return;
  const long d = g.ld + cb;  // odd site
  loc[d] -= nf * log(ldet[d]);
}

__global__ void k_pf_local_action(double *loc, const double2 *pf, int par, int nf, Geo g) {
  const long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long nsites = (par == HRGPU_FULL ? 2L : 1L) * g.ld;
  if (d >= nsites) return;
  const int p = par == HRGPU_FULL ? (int)(d / g.ld) : par;
  const long cb = par == HRGPU_FULL ? d - (long)p * g.ld : d;
  if (cb >= g.VH) return;
  const double2 *f = pf + (par == HRGPU_FULL ? (long)p * 4 * nf * g.ld : 0) + cb;
  double a = 0;
  for (int c = 0; c < 4 * nf; c++) {
    const double2 v = f[(long)c * g.ld];
    a += v.x * v.x + v.y * v.y;
  }
  loc[(long)p * g.ld + cb] += a;
}

__global__ void k_sum_partials(const double *v, long n, double *partials) {
  __shared__ double sh[RED_THREADS];
  double s = 0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) s += v[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}

__global__ void k_add(double *a, const double *b, long n) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) a[i] += b[i];
}

#define HR_NG_DISPATCH(NGV, CALL)                                                       \
  do {                                                                                  \
    switch (NGV) {                                                                      \
      case 2: { constexpr int N_ = 2; CALL; } break;                                     \
      case 3: { constexpr int N_ = 3; CALL; } break;                                     \
      case 4: { constexpr int N_ = 4; CALL; } break;                                     \
      case 5: { constexpr int N_ = 5; CALL; } break;                                     \
      case 6: { constexpr int N_ = 6; CALL; } break;                                     \
      case 7: { constexpr int N_ = 7; CALL; } break;                                     \
      case 8: { constexpr int N_ = 8; CALL; } break;                                     \
      default: set_error("no HMC kernel for NG=%d", (int)(NGV)); return HRGPU_E_NF;       \
    }                                                                                   \
  } while (0)

static unsigned nb128(long n) { return (unsigned)((n + 127) / 128); }

// ---------------------------------------------------------------------------
// Gaussian draws on the device (rng.cuh): the generator key is set by
// hrgpu_random_seed, and every draw takes the next stream number, so
// successive draws are independent and a seed replays its sequence of draws.
// ---------------------------------------------------------------------------
static uint32_t g_rng_key[2] = {0u, 0u};
static uint64_t g_rng_stream = 0;

static unsigned rng_grid(long n) {
  const long b = (n + 255) / 256;
  return (unsigned)(b < 148L * 16 ? b : 148L * 16);
}

// element e of a spinor field ([planes][ld] complex): a complex Gaussian of
// variance 2 scale^2 at real sites, zero in the padding (cb >= VH)
template <typename V>
__global__ void k_gauss_spinor(V *s, long n, int ld, int VH, uint64_t stream, uint32_t k0, uint32_t k1, double scale) {
  typedef decltype(s[0].x) R;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    V o;
    o.x = (R)0;
    o.y = (R)0;
    if ((int)(e % ld) < VH) {
      const double2 z = gauss_pair((uint64_t)e, stream, k0, k1);
      o.x = (R)(scale * z.x);
      o.y = (R)(scale * z.y);
    }
    s[e] = o;
  }
}

// momenta [4][dimg][2 ld] doubles: entries 2q and 2q+1 (one row, as 2 ld is
// even) take the two Gaussians of block q, times scale; padding sites stay zero
__global__ void k_gauss_momenta(double *mom, long npairs, int ld, int VH, uint64_t stream, uint32_t k0, uint32_t k1,
                                double scale) {
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < npairs; q += (long)gridDim.x * blockDim.x) {
    const double2 z = gauss_pair((uint64_t)q, stream, k0, k1);
    const long d0 = (2 * q) % (2L * ld);
    const long c0 = d0 >= ld ? d0 - ld : d0, c1 = d0 + 1 >= ld ? d0 + 1 - ld : d0 + 1;
    mom[2 * q] = c0 < VH ? scale * z.x : 0.0;
    mom[2 * q + 1] = c1 < VH ? scale * z.y : 0.0;
  }
}

}  // namespace hrgpu

using namespace hrgpu;

extern "C" {

int hrgpu_momenta_set(const double *host) {
  if (int rc = hmc_setup()) return rc;
  HR_REQUIRE(host, HRGPU_E_ARG, "momenta_set: NULL field");
  const size_t bytes = sizeof(double) * (size_t)L.V * 4 * L.dimg;
  if (int rc = ensure_stage(bytes)) return rc;
  HR_CUDA(cudaMemcpyAsync(L.stage, host, bytes, cudaMemcpyHostToDevice, L.stream));
  if (int rc = launch_links_in(L.mom, L.stage, L.dimg, 1, 4)) return rc;
  HR_CUDA(cudaStreamSynchronize(L.stream));  // the staging buffer is reused by the next transfer
  return 0;
}

int hrgpu_momenta_get(double *host) {
  if (int rc = hmc_setup()) return rc;
  HR_REQUIRE(host, HRGPU_E_ARG, "momenta_get: NULL field");
  return links_out(host, L.mom, L.dimg, 8, 4);
}

int hrgpu_random_seed(unsigned long long seed) {
  g_rng_key[0] = (uint32_t)seed;
  g_rng_key[1] = (uint32_t)(seed >> 32);
  g_rng_stream = 0;
  return 0;
}

// gaussian_momenta (LibHR/Update/random_momenta.c:18-38): every generator
// component N(0, 1) / sqrt(C(fund)); apply_BCs_on_momentum_field is the
// identity for the periodic / antiperiodic boundary conditions of this library
int hrgpu_gaussian_momenta(void) {
  if (int rc = hmc_setup()) return rc;
  const long n = 4L * L.dimg * 2L * L.ld;
  k_gauss_momenta<<<rng_grid(n / 2), 256, 0, L.stream>>>(L.mom, n / 2, L.ld, (int)L.VH, g_rng_stream++, g_rng_key[0],
                                                         g_rng_key[1], 1.0 / sqrt(L.fund_norm2));
  HR_LAUNCH_CHECK();
  return 0;
}

// gaussian_spinor_field (LibHR/Update/random_spinor_field.c:14-25): every real
// component N(0, 1) / sqrt(2); the FP32 field is the FP64 draw rounded
// (gaussian_spinor_field_flt, :27-36, draws in single precision)
int hrgpu_gaussian_spinor_field(int par, int prec, void *s) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "gaussian_spinor_field: lattice not initialised");
  HR_REQUIRE(s && par >= 0 && par <= 2 && (prec == HRGPU_DOUBLE || prec == HRGPU_FLOAT), HRGPU_E_ARG,
             "gaussian_spinor_field: bad arguments");
  const long n = (long)spinor_elems(par);
  const double c1 = 1.0 / sqrt(2.0);
  if (prec == HRGPU_DOUBLE)
    k_gauss_spinor<double2><<<rng_grid(n), 256, 0, L.stream>>>((double2 *)s, n, L.ld, (int)L.VH, g_rng_stream++,
                                                               g_rng_key[0], g_rng_key[1], c1);
  else
    k_gauss_spinor<float2><<<rng_grid(n), 256, 0, L.stream>>>((float2 *)s, n, L.ld, (int)L.VH, g_rng_stream++,
                                                              g_rng_key[0], g_rng_key[1], c1);
  HR_LAUNCH_CHECK();
  return 0;
}

int hrgpu_gauge_get(double *u_host) {
  HR_REQUIRE(L.ready && L.have_fund, HRGPU_E_STATE, "gauge_get: no fundamental gauge field");
  HR_REQUIRE(u_host, HRGPU_E_ARG, "gauge_get: NULL field");
  return links_out(u_host, L.Ug, L.ng * L.ng, 16, 4);
}

int hrgpu_force0(double dt, double beta) {
  if (int rc = hmc_setup()) return rc;
  HR_REQUIRE(L.have_fund, HRGPU_E_STATE, "force0: no fundamental gauge field");
  const Geo g = make_geo();
  const double coeff = -dt * beta / L.ng;
  HR_NG_DISPATCH(L.ng, (k_force0<N_><<<dim3(nb128(2L * L.ld), 4), 128, 0, L.stream>>>(L.mom, L.Ug, g_gT, g, L.dimg, coeff)));
  HR_LAUNCH_CHECK();
  return 0;
}

int hrgpu_project_gauge_field(void) {
  HR_REQUIRE(L.ready && L.have_fund, HRGPU_E_STATE, "project_gauge_field: no fundamental gauge field");
  const Geo g = make_geo();
  HR_NG_DISPATCH(L.ng, (k_project_suNg<N_><<<dim3(nb128(2L * L.ld), 4), 128, 0, L.stream>>>(L.Ug, g)));
  HR_LAUNCH_CHECK();
  fund_links_changed();
  return 0;
}

int hrgpu_update_gauge_field(double dt) {
  if (int rc = hmc_setup()) return rc;
  HR_REQUIRE(L.have_fund, HRGPU_E_STATE, "update_gauge_field: no fundamental gauge field");
  const Geo g = make_geo();
  HR_NG_DISPATCH(L.ng, (k_update_gauge<N_><<<dim3(nb128(2L * L.ld), 4), 128, 0, L.stream>>>(L.Ug, L.mom, g_gT, g, L.dimg, dt)));
  HR_LAUNCH_CHECK();
  fund_links_changed();
  // reunitarise every 17th call, as the reference's counter does (field_update.c:45-57)
  if (g_upd_count & 16) {
    g_upd_count = 0;
    if (int rc = hrgpu_project_gauge_field()) return rc;
  } else {
    g_upd_count++;
  }
  return hrgpu_represent_gauge_field(L.bc_t);
}

int hrgpu_local_hmc_action(int type, double beta) {
  if (int rc = hmc_setup()) return rc;
  HR_REQUIRE(type == HRGPU_ACTION_NEW || type == HRGPU_ACTION_DELTA, HRGPU_E_ARG,
             "local_hmc_action: type must be HRGPU_ACTION_NEW or HRGPU_ACTION_DELTA");
  HR_REQUIRE(L.have_fund, HRGPU_E_STATE, "local_hmc_action: no fundamental gauge field");
  if (!g_loc) {
    HR_CUDA(cudaMalloc(&g_loc, sizeof(double) * 2 * L.ld));
    HR_CUDA(cudaMemsetAsync(g_loc, 0, sizeof(double) * 2 * L.ld, L.stream));
  }
  const Geo g = make_geo();
  HR_NG_DISPATCH(L.ng, (k_local_action<N_><<<nb128(2L * L.ld), 128, 0, L.stream>>>(g_loc, L.mom, L.Ug, g, L.dimg, beta, L.fund_norm2, type)));
  HR_LAUNCH_CHECK();
  return 0;
}

int hrgpu_pf_local_action(const void *pf, int par) {
  HR_REQUIRE(L.ready && g_loc, HRGPU_E_STATE, "pf_local_action: call hrgpu_local_hmc_action first");
  HR_REQUIRE(pf && par >= 0 && par <= 2, HRGPU_E_ARG, "pf_local_action: bad arguments");
  const Geo g = make_geo();
  const long n = (par == HRGPU_FULL ? 2L : 1L) * L.ld;
  k_pf_local_action<<<nb128(n), 128, 0, L.stream>>>(g_loc, (const double2 *)pf, par, L.nf, g);
  HR_LAUNCH_CHECK();
  return 0;
}

static int sum_sites(const double *v, double *sum) {
  const long n = 2L * L.ld;
  long b = (n + RED_THREADS - 1) / RED_THREADS;
  if (b > RED_MAX_BLOCKS) b = RED_MAX_BLOCKS;
  k_sum_partials<<<(unsigned)b, RED_THREADS, 0, L.stream>>>(v, n, L.partials);
  HR_LAUNCH_CHECK();
  return finish_reduction((int)b, 1, sum);
}

// clover_la_logdet (clover_tools.c:312-331): loc -= nf log det D_oo on the odd
// sites, det D_oo the product of the LDL diagonals of the two chiral blocks of
// (4+m) + A at the mass given
int hrgpu_clover_la_logdet(double nf, double mass) {
  HR_REQUIRE(L.ready && g_loc, HRGPU_E_STATE, "clover_la_logdet: call hrgpu_local_hmc_action first");
  HR_REQUIRE(L.clover, HRGPU_E_STATE, "clover_la_logdet: no clover term");
  HR_REQUIRE(!L.expclover, HRGPU_E_STATE,
             "clover_la_logdet: the exponential clover term has no log-det term (its blocks are traceless)");
  if (int rc = clover_prepare(mass, HRGPU_DOUBLE)) return rc;
  const Geo g = make_geo();
  k_clover_la_logdet<<<nb128(g.VH), 128, 0, L.stream>>>(g_loc, L.cl_ldet, nf, g);
  HR_LAUNCH_CHECK();
  return 0;
}

int hrgpu_local_action_sum(double *sum) {
  HR_REQUIRE(L.ready && g_loc, HRGPU_E_STATE, "local_action_sum: no local action");
  HR_REQUIRE(sum, HRGPU_E_ARG, "local_action_sum: NULL output");
  return sum_sites(g_loc, sum);
}

int hrgpu_local_action_get(double *host) {
  HR_REQUIRE(L.ready && g_loc, HRGPU_E_STATE, "local_action_get: no local action");
  HR_REQUIRE(host, HRGPU_E_ARG, "local_action_get: NULL output");
  return links_out(host, g_loc, 1, 8, 1);
}

// avr_plaquette (LibHR/Observables/avr_plaquette.c:84-110): the mean of Re Tr P / NG
int hrgpu_avr_plaquette(double *plaq) {
  if (int rc = hmc_setup()) return rc;
  HR_REQUIRE(plaq, HRGPU_E_ARG, "avr_plaquette: NULL output");
  HR_REQUIRE(L.have_fund, HRGPU_E_STATE, "avr_plaquette: no fundamental gauge field");
  if (!g_plaq) HR_CUDA(cudaMalloc(&g_plaq, sizeof(double) * 2 * L.ld));
  const Geo g = make_geo();
  // the gauge part of the local action with beta = -NG and no momenta: the plaquette sum
  HR_NG_DISPATCH(L.ng, (k_local_action<N_><<<nb128(2L * L.ld), 128, 0, L.stream>>>(g_plaq, nullptr, L.Ug, g, L.dimg, -(double)L.ng, L.fund_norm2, 0)));
  HR_LAUNCH_CHECK();
  double s = 0;
  if (int rc = sum_sites(g_plaq, &s)) return rc;
  *plaq = s / (6.0 * L.ng * (double)L.V);
  return 0;
}

// fermion_force_end (force_fermion_core.c:964-993) into the device momenta
int hrgpu_fermion_force_end_momenta(double dt) {
  if (int rc = hmc_setup()) return rc;
  HR_REQUIRE(L.force_sum, HRGPU_E_STATE, "fermion_force_end_momenta: no force accumulated");
  if (int rc = fermion_force_finish(dt)) return rc;
  const long n = 4L * L.dimg * 2 * L.ld;
  k_add<<<nb128(n) < 148 * 16 ? nb128(n) : 148 * 16, 128, 0, L.stream>>>(L.mom, L.force_sum, n);
  HR_LAUNCH_CHECK();
  return 0;
}

}  // extern "C"
