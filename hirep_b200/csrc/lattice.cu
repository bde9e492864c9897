// lattice.cu -- library state, lattice setup, layout translation at the boundary,
// representation generators, reductions.
#include <stdarg.h>
#include <string.h>

#include <complex>
#include <vector>

#include <cuda_bf16.h>

#include "hrgpu_internal.cuh"

namespace hrgpu {

Lattice L;
static std::string g_err;
static int g_device = -1;
static cudaStream_t g_own_stream = 0;
static bool g_stream_chosen = false;

void set_error(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
}

int fail_cuda(cudaError_t e, const char *what, const char *file, int line) {
  set_error("CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what, file, line);
  return HRGPU_E_CUDA;
}

int ensure_tmp(void **p, size_t bytes) {
  if (*p) return 0;
  HR_CUDA(cudaMalloc(p, bytes));
  HR_CUDA(cudaMemsetAsync(*p, 0, bytes, L.stream));
  return 0;
}

int ensure_stage(size_t bytes) {
  if (L.stage_bytes >= bytes) return 0;
  if (L.stage) HR_CUDA(cudaFree(L.stage));
  L.stage = nullptr;
  HR_CUDA(cudaMalloc(&L.stage, bytes));
  L.stage_bytes = bytes;
  return 0;
}

Geo make_geo() {
  Geo g;
  g.X = L.X; g.Y = L.Y; g.Z = L.Z; g.T = L.T;
  g.Xh = L.X / 2;
  g.ld = L.ld;
  g.VH = (int)L.VH;
  return g;
}

static void free_ptr(void *p) {
  if (p) cudaFree(p);
}

static void free_all() {
  cg_release();
  void *ptrs[] = {L.d_h2d, L.d_d2h, L.U, L.Uf, L.Ubf, L.Ug, L.Ugf, L.mom, L.cl_term, L.cl_dg, L.cl_od, L.cl_idg, L.cl_iod,
                  L.cl_dg_f, L.cl_idg_f, L.cl_od_f, L.cl_iod_f, L.cl_ldet, L.force_sum, L.cl_force, L.d_proj_off,
                  L.d_proj_k, L.d_proj_c, L.d_projk_off, L.d_projk_A, L.d_projk_c, L.partials, L.d_scalars, L.tmp_o, L.tmp_e, L.tmp_e2, L.tmp_full,
                  L.tmp_full2, L.tmp_o_f, L.tmp_e_f, L.tmp_full_f, L.stage, L.hop_err, L.hopb_err};
  for (void *p : ptrs) free_ptr(p);
  if (L.h_partials) cudaFreeHost(L.h_partials);
  delete[] L.h_h2d;
  delete[] L.h_rT;
  delete[] L.h_gT;
  cudaStream_t s = L.stream;
  L = Lattice();
  L.stream = s;
}

// ---------------------------------------------------------------------------
// generators (same conventions as HiRep's autosun generator:
// Make/Utils/autosun/sun.h:27-74 for T_A with Tr T_A T_B = delta/2,
// fundamental.h, adjoint.h, symmetric.h, antisymmetric.h for R(iT_A) and C(R))
// ---------------------------------------------------------------------------
typedef std::complex<double> cd;
typedef std::vector<cd> Mat;

static Mat mmul(int n, const Mat &a, const Mat &b) {
  Mat c(n * n, 0.0);
  for (int i = 0; i < n; i++)
    for (int k = 0; k < n; k++)
      for (int j = 0; j < n; j++) c[i * n + j] += a[i * n + k] * b[k * n + j];
  return c;
}

static cd mtrace(int n, const Mat &a) {
  cd s = 0;
  for (int i = 0; i < n; i++) s += a[i * n + i];
  return s;
}

static void build_generators(std::vector<Mat> &gT, std::vector<Mat> &rT, double &rnorm) {
  const int N = L.ng, F = L.nf, D = N * N - 1;
  gT.assign(D, Mat(N * N, 0.0));
  int A = 0;
  for (int a = 0; a < N; a++)
    for (int b = 0; b < N; b++) {
      if (a > b) { gT[A][a * N + b] = 1.0; gT[A][b * N + a] = 1.0; A++; }
      else if (a < b) { gT[A][a * N + b] = cd(0, 1); gT[A][b * N + a] = cd(0, -1); A++; }
      else if (a != 0) {
        double nn = sqrt(2. / (a * (a + 1.)));
        for (int k = 0; k < a; k++) gT[A][k * N + k] = nn;
        gT[A][a * N + a] = -a * nn;
        A++;
      }
    }
  for (auto &m : gT)
    for (auto &x : m) x *= 0.5;
  rT.assign(D, Mat(F * F, 0.0));
  if (L.repr == HRGPU_FUND) {
    for (int C = 0; C < D; C++)
      for (int k = 0; k < N * N; k++) rT[C][k] = cd(0, 1) * gT[C][k];
    rnorm = 0.5;
    return;
  }
  std::vector<Mat> e(F, Mat(N * N, 0.0));
  if (L.repr == HRGPU_ADJ) {
    for (int C = 0; C < F; C++)
      for (int k = 0; k < N * N; k++) e[C][k] = gT[C][k] / sqrt(0.5);
    for (int C = 0; C < D; C++)
      for (int a = 0; a < F; a++) {
        Mat t1 = mmul(N, e[a], gT[C]), t2 = mmul(N, gT[C], e[a]);
        Mat c(N * N);
        for (int k = 0; k < N * N; k++) c[k] = t2[k] - t1[k];
        for (int b = 0; b < F; b++) rT[C][b * F + a] = -mtrace(N, mmul(N, c, e[b])).imag();
      }
    rnorm = 2. * 0.5 * N;
    return;
  }
  int C = 0;
  if (L.repr == HRGPU_SYM) {
    for (int a = 0; a < N; a++) {
      for (int b = 0; b < a; b++) {
        e[C][a * N + b] = sqrt(.5);
        e[C][b * N + a] = sqrt(.5);
        C++;
      }
      e[C][a * N + a] = 1.0;
      C++;
    }
  } else {
    for (int a = 1; a < N; a++)
      for (int b = 0; b < a; b++) {
        e[C][a * N + b] = sqrt(.5);
        e[C][b * N + a] = -sqrt(.5);
        C++;
      }
  }
  cd fac = (L.repr == HRGPU_SYM) ? cd(0, 2) : cd(0, -2);
  for (C = 0; C < D; C++)
    for (int a = 0; a < F; a++) {
      Mat t = mmul(N, e[a], gT[C]);
      for (int b = 0; b < F; b++) rT[C][a * F + b] = fac * mtrace(N, mmul(N, t, e[b]));
    }
  rnorm = (L.repr == HRGPU_SYM) ? (N + 2.) * 0.5 : (N - 2.) * 0.5;
}

static int upload_projection_tables() {
  std::vector<Mat> gT, rT;
  double rnorm = 0;
  build_generators(gT, rT, rnorm);
  const int D = L.dimg, F2 = L.nf * L.nf, N2 = L.ng * L.ng;
  L.repr_norm2 = rnorm;
  L.fund_norm2 = 0.5;
  L.h_rT = new double[(size_t)D * F2 * 2];
  L.h_gT = new double[(size_t)D * N2 * 2];
  std::vector<int> off(D + 1, 0), ks;
  std::vector<double2> cs;
  for (int A = 0; A < D; A++) {
    for (int k = 0; k < F2; k++) {
      L.h_rT[((size_t)A * F2 + k) * 2 + 0] = rT[A][k].real();
      L.h_rT[((size_t)A * F2 + k) * 2 + 1] = rT[A][k].imag();
      if (std::abs(rT[A][k]) > 1e-14) {
        cd c = std::conj(rT[A][k]) / rnorm;
        ks.push_back(k);
        cs.push_back(make_double2(c.real(), c.imag()));
      }
    }
    off[A + 1] = (int)ks.size();
    for (int k = 0; k < N2; k++) {
      L.h_gT[((size_t)A * N2 + k) * 2 + 0] = gT[A][k].real();
      L.h_gT[((size_t)A * N2 + k) * 2 + 1] = gT[A][k].imag();
    }
  }
  HR_CUDA(cudaMalloc(&L.d_proj_off, sizeof(int) * (D + 1)));
  HR_CUDA(cudaMalloc(&L.d_proj_k, sizeof(int) * ks.size()));
  HR_CUDA(cudaMalloc(&L.d_proj_c, sizeof(double2) * cs.size()));
  HR_CUDA(cudaMemcpy(L.d_proj_off, off.data(), sizeof(int) * (D + 1), cudaMemcpyHostToDevice));
  HR_CUDA(cudaMemcpy(L.d_proj_k, ks.data(), sizeof(int) * ks.size(), cudaMemcpyHostToDevice));
  HR_CUDA(cudaMemcpy(L.d_proj_c, cs.data(), sizeof(double2) * cs.size(), cudaMemcpyHostToDevice));
  // inverted by matrix element k, for kernels that form one element at a time
  std::vector<int> koff(F2 + 1, 0), kA;
  std::vector<double2> kc;
  for (int k = 0; k < F2; k++) {
    for (int A = 0; A < D; A++)
      if (std::abs(rT[A][k]) > 1e-14) {
        cd c = std::conj(rT[A][k]) / rnorm;
        kA.push_back(A);
        kc.push_back(make_double2(c.real(), c.imag()));
      }
    koff[k + 1] = (int)kA.size();
  }
  HR_CUDA(cudaMalloc(&L.d_projk_off, sizeof(int) * (F2 + 1)));
  HR_CUDA(cudaMalloc(&L.d_projk_A, sizeof(int) * kA.size()));
  HR_CUDA(cudaMalloc(&L.d_projk_c, sizeof(double2) * kc.size()));
  HR_CUDA(cudaMemcpy(L.d_projk_off, koff.data(), sizeof(int) * (F2 + 1), cudaMemcpyHostToDevice));
  HR_CUDA(cudaMemcpy(L.d_projk_A, kA.data(), sizeof(int) * kA.size(), cudaMemcpyHostToDevice));
  HR_CUDA(cudaMemcpy(L.d_projk_c, kc.data(), sizeof(double2) * kc.size(), cudaMemcpyHostToDevice));
  return 0;
}

// ---------------------------------------------------------------------------
// layout translation kernels (boundary only, never per operator application)
// ---------------------------------------------------------------------------
// host spinor element (site s of the field, complex component c) -> device
template <typename V>
__global__ void k_spinor_in(V *dev, const V *host, const int *h2d, int base, int nsites, int ncomp, int ld, int full) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)nsites * ncomp) return;
  int s = (int)(i / ncomp), c = (int)(i % ncomp);
  int d = h2d[base + s];
  int p = d >= ld ? 1 : 0, cb = d - p * ld;
  long o = full ? ((long)p * ncomp + c) * ld + cb : (long)c * ld + cb;
  dev[o] = host[i];
}

template <typename V>
__global__ void k_spinor_out(V *host, const V *dev, const int *h2d, int base, int nsites, int ncomp, int ld, int full) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)nsites * ncomp) return;
  int s = (int)(i / ncomp), c = (int)(i % ncomp);
  int d = h2d[base + s];
  int p = d >= ld ? 1 : 0, cb = d - p * ld;
  long o = full ? ((long)p * ncomp + c) * ld + cb : (long)c * ld + cb;
  host[i] = dev[o];
}

// per-site per-direction matrices: host [V][4][nel] -> device [4][nel][2ld]
template <typename E>
__global__ void k_links_in(E *dev, const E *host, const int *h2d, long V, int nel, int ld) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V * 4 * nel) return;
  long ix = i / (4 * nel);
  int r = (int)(i % (4 * nel)), mu = r / nel, e = r % nel;
  int d = h2d[ix];
  dev[((long)mu * nel + e) * 2 * ld + d] = host[i];
}

template <typename E>
__global__ void k_links_out(E *host, const E *dev, const int *h2d, long V, int nel, int ld, int ndir) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V * ndir * nel) return;
  long ix = i / (ndir * nel);
  int r = (int)(i % (ndir * nel)), mu = r / nel, e = r % nel;
  int d = h2d[ix];
  host[i] = dev[((long)mu * nel + e) * 2 * ld + d];
}

template <typename DST, typename SRC>
__global__ void k_convert(DST *dst, const SRC *src, long n) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (DST)src[i];
}

static inline unsigned nblk(long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

int launch_links_in(void *dev, const void *host_stage, int nel, int real, int ndir) {
  (void)ndir;
  long n = L.V * 4 * nel;
  if (real)
    k_links_in<double><<<nblk(n), 256, 0, L.stream>>>((double *)dev, (const double *)host_stage, L.d_h2d, L.V, nel, L.ld);
  else
    k_links_in<double2><<<nblk(n), 256, 0, L.stream>>>((double2 *)dev, (const double2 *)host_stage, L.d_h2d, L.V, nel, L.ld);
  HR_LAUNCH_CHECK();
  return 0;
}

int links_out(void *host, const void *dev, int nel, int elem_bytes, int ndir) {
  size_t bytes = (size_t)L.V * ndir * nel * elem_bytes;
  if (int rc = ensure_stage(bytes)) return rc;
  long n = L.V * ndir * nel;
  if (elem_bytes == 8)
    k_links_out<double><<<nblk(n), 256, 0, L.stream>>>((double *)L.stage, (const double *)dev, L.d_h2d, L.V, nel, L.ld, ndir);
  else
    k_links_out<double2><<<nblk(n), 256, 0, L.stream>>>((double2 *)L.stage, (const double2 *)dev, L.d_h2d, L.V, nel, L.ld, ndir);
  HR_LAUNCH_CHECK();
  HR_CUDA(cudaMemcpyAsync(host, L.stage, bytes, cudaMemcpyDeviceToHost, L.stream));
  HR_CUDA(cudaStreamSynchronize(L.stream));
  return 0;
}

// ---------------------------------------------------------------------------
// deterministic reductions: kernels leave nblocks x nvals partials in
// L.partials; one block folds them in a fixed order.
// ---------------------------------------------------------------------------
__global__ void k_fold(double *partials, int nblocks, int nvals, double *out) {
  for (int v = 0; v < nvals; v++) {
    double s = 0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partials[(long)b * nvals + v];
    s = block_sum(s);
    if (threadIdx.x == 0) out[v] = s;
  }
}

int finish_reduction(int nblocks, int nvals, double *host_out) {
  double *dres = L.partials + L.npart;
  k_fold<<<1, RED_THREADS, 0, L.stream>>>(L.partials, nblocks, nvals, dres);
  HR_LAUNCH_CHECK();
  HR_CUDA(cudaMemcpyAsync(L.h_partials, dres, sizeof(double) * nvals, cudaMemcpyDeviceToHost, L.stream));
  HR_CUDA(cudaStreamSynchronize(L.stream));
  for (int v = 0; v < nvals; v++) host_out[v] = L.h_partials[v];
  return 0;
}

// the device the library was initialised on (hrgpu_init), -1 before
int library_device() { return g_device; }

}  // namespace hrgpu

using namespace hrgpu;

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char *hrgpu_last_error(void) { return g_err.c_str(); }

int hrgpu_init(int device) {
  int n = 0;
  HR_CUDA(cudaGetDeviceCount(&n));
  HR_REQUIRE(device >= 0 && device < n, HRGPU_E_ARG, "hrgpu_init: device %d not present (%d devices)", device, n);
  HR_CUDA(cudaSetDevice(device));
  if (!g_own_stream) HR_CUDA(cudaStreamCreateWithFlags(&g_own_stream, cudaStreamNonBlocking));
  if (!L.stream && !g_stream_chosen) L.stream = g_own_stream;
  g_device = device;
  return 0;
}

// HiRep's serial even-odd walk (LibHR/Geometry/geometry_mpi_eo.c:449-498 with
// set_border_pointer :713-729 and fix_next_neightbours :1327-1352): sites are
// numbered in 2x2x2x2 path blocks, blocks walked T (outermost), Z, Y, X and the
// sites of a block in the same order, all even sites first, then all odd ones.
int hrgpu_geometry(int T, int X, int Y, int Z, int *ipt, int *iup, int *idn) {
  HR_REQUIRE(T > 0 && X > 0 && Y > 0 && Z > 0 && ipt, HRGPU_E_ARG, "hrgpu_geometry: bad arguments");
  const long V = (long)T * X * Y * Z;
  auto lex = [&](int t, int x, int y, int z) {
    t = (t + T) % T; x = (x + X) % X; y = (y + Y) % Y; z = (z + Z) % Z;
    return (long)t + T * ((long)x + X * ((long)y + (long)Y * z));
  };
  std::vector<int> map(V, -1);
  int id = 0;
  for (int eo = 0; eo < 2; eo++)
    for (int bt = 0; bt < T; bt += 2)
      for (int bz = 0; bz < Z; bz += 2)
        for (int by = 0; by < Y; by += 2)
          for (int bx = 0; bx < X; bx += 2)
            for (int t = bt; t < bt + 2 && t < T; t++)
              for (int z = bz; z < bz + 2 && z < Z; z++)
                for (int y = by; y < by + 2 && y < Y; y++)
                  for (int x = bx; x < bx + 2 && x < X; x++)
                    if ((t + x + y + z) % 2 == eo && map[lex(t, x, y, z)] == -1) map[lex(t, x, y, z)] = id++;
  for (int t = 0; t < T; t++)
    for (int x = 0; x < X; x++)
      for (int y = 0; y < Y; y++)
        for (int z = 0; z < Z; z++) {
          int ix = map[lex(t, x, y, z)];
          ipt[((t * X + x) * Y + y) * Z + z] = ix;
          if (iup) {
            iup[4 * ix + 0] = map[lex(t + 1, x, y, z)];
            iup[4 * ix + 1] = map[lex(t, x + 1, y, z)];
            iup[4 * ix + 2] = map[lex(t, x, y + 1, z)];
            iup[4 * ix + 3] = map[lex(t, x, y, z + 1)];
          }
          if (idn) {
            idn[4 * ix + 0] = map[lex(t - 1, x, y, z)];
            idn[4 * ix + 1] = map[lex(t, x - 1, y, z)];
            idn[4 * ix + 2] = map[lex(t, x, y - 1, z)];
            idn[4 * ix + 3] = map[lex(t, x, y, z - 1)];
          }
        }
  return 0;
}

int hrgpu_set_stream(void *s) {
  // NULL selects the legacy default stream (stream 0), which is what PyTorch's
  // default stream reports; the library's own stream is used until this is called
  if (L.stream) HR_CUDA(cudaStreamSynchronize(L.stream));
  L.stream = (cudaStream_t)s;
  g_stream_chosen = true;
  return 0;
}

int hrgpu_synchronize(void) {
  HR_CUDA(cudaStreamSynchronize(L.stream));
  return 0;
}

int hrgpu_finalize(void) {
  if (L.stream) cudaStreamSynchronize(L.stream);
  free_all();
  return 0;
}

int hrgpu_nf(void) { return L.nf; }

int hrgpu_algebra_generators(double *T) {
  HR_REQUIRE(L.ready && L.h_gT, HRGPU_E_STATE, "algebra_generators: lattice not initialised");
  HR_REQUIRE(T, HRGPU_E_ARG, "algebra_generators: NULL output");
  memcpy(T, L.h_gT, sizeof(double) * 2 * (size_t)L.dimg * L.ng * L.ng);
  return 0;
}

size_t hrgpu_spinor_bytes(int par, int prec) {
  if (!L.ready) return 0;
  return spinor_bytes(par, prec);
}

int hrgpu_lattice_init(int T, int X, int Y, int Z, int ng, int repr, const int *ipt) {
  if (g_device < 0) {
    if (int rc = hrgpu_init(0)) return rc;
  }
  HR_REQUIRE(T > 0 && X > 0 && Y > 0 && Z > 0, HRGPU_E_ARG, "hrgpu_lattice_init: bad sizes");
  HR_REQUIRE(T % 2 == 0 && X % 2 == 0 && Y % 2 == 0 && Z % 2 == 0, HRGPU_E_ARG,
             "hrgpu_lattice_init: even-odd preconditioning needs even sizes (%dx%dx%dx%d)", T, X, Y, Z);
  HR_REQUIRE(ng >= 2 && repr >= 0 && repr <= 3, HRGPU_E_ARG, "hrgpu_lattice_init: bad NG/representation");
  HR_REQUIRE(!(repr == HRGPU_ASYM && ng < 3), HRGPU_E_ARG, "hrgpu_lattice_init: antisymmetric needs NG >= 3");
  HR_REQUIRE(ipt != nullptr, HRGPU_E_ARG, "hrgpu_lattice_init: ipt is NULL");
  long V = (long)T * X * Y * Z;
  HR_REQUIRE(V < (1L << 30), HRGPU_E_ARG, "hrgpu_lattice_init: lattice too large");
  cudaStreamSynchronize(L.stream);
  free_all();
  L.T = T; L.X = X; L.Y = Y; L.Z = Z;
  L.V = V; L.VH = V / 2;
  L.ld = (int)((L.VH + 31) / 32 * 32);
  L.ng = ng; L.repr = repr; L.real = (repr == HRGPU_ADJ);
  L.nf = repr == HRGPU_FUND ? ng : repr == HRGPU_ADJ ? ng * ng - 1 : repr == HRGPU_SYM ? ng * (ng + 1) / 2 : ng * (ng - 1) / 2;
  L.dimg = ng * ng - 1;
  HR_REQUIRE(L.nf <= MAXNF, HRGPU_E_NF, "hrgpu_lattice_init: NF=%d exceeds %d", L.nf, MAXNF);
  // permutation: HiRep index -> device index; check that ipt is a bijection
  // with the even-first ordering HiRep's serial walk produces
  L.h_h2d = new int[V];
  std::vector<int> d2h(2 * (size_t)L.ld, -1);
  for (long i = 0; i < V; i++) L.h_h2d[i] = -1;
  for (int t = 0; t < T; t++)
    for (int x = 0; x < X; x++)
      for (int y = 0; y < Y; y++)
        for (int z = 0; z < Z; z++) {
          int ix = ipt[((t * X + x) * Y + y) * Z + z];
          HR_REQUIRE(ix >= 0 && ix < V && L.h_h2d[ix] == -1, HRGPU_E_ARG, "hrgpu_lattice_init: ipt is not a permutation");
          int p = (t + x + y + z) & 1;
          HR_REQUIRE((ix < L.VH) == (p == 0), HRGPU_E_ARG,
                     "hrgpu_lattice_init: ipt does not place even sites first (site %d)", ix);
          int cb = ((((t * Z + z) * Y + y) * X + x) >> 1);
          int d = p * L.ld + cb;
          L.h_h2d[ix] = d;
          d2h[d] = (int)ix;
        }
  HR_CUDA(cudaMalloc(&L.d_h2d, sizeof(int) * V));
  HR_CUDA(cudaMalloc(&L.d_d2h, sizeof(int) * 2 * L.ld));
  HR_CUDA(cudaMemcpy(L.d_h2d, L.h_h2d, sizeof(int) * V, cudaMemcpyHostToDevice));
  HR_CUDA(cudaMemcpy(L.d_d2h, d2h.data(), sizeof(int) * 2 * L.ld, cudaMemcpyHostToDevice));
  if (int rc = upload_projection_tables()) return rc;
  {
    long hop_blocks = (L.VH + 127) / 128 + 1;
    L.npart = 8L * (hop_blocks > RED_MAX_BLOCKS ? hop_blocks : RED_MAX_BLOCKS);
  }
  HR_CUDA(cudaMalloc(&L.partials, sizeof(double) * (L.npart + 64)));
  HR_CUDA(cudaMallocHost(&L.h_partials, sizeof(double) * 64));
  HR_CUDA(cudaMalloc(&L.d_scalars, sizeof(double) * 4096));
  L.ready = true;
  return 0;
}

}  // extern "C"

namespace hrgpu {
// host-order staging buffer <-> even-parity device field, for the host sites
// [base, base+nsites) (stage points at host site base)
int spinor_scatter_even(void *dev, const void *stage, int base, int nsites, int prec, cudaStream_t s) {
  const int ncomp = 4 * L.nf;
  const long n = (long)nsites * ncomp;
  if (n == 0) return 0;
  if (prec == HRGPU_DOUBLE)
    k_spinor_in<double2><<<nblk(n), 256, 0, s>>>((double2 *)dev, (const double2 *)stage, L.d_h2d, base, nsites, ncomp, L.ld, 0);
  else
    k_spinor_in<float2><<<nblk(n), 256, 0, s>>>((float2 *)dev, (const float2 *)stage, L.d_h2d, base, nsites, ncomp, L.ld, 0);
  HR_LAUNCH_CHECK();
  return 0;
}
int spinor_gather_even(void *stage, const void *dev, int base, int nsites, int prec, cudaStream_t s) {
  const int ncomp = 4 * L.nf;
  const long n = (long)nsites * ncomp;
  if (n == 0) return 0;
  if (prec == HRGPU_DOUBLE)
    k_spinor_out<double2><<<nblk(n), 256, 0, s>>>((double2 *)stage, (const double2 *)dev, L.d_h2d, base, nsites, ncomp, L.ld, 0);
  else
    k_spinor_out<float2><<<nblk(n), 256, 0, s>>>((float2 *)stage, (const float2 *)dev, L.d_h2d, base, nsites, ncomp, L.ld, 0);
  HR_LAUNCH_CHECK();
  return 0;
}
}  // namespace hrgpu

extern "C" {

int hrgpu_spinor_upload(void *dev, const void *host, int par, int prec) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "hrgpu_spinor_upload: lattice not initialised");
  HR_REQUIRE(dev && host && par >= 0 && par <= 2 && (prec == 0 || prec == 1), HRGPU_E_ARG, "hrgpu_spinor_upload: bad arguments");
  int nsites = par == HRGPU_FULL ? (int)L.V : (int)L.VH;
  int base = par == HRGPU_ODD ? (int)L.VH : 0;
  int ncomp = 4 * L.nf;
  size_t esz = prec == HRGPU_DOUBLE ? sizeof(double2) : sizeof(float2);
  size_t bytes = (size_t)nsites * ncomp * esz;
  if (int rc = ensure_stage(bytes)) return rc;
  HR_CUDA(cudaMemsetAsync(dev, 0, spinor_bytes(par, prec), L.stream));
  HR_CUDA(cudaMemcpyAsync(L.stage, host, bytes, cudaMemcpyHostToDevice, L.stream));
  long n = (long)nsites * ncomp;
  if (prec == HRGPU_DOUBLE)
    k_spinor_in<double2><<<nblk(n), 256, 0, L.stream>>>((double2 *)dev, (const double2 *)L.stage, L.d_h2d, base, nsites, ncomp, L.ld, par == HRGPU_FULL);
  else
    k_spinor_in<float2><<<nblk(n), 256, 0, L.stream>>>((float2 *)dev, (const float2 *)L.stage, L.d_h2d, base, nsites, ncomp, L.ld, par == HRGPU_FULL);
  HR_LAUNCH_CHECK();
  HR_CUDA(cudaStreamSynchronize(L.stream));
  return 0;
}

int hrgpu_spinor_download(void *host, const void *dev, int par, int prec) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "hrgpu_spinor_download: lattice not initialised");
  HR_REQUIRE(dev && host && par >= 0 && par <= 2 && (prec == 0 || prec == 1), HRGPU_E_ARG, "hrgpu_spinor_download: bad arguments");
  int nsites = par == HRGPU_FULL ? (int)L.V : (int)L.VH;
  int base = par == HRGPU_ODD ? (int)L.VH : 0;
  int ncomp = 4 * L.nf;
  size_t esz = prec == HRGPU_DOUBLE ? sizeof(double2) : sizeof(float2);
  size_t bytes = (size_t)nsites * ncomp * esz;
  if (int rc = ensure_stage(bytes)) return rc;
  long n = (long)nsites * ncomp;
  if (prec == HRGPU_DOUBLE)
    k_spinor_out<double2><<<nblk(n), 256, 0, L.stream>>>((double2 *)L.stage, (const double2 *)dev, L.d_h2d, base, nsites, ncomp, L.ld, par == HRGPU_FULL);
  else
    k_spinor_out<float2><<<nblk(n), 256, 0, L.stream>>>((float2 *)L.stage, (const float2 *)dev, L.d_h2d, base, nsites, ncomp, L.ld, par == HRGPU_FULL);
  HR_LAUNCH_CHECK();
  HR_CUDA(cudaMemcpyAsync(host, L.stage, bytes, cudaMemcpyDeviceToHost, L.stream));
  HR_CUDA(cudaStreamSynchronize(L.stream));
  return 0;
}

int hrgpu_assign_sd2s(void *out, const void *in, int par) {
  HR_REQUIRE(L.ready && out && in, HRGPU_E_ARG, "hrgpu_assign_sd2s: bad arguments");
  long n = (long)spinor_elems(par) * 2;
  k_convert<float, double><<<nblk(n), 256, 0, L.stream>>>((float *)out, (const double *)in, n);
  HR_LAUNCH_CHECK();
  return 0;
}

int hrgpu_assign_s2sd(void *out, const void *in, int par) {
  HR_REQUIRE(L.ready && out && in, HRGPU_E_ARG, "hrgpu_assign_s2sd: bad arguments");
  long n = (long)spinor_elems(par) * 2;
  k_convert<double, float><<<nblk(n), 256, 0, L.stream>>>((double *)out, (const float *)in, n);
  HR_LAUNCH_CHECK();
  return 0;
}

int hrgpu_gauge_set_f(const void *uf_host) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "hrgpu_gauge_set_f: lattice not initialised");
  HR_REQUIRE(uf_host, HRGPU_E_ARG, "hrgpu_gauge_set_f: NULL field");
  int nel = L.nf * L.nf;
  size_t esz = L.real ? sizeof(double) : sizeof(double2);
  size_t bytes = (size_t)L.V * 4 * nel * esz;
  if (!L.U) HR_CUDA(cudaMalloc(&L.U, (size_t)4 * nel * 2 * L.ld * esz));
  if (int rc = ensure_stage(bytes)) return rc;
  HR_CUDA(cudaMemcpyAsync(L.stage, uf_host, bytes, cudaMemcpyHostToDevice, L.stream));
  if (int rc = launch_links_in(L.U, L.stage, nel, L.real, 4)) return rc;
  L.have_gauge = true;
  if (int rc = detect_recon12()) return rc;
  if (int rc = hrgpu_assign_ud2u_f()) return rc;
  if (L.clover) {
    if (int rc = compute_clover_term_dev()) return rc;
  }
  HR_CUDA(cudaStreamSynchronize(L.stream));
  L.sigma = 0xF00F;
  L.sigma_diag = 0xF00F;
  L.sigma_flt = 0xF00F;
  return 0;
}

int hrgpu_gauge_get_f(void *uf_host) {
  HR_REQUIRE(L.ready && L.have_gauge, HRGPU_E_STATE, "hrgpu_gauge_get_f: no gauge field");
  return links_out(uf_host, L.U, L.nf * L.nf, L.real ? 8 : 16, 4);
}

}  // extern "C"

namespace hrgpu {

__global__ void k_links_bf16(void *dst, const double *src, long n, int real) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    if (real) ((__nv_bfloat16 *)dst)[i] = __double2bfloat16(src[i]);
    else ((__nv_bfloat162 *)dst)[i] = __halves2bfloat162(__double2bfloat16(src[2 * i]), __double2bfloat16(src[2 * i + 1]));
  }
}

int ensure_links_bf16() {
  HR_REQUIRE(L.have_gauge, HRGPU_E_STATE, "no gauge field set");
  if (L.Ubf && L.ubf_gen == L.gauge_gen) return 0;
  const long n = (long)4 * L.nf * L.nf * 2 * L.ld;  // link elements (complex or real)
  if (!L.Ubf) HR_CUDA(cudaMalloc(&L.Ubf, n * (L.real ? sizeof(__nv_bfloat16) : sizeof(__nv_bfloat162))));
  k_links_bf16<<<nblk(n), 256, 0, L.stream>>>(L.Ubf, (const double *)L.U, n, L.real);
  HR_LAUNCH_CHECK();
  L.ubf_gen = L.gauge_gen;
  return 0;
}

}  // namespace hrgpu

extern "C" {

int hrgpu_assign_ud2u_f(void) {
  HR_REQUIRE(L.ready && L.have_gauge, HRGPU_E_STATE, "hrgpu_assign_ud2u_f: no gauge field");
  int nel = L.nf * L.nf;
  long n = (long)4 * nel * 2 * L.ld * (L.real ? 1 : 2);
  if (!L.Uf) HR_CUDA(cudaMalloc(&L.Uf, n * sizeof(float)));
  k_convert<float, double><<<nblk(n), 256, 0, L.stream>>>((float *)L.Uf, (const double *)L.U, n);
  HR_LAUNCH_CHECK();
  if (L.recon12 >= 3) {  // the FP32 hop may build its links from these (variant 6)
    const long ng = (long)4 * L.ng * L.ng * 2 * L.ld * 2;
    if (!L.Ugf) HR_CUDA(cudaMalloc(&L.Ugf, ng * sizeof(float)));
    k_convert<float, double><<<nblk(ng), 256, 0, L.stream>>>((float *)L.Ugf, (const double *)L.Ug, ng);
    HR_LAUNCH_CHECK();
  }
  L.have_gauge_flt = true;
  L.gauge_gen++;  // every write of the double links is followed by this call
  return 0;
}

int hrgpu_gauge_set(const double *u_host) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "hrgpu_gauge_set: lattice not initialised");
  HR_REQUIRE(u_host, HRGPU_E_ARG, "hrgpu_gauge_set: NULL field");
  int nel = L.ng * L.ng;
  size_t bytes = (size_t)L.V * 4 * nel * sizeof(double2);
  if (!L.Ug) HR_CUDA(cudaMalloc(&L.Ug, (size_t)4 * nel * 2 * L.ld * sizeof(double2)));
  if (int rc = ensure_stage(bytes)) return rc;
  HR_CUDA(cudaMemcpyAsync(L.stage, u_host, bytes, cudaMemcpyHostToDevice, L.stream));
  long n = L.V * 4 * nel;
  k_links_in<double2><<<nblk(n), 256, 0, L.stream>>>(L.Ug, (const double2 *)L.stage, L.d_h2d, L.V, nel, L.ld);
  HR_LAUNCH_CHECK();
  fund_links_changed();
  HR_CUDA(cudaStreamSynchronize(L.stream));
  L.have_fund = true;
  return 0;
}

}  // extern "C"
