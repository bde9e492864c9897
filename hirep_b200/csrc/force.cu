// force.cu -- pseudofermion force on the device (LibHR/Update/force_fermion_core.c
// and the clover derivative of LibHR/Update/clover_tools.c:208-310).
//
// The force is the adjoint of the hopping term: per link, the spin-projected
// colour outer products of X and Y at x and x+mu (HiRep's _F_DIR0.._F_DIR3 and
// _suNf_FMAT) times the link, projected onto the algebra with the generators of
// the representation (a sparse table built at lattice set-up), scaled by
// -residue*dt*C(R)/C(F).  One thread per (site, direction).
#include <vector>

#include "dirac.cuh"
#include "hop_async.cuh"

namespace hrgpu {

static inline unsigned nb(long n, int t = 128) { return (unsigned)((n + t - 1) / t); }

struct ProjTab {
  const int *off, *k;
  const double2 *c;
  int dimg;
};

// h_A += coeff * Re sum_k c_Ak m_k, into force planes [mu][A][2ld]
template <int N>
__device__ __forceinline__ void project_add(const double2 (&m)[N * N], const ProjTab &P, double *f, long lp, int mu,
                                            long d, double coeff) {
  for (int A = 0; A < P.dimg; A++) {
    double s = 0.0;
    for (int q = P.off[A]; q < P.off[A + 1]; q++) {
      double2 c = P.c[q], v = m[P.k[q]];
      s += c.x * v.x - c.y * v.y;
    }
    f[((long)mu * P.dimg + A) * lp + d] += coeff * s;
  }
}

// full-lattice spinor element (component c) at device site d
__device__ __forceinline__ const double2 *sp_at(const double2 *f, long d, int c, int ld, int nf) {
  int p = d >= ld ? 1 : 0;
  return f + ((long)p * 4 * nf + c) * ld + (d - (long)p * ld);
}

// one _F_DIRmu(s1, chi1, chi2) accumulation: chi1 at x, chi2 at x+mu
template <int N, bool REAL>
__device__ __forceinline__ void f_dir(double2 (&s1)[N * N], const void *U, long lp, int mu, long dx, long dy,
                                      const double2 *c1, const double2 *c2, int ld) {
  double2 pt[N], pt2[N], p0[N], p1[N], p2[N], p3[N];
  for (int i = 0; i < N; i++) {
    double2 a0 = *sp_at(c2, dy, i, ld, N), a1 = *sp_at(c2, dy, N + i, ld, N);
    double2 a2 = *sp_at(c2, dy, 2 * N + i, ld, N), a3 = *sp_at(c2, dy, 3 * N + i, ld, N);
    double2 b0 = *sp_at(c1, dx, i, ld, N), b1 = *sp_at(c1, dx, N + i, ld, N);
    double2 b2 = *sp_at(c1, dx, 2 * N + i, ld, N), b3 = *sp_at(c1, dx, 3 * N + i, ld, N);
    if (mu == 0) { pt[i] = cadd(a0, a2); pt2[i] = cadd(a1, a3); p2[i] = csub(b0, b2); p3[i] = csub(b1, b3); }
    if (mu == 1) { pt[i] = caddi(a0, a3); pt2[i] = caddi(a1, a2); p2[i] = csubi(b0, b3); p3[i] = csubi(b1, b2); }
    if (mu == 2) { pt[i] = cadd(a0, a3); pt2[i] = csub(a1, a2); p2[i] = csub(b0, b3); p3[i] = cadd(b1, b2); }
    if (mu == 3) { pt[i] = caddi(a0, a2); pt2[i] = csubi(a1, a3); p2[i] = csubi(b0, b2); p3[i] = caddi(b1, b3); }
  }
  for (int i = 0; i < N; i++) {
    double2 u0 = make_double2(0, 0), u1 = make_double2(0, 0);
    for (int j = 0; j < N; j++) {
      long idx = ((long)mu * N * N + i * N + j) * lp + dx;
      if (REAL) {
        double u = ((const double *)U)[idx];
        rmac(u0, u, pt[j]);
        rmac(u1, u, pt2[j]);
      } else {
        double2 u = ((const double2 *)U)[idx];
        cmac(u0, u, pt[j]);
        cmac(u1, u, pt2[j]);
      }
    }
    p0[i] = u0;
    p1[i] = u1;
  }
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++) {
      // s1_ij += p0_i conj(p2_j) + p1_i conj(p3_j)   (real part only for real representations)
      double2 &s = s1[i * N + j];
      s.x += p0[i].x * p2[j].x + p0[i].y * p2[j].y + p1[i].x * p3[j].x + p1[i].y * p3[j].y;
      if (!REAL) s.y += p0[i].y * p2[j].x - p0[i].x * p2[j].y + p1[i].y * p3[j].x - p1[i].x * p3[j].y;
    }
}

// force_fermion_core hopping part (force_fermion_core.c:848-923), one thread per
// link with the projections and s1 in registers: the form kept for the
// representations k_force_hop_w does not cover (complex NF > 6, real NF > 3)
template <int N, bool REAL>
__global__ void k_force_hop(double *fsum, const void *U, const double2 *X, const double2 *Y, Geo g, ProjTab P,
                            double coeff) {
  long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int mu = blockIdx.y;
  if (d >= 2L * g.ld) return;
  int p = d >= g.ld ? 1 : 0;
  if (d - p * g.ld >= g.VH) return;
  int t, x, y, z;
  dev_coords(g, (int)d, t, x, y, z);
  long dy = nbr_index(g, t, x, y, z, mu, +1);
  const long lp = 2L * g.ld;
  double2 s1[N * N];
  for (int k = 0; k < N * N; k++) s1[k] = make_double2(0, 0);
  f_dir<N, REAL>(s1, U, lp, mu, d, dy, X, Y, g.ld);
  f_dir<N, REAL>(s1, U, lp, mu, d, dy, Y, X, g.ld);
  project_add<N>(s1, P, fsum, lp, mu, d, coeff);
}

// The same hopping force with the link pulled out of the outer products.  Per
// link (x, mu) HiRep forms s1 = sum of four terms (U A_k) B_k^+, k over the two
// spin projections of the two pairings (X at x with Y at x+mu, and Y at x with
// X at x+mu): A_k are projections at x+mu, B_k at x (_F_DIRmu,
// force_fermion_core.c:72-114).  Here the four U A_k are formed first (the
// link read once, row by row), then the B_k, and each element s1_ij is built
// from them and at once projected onto the algebra, element by element, with
// the table by element (its A and coefficient pairs).  So neither s1 nor the
// projections of the old form live in registers together, every array index is
// known at compile time (no local memory), and the per-generator sums go to a
// column of shared memory owned by the thread; the force planes get one
// read-modify-write per generator at the end.  For the complex representations
// up to NF = 6 and the real NF = 3 (the register budget of the four U A_k and
// B_k); the other representations keep k_force_hop.  (Four lanes per link, one
// term each, was measured too: 100 registers and twice the resident warps, but
// three times the instructions, each lane projecting its own partial sums,
// and 1.6x slower at 16^4 NF = 6.)
struct ProjTabK {
  const int *off, *A;
  const double2 *c;
  int dimg;
};

template <int N, bool REAL>
__global__ void __launch_bounds__(128) k_force_hop_w(double *fsum, const void *U, const double2 *X,
                                                      const double2 *Y, Geo g, ProjTabK P, double coeff) {
  extern __shared__ double hs[];  // [dimg][128]: this thread's generator sums in column tid
  const int tid = threadIdx.x;
  const long d = (long)blockIdx.x * 128 + tid;
  const int mu = blockIdx.y;
  if (d >= 2L * g.ld) return;
  const int p = d >= g.ld ? 1 : 0;
  if (d - p * g.ld >= g.VH) return;
  for (int A = 0; A < P.dimg; A++) hs[A * 128 + tid] = 0.0;
  int t, x, y, z;
  dev_coords(g, (int)d, t, x, y, z);
  const long dy = nbr_index(g, t, x, y, z, mu, +1);
  const long lp = 2L * g.ld;
  // A_k at x+mu: k = 0, 1 from Y (pairing X at x), k = 2, 3 from X (pairing Y at x)
  double2 a[4][N];
#pragma unroll
  for (int pr = 0; pr < 2; pr++) {
    const double2 *c2 = pr ? X : Y;
#pragma unroll
    for (int i = 0; i < N; i++) {
      const double2 a0 = *sp_at(c2, dy, i, g.ld, N), a1 = *sp_at(c2, dy, N + i, g.ld, N);
      const double2 a2 = *sp_at(c2, dy, 2 * N + i, g.ld, N), a3 = *sp_at(c2, dy, 3 * N + i, g.ld, N);
      double2 &pt = a[2 * pr][i], &pt2 = a[2 * pr + 1][i];
      if (mu == 0) { pt = cadd(a0, a2); pt2 = cadd(a1, a3); }
      if (mu == 1) { pt = caddi(a0, a3); pt2 = caddi(a1, a2); }
      if (mu == 2) { pt = cadd(a0, a3); pt2 = csub(a1, a2); }
      if (mu == 3) { pt = caddi(a0, a2); pt2 = csubi(a1, a3); }
    }
  }
  // U A_k, the link read once, row by row
  double2 ua[4][N];
#pragma unroll
  for (int i = 0; i < N; i++) {
#pragma unroll
    for (int k = 0; k < 4; k++) ua[k][i] = make_double2(0, 0);
#pragma unroll
    for (int j = 0; j < N; j++) {
      const long idx = ((long)mu * N * N + i * N + j) * lp + d;
      if (REAL) {
        const double u = ((const double *)U)[idx];
#pragma unroll
        for (int k = 0; k < 4; k++) rmac(ua[k][i], u, a[k][j]);
      } else {
        const double2 u = ((const double2 *)U)[idx];
#pragma unroll
        for (int k = 0; k < 4; k++) cmac(ua[k][i], u, a[k][j]);
      }
    }
  }
  // B_k at x: k = 0, 1 from X, k = 2, 3 from Y (reusing a's registers)
  double2 (&b)[4][N] = a;
#pragma unroll
  for (int pr = 0; pr < 2; pr++) {
    const double2 *c1 = pr ? Y : X;
#pragma unroll
    for (int i = 0; i < N; i++) {
      const double2 b0 = *sp_at(c1, d, i, g.ld, N), b1 = *sp_at(c1, d, N + i, g.ld, N);
      const double2 b2 = *sp_at(c1, d, 2 * N + i, g.ld, N), b3 = *sp_at(c1, d, 3 * N + i, g.ld, N);
      double2 &p2 = b[2 * pr][i], &p3 = b[2 * pr + 1][i];
      if (mu == 0) { p2 = csub(b0, b2); p3 = csub(b1, b3); }
      if (mu == 1) { p2 = csubi(b0, b3); p3 = csubi(b1, b2); }
      if (mu == 2) { p2 = csub(b0, b3); p3 = cadd(b1, b2); }
      if (mu == 3) { p2 = csubi(b0, b2); p3 = caddi(b1, b3); }
    }
  }
  // s1_ij = sum_k (U A_k)_i conj(B_k)_j (real part only for real representations),
  // projected element by element
#pragma unroll
  for (int i = 0; i < N; i++) {
#pragma unroll
    for (int j = 0; j < N; j++) {
      double mr = 0.0, mi = 0.0;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        mr += ua[k][i].x * b[k][j].x + ua[k][i].y * b[k][j].y;
        if (!REAL) mi += ua[k][i].y * b[k][j].x - ua[k][i].x * b[k][j].y;
      }
      const int kk = i * N + j;
      const int q1 = __ldg(P.off + kk + 1);
      for (int q = __ldg(P.off + kk); q < q1; q++) {
        const double2 c = __ldg(P.c + q);
        hs[__ldg(P.A + q) * 128 + tid] += c.x * mr - c.y * mi;
      }
    }
  }
  for (int A = 0; A < P.dimg; A++) fsum[((long)mu * P.dimg + A) * lp + d] += coeff * hs[A * 128 + tid];
}

// The projection table again, element-major and padded to E entries per
// element (A = 0, c = 0 for padding), in constant memory: with the element and
// the entry known at compile time, every coefficient and generator index is a
// constant operand and the projection needs no loads.  At most 5 entries per
// element occur (SU(6) fundamental); 3 for the SU(4) two-index antisymmetric,
// 2 for the SU(3) symmetric and the fundamentals up to SU(3).
constexpr int FT_MAX = 6 * 6 * 5;
__constant__ double2 c_ftc[FT_MAX];
__constant__ int c_ftA[FT_MAX];
static int ft_E = 0, ft_key = -1;  // entries per element of the uploaded table; (ng, repr) it was made for

__device__ __forceinline__ void prefetch_l2(const void *p) {
  asm volatile("{\n .reg .u64 g;\n cvta.to.global.u64 g, %0;\n prefetch.global.L2 [g];\n}\n" ::"l"(p));
}

// k_force_hop_w on two lanes per link, in two different warps: warp w of a
// block takes pairing h = w & 1 (h = 0: A_k from Y at x+mu, B_k from X at x;
// h = 1: A_k from X at x+mu, B_k from Y at x) of the sites (w >> 1) * 32 +
// lane, so a lane holds two U A_k and two B_k instead of four (128 registers,
// four blocks of 128 per SM against two) and loads half of the spinor
// components.  The projection is linear, so each lane projects its own terms
// of every s1 element onto the algebra; the table addresses are then the same
// for the whole warp and known at compile time (constant operands, no loads
// and no exchange between lanes), and the two warps' generator sums meet in
// shared memory at the end, the even generators written by the h = 0 lane and
// the odd ones by the h = 1 lane.  The four directions of a block of sites are
// adjacent blocks.  Lanes past the end of the lattice work on site 0 and write
// nothing, so every lane reaches the barrier.  PF: first ask L2 for the link
// and the spinor at x (prefetch.global.L2, no registers held), so that their
// loads, issued a few at a time after the neighbour's, wait for L2 rather than
// for DRAM.
//
// FR (NF = 6 two-index representations, link modes 3 and 4): the link is
// built from the fundamental one (Ug, 9 or 16 complex numbers) as the hop's
// variant 6 does (two_idx_elem), with the antiperiodic sign when frbc is set;
// the register budget is that of 3 blocks per SM.
//
// ST (complex links): the operands at x are copied into shared memory with
// cp.async at the start, so that they are in flight while the neighbour's
// spinor is loaded and projected without holding registers: ST = 1 the link
// (each of the two warps of a site copies half its elements, read by both
// after a barrier), ST = 2 the link and the lane's spinor at x (its own
// copies, read back after its own wait; the register budget of 2 blocks per
// SM, which its shared memory allows).  Shared memory after the generator
// sums: the link [N*N][64 sites], then (ST = 2) the spinors [4 warps][4N][32].
template <int N, bool REAL, int E, bool PF, int FR = 0, int ST = 0>
__global__ void __launch_bounds__(128, FR ? 3 : ST == 2 ? 2 : 4)
    k_force_hop_w3(double *fsum, const void *U, const double2 *X, const double2 *Y, Geo g, int dimg, double coeff,
                   const double2 *Ug = nullptr, int frbc = 0) {
  extern __shared__ double hs[];  // [dimg][128]: this lane's generator sums in column tid
  const int tid = threadIdx.x, w = tid >> 5, h = w & 1;
  const int sl = (w >> 1) * 32 + (tid & 31);  // this lane's site in the block
  const long d0 = (long)(blockIdx.x >> 2) * 64 + sl;
  const int mu = blockIdx.x & 3;
  const int p0 = d0 >= g.ld ? 1 : 0;
  const bool valid = d0 < 2L * g.ld && d0 - p0 * g.ld < g.VH;
  const long d = valid ? d0 : 0;
  const long lp = 2L * g.ld;
  const double2 *c2 = h ? X : Y, *c1 = h ? Y : X;
  double2 *sU = (double2 *)(hs + (long)dimg * 128);
  double2 *sC = sU + N * N * 64 + (long)w * 4 * N * 32 + (tid & 31);
  if constexpr (ST != 0) {
    static_assert(!REAL && FR == 0 && !PF, "ST: complex stored links");
#pragma unroll
    for (int k = 0; k < (N * N + 1) / 2; k++) {
      const int e = 2 * k + h;
      if (e < N * N) cp_async16(sU + e * 64 + sl, (const double2 *)U + ((long)mu * N * N + e) * lp + d);
    }
    if constexpr (ST == 2) {
#pragma unroll
      for (int c = 0; c < 4 * N; c++) cp_async16(sC + c * 32, sp_at(c1, d, c, g.ld, N));
    }
    cp_async_commit();
  }
  for (int A = 0; A < dimg; A++) hs[A * 128 + tid] = 0.0;
  int t, x, y, z;
  dev_coords(g, (int)d, t, x, y, z);
  const long dy = nbr_index(g, t, x, y, z, mu, +1);
  if (PF) {
#pragma unroll
    for (int e = 0; e < N * N; e++)
      prefetch_l2(REAL ? (const void *)((const double *)U + ((long)mu * N * N + e) * lp + d)
                       : (const void *)((const double2 *)U + ((long)mu * N * N + e) * lp + d));
#pragma unroll
    for (int c = 0; c < 4 * N; c++) prefetch_l2(sp_at(c1, d, c, g.ld, N));
  }
  double2 a[2][N];
#pragma unroll
  for (int i = 0; i < N; i++) {
    const double2 a0 = *sp_at(c2, dy, i, g.ld, N), a1 = *sp_at(c2, dy, N + i, g.ld, N);
    const double2 a2 = *sp_at(c2, dy, 2 * N + i, g.ld, N), a3 = *sp_at(c2, dy, 3 * N + i, g.ld, N);
    double2 &pt = a[0][i], &pt2 = a[1][i];
    if (mu == 0) { pt = cadd(a0, a2); pt2 = cadd(a1, a3); }
    if (mu == 1) { pt = caddi(a0, a3); pt2 = caddi(a1, a2); }
    if (mu == 2) { pt = cadd(a0, a3); pt2 = csub(a1, a2); }
    if (mu == 3) { pt = caddi(a0, a2); pt2 = csubi(a1, a3); }
  }
  double2 ua[2][N];
  if constexpr (FR != 0) {
    static_assert(N == 6 && !REAL, "FR: the NF = 6 two-index representations");
    constexpr int NG = TwoIdx<FR>::NG;
    double2 fu[NG * NG];
#pragma unroll
    for (int k = 0; k < NG * NG; k++) fu[k] = __ldg(Ug + ((long)mu * NG * NG + k) * lp + d);
    const double sg = (frbc && mu == 0 && t == 0) ? -1.0 : 1.0;
#pragma unroll
    for (int i = 0; i < N; i++) {
      ua[0][i] = ua[1][i] = make_double2(0, 0);
#pragma unroll
      for (int j = 0; j < N; j++) {
        const double2 u = two_idx_elem<FR>(fu, i, j, sg);
        cmac(ua[0][i], u, a[0][j]);
        cmac(ua[1][i], u, a[1][j]);
      }
    }
  } else {
    if constexpr (ST != 0) {
      cp_async_wait<0>();
      __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < N; i++) {
      ua[0][i] = ua[1][i] = make_double2(0, 0);
#pragma unroll
      for (int j = 0; j < N; j++) {
        const long idx = ((long)mu * N * N + i * N + j) * lp + d;
        if constexpr (ST != 0) {
          const double2 u = sU[(i * N + j) * 64 + sl];
          cmac(ua[0][i], u, a[0][j]);
          cmac(ua[1][i], u, a[1][j]);
        } else if (REAL) {
          const double u = ((const double *)U)[idx];
          rmac(ua[0][i], u, a[0][j]);
          rmac(ua[1][i], u, a[1][j]);
        } else {
          const double2 u = ((const double2 *)U)[idx];
          cmac(ua[0][i], u, a[0][j]);
          cmac(ua[1][i], u, a[1][j]);
        }
      }
    }
  }
  double2 (&b)[2][N] = a;
#pragma unroll
  for (int i = 0; i < N; i++) {
    double2 b0, b1, b2, b3;
    if constexpr (ST == 2) {
      b0 = sC[i * 32];
      b1 = sC[(N + i) * 32];
      b2 = sC[(2 * N + i) * 32];
      b3 = sC[(3 * N + i) * 32];
    } else {
      b0 = *sp_at(c1, d, i, g.ld, N);
      b1 = *sp_at(c1, d, N + i, g.ld, N);
      b2 = *sp_at(c1, d, 2 * N + i, g.ld, N);
      b3 = *sp_at(c1, d, 3 * N + i, g.ld, N);
    }
    double2 &p2 = b[0][i], &p3 = b[1][i];
    if (mu == 0) { p2 = csub(b0, b2); p3 = csub(b1, b3); }
    if (mu == 1) { p2 = csubi(b0, b3); p3 = csubi(b1, b2); }
    if (mu == 2) { p2 = csub(b0, b3); p3 = cadd(b1, b2); }
    if (mu == 3) { p2 = csubi(b0, b2); p3 = caddi(b1, b3); }
  }
#pragma unroll
  for (int i = 0; i < N; i++) {
#pragma unroll
    for (int j = 0; j < N; j++) {
      const double mr = ua[0][i].x * b[0][j].x + ua[0][i].y * b[0][j].y + ua[1][i].x * b[1][j].x + ua[1][i].y * b[1][j].y;
      const double mi =
          REAL ? 0.0 : ua[0][i].y * b[0][j].x - ua[0][i].x * b[0][j].y + ua[1][i].y * b[1][j].x - ua[1][i].x * b[1][j].y;
#pragma unroll
      for (int e = 0; e < E; e++) {
        const double2 c = c_ftc[(i * N + j) * E + e];
        hs[c_ftA[(i * N + j) * E + e] * 128 + tid] += c.x * mr - c.y * mi;
      }
    }
  }
  __syncthreads();
  if (valid)
    for (int A = h; A < dimg; A += 2)
      fsum[((long)mu * dimg + A) * lp + d] += coeff * (hs[A * 128 + tid] + hs[A * 128 + (tid ^ 32)]);
}

// the padded table for the current representation, uploaded when it changes
// (ft_E = 0: some element has more than 5 entries, and k_force_hop_w serves)
static int force_table_upload() {
  const int key = L.ng * 16 + L.repr;
  if (key == ft_key) return 0;
  const int F2 = L.nf * L.nf, D = L.dimg;
  auto nz = [&](int A, int k) {
    return std::hypot(L.h_rT[((size_t)A * F2 + k) * 2], L.h_rT[((size_t)A * F2 + k) * 2 + 1]) > 1e-14;
  };
  int emax = 0;
  for (int k = 0; k < F2; k++) {
    int n = 0;
    for (int A = 0; A < D; A++) n += nz(A, k);
    emax = std::max(emax, n);
  }
  const int E = emax <= 2 ? 2 : emax <= 3 ? 3 : 5;
  ft_E = 0;
  ft_key = key;
  if (emax > 5 || F2 * E > FT_MAX) return 0;
  std::vector<double2> c(FT_MAX, make_double2(0.0, 0.0));
  std::vector<int> a(FT_MAX, 0);
  for (int k = 0; k < F2; k++) {
    int n = 0;
    for (int A = 0; A < D; A++)
      if (nz(A, k)) {
        // c = conj(T_A^R)_k / C(R), as in the table by element
        const double re = L.h_rT[((size_t)A * F2 + k) * 2], im = L.h_rT[((size_t)A * F2 + k) * 2 + 1];
        c[k * E + n] = make_double2(re / L.repr_norm2, -im / L.repr_norm2);
        a[k * E + n] = A;
        n++;
      }
  }
  ft_key = -1;
  HR_CUDA(cudaMemcpyToSymbol(c_ftc, c.data(), sizeof(double2) * FT_MAX));
  HR_CUDA(cudaMemcpyToSymbol(c_ftA, a.data(), sizeof(int) * FT_MAX));
  ft_E = E;
  ft_key = key;
  return 0;
}

// g5 sigma_{mu nu} on a spinor held as [4][N] (force_fermion_core.c:123-250)
template <int N>
__device__ __forceinline__ void g5_sigma(double2 (&s)[4][N], const double2 (&u)[4][N], int q) {
  // q enumerates (0,1),(0,2),(1,2),(0,3),(1,3),(2,3) as cl_force does
  const int srcs[6][4] = {{1, 0, 3, 2}, {1, 0, 3, 2}, {0, 1, 2, 3}, {0, 1, 2, 3}, {1, 0, 3, 2}, {1, 0, 3, 2}};
  // factors (re, im)
  const double fr[6][4] = {{0, 0, 0, 0}, {-1, 1, -1, 1}, {0, 0, 0, 0}, {0, 0, 0, 0}, {-1, 1, 1, -1}, {0, 0, 0, 0}};
  const double fi[6][4] = {{-1, -1, -1, -1}, {0, 0, 0, 0}, {1, -1, -1, 1}, {-1, 1, -1, 1}, {0, 0, 0, 0}, {1, 1, -1, -1}};
  for (int c = 0; c < 4; c++)
    for (int i = 0; i < N; i++) {
      double2 a = u[srcs[q][c]][i];
      s[c][i] = make_double2(fr[q][c] * a.x - fi[q][c] * a.y, fr[q][c] * a.y + fi[q][c] * a.x);
    }
}

// force_clover_fermion (force_fermion_core.c:384-454)
template <int N, bool REAL>
__global__ void k_force_clover_fermion(double2 *clf, const double2 *X, const double2 *Y, Geo g, double residue) {
  long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int q = blockIdx.y;
  if (d >= 2L * g.ld) return;
  int p = d >= g.ld ? 1 : 0;
  if (d - p * g.ld >= g.VH) return;
  double2 xs[4][N], ys[4][N], tl[4][N], tr[4][N];
  for (int c = 0; c < 4; c++)
    for (int i = 0; i < N; i++) {
      xs[c][i] = *sp_at(X, d, c * N + i, g.ld, N);
      ys[c][i] = *sp_at(Y, d, c * N + i, g.ld, N);
    }
  g5_sigma<N>(tr, xs, q);
  g5_sigma<N>(tl, ys, q);
  const long lp = 2L * g.ld;
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++) {
      double2 s = make_double2(0, 0);
      for (int k = 0; k < 4; k++) {
        cmacc(s, xs[k][j], tl[k][i]);  // tl_i conj(X_j)
        cmacc(s, ys[k][j], tr[k][i]);  // tr_i conj(Y_j)
      }
      if (REAL) s.y = 0.0;
      double2 &o = clf[((long)q * N * N + i * N + j) * lp + d];
      o.x += residue * s.x;
      o.y += residue * s.y;
    }
}

// The exponential clover's force matrices (force_fermion_core.c:484-772).  With
// D = (4+m) exp(Ah), Ah = A/(4+m) on each chirality block, the derivative of
// the block along dA is the Frechet derivative of the exponential,
//   L(Ah, dA) = sum_{k,l} Ah^k dA Ah^l / (k+l+1)! ,
// which the reference expands in powers of Ah (its Taylor or Cayley-Hamilton
// coefficients C_kl).  Contracted with the fields it turns Y X^+, the matrix of
// the linear term's sigma insertions, into P = L(Ah, Y X^+) per block.  Here P
// is computed by scaling and squaring instead of a power expansion: with Ah and
// E = Y X^+ scaled by 2^-s (|Ah|_F <= 1/4), the Taylor recursions
//   T_k = T_{k-1} Ah / k ,  S_k = (T_{k-1} E + S_{k-1} Ah) / k      (k <= 16)
// sum to e = exp(Ah) and P = L(Ah, E), then s doublings P <- e P + P e,
// e <- e e.  One block of (2NF)^2 threads per site, one matrix element each,
// seven 2NF x 2NF matrices in dynamic shared memory.
constexpr int EXPF_TAYLOR = 16;
// g5 sigma_{mu nu} for the six (mu,nu) of cl_force: component c of the result is
// (fr + i fi) times component src of the input (the tables of g5_sigma above)
__constant__ int c_sig_src[6][4] = {{1, 0, 3, 2}, {1, 0, 3, 2}, {0, 1, 2, 3}, {0, 1, 2, 3}, {1, 0, 3, 2}, {1, 0, 3, 2}};
__constant__ double c_sig_fr[6][4] = {{0, 0, 0, 0}, {-1, 1, -1, 1}, {0, 0, 0, 0}, {0, 0, 0, 0}, {-1, 1, 1, -1}, {0, 0, 0, 0}};
__constant__ double c_sig_fi[6][4] = {{-1, -1, -1, -1}, {0, 0, 0, 0}, {1, -1, -1, 1}, {-1, 1, -1, 1}, {0, 0, 0, 0}, {1, 1, -1, -1}};
template <int N>
constexpr size_t expf_smem() { return sizeof(double2) * 7 * (2 * N) * (2 * N); }

template <int N, bool REAL>
__global__ void __launch_bounds__(4 * N * N) k_force_expclover_fermion(double2 *clf, const double2 *cl, const double2 *X,
                                                                       const double2 *Y, Geo g, double sigma,
                                                                       double residue) {
  constexpr int n = 2 * N, nn = n * n;
  extern __shared__ double2 sm[];
  double2 *A = sm, *E = sm + nn, *T = sm + 2 * nn, *S = sm + 3 * nn, *Ex = sm + 4 * nn, *P0 = sm + 5 * nn,
          *P1 = sm + 6 * nn;
  __shared__ int s_sq;
  const long d = blockIdx.x;
  const int p = d >= g.ld ? 1 : 0;
  if (d - p * g.ld >= g.VH) return;  // padding site: the whole block leaves
  const long lp = 2L * g.ld;
  const int t = threadIdx.x, i = t / n, j = t % n;
  for (int b = 0; b < 2; b++) {
    double2 *P = b ? P1 : P0;
    double2 v = (i >= j) ? hblock<N>(cl, b, i, j, lp, d, 0.0) : hblock<N>(cl, b, j, i, lp, d, 0.0);
    if (i < j) v.y = -v.y;
    A[t] = make_double2(v.x / sigma, v.y / sigma);
    const double2 yi = *sp_at(Y, d, 2 * b * N + i, g.ld, N), xj = *sp_at(X, d, 2 * b * N + j, g.ld, N);
    E[t] = make_double2(yi.x * xj.x + yi.y * xj.y, yi.y * xj.x - yi.x * xj.y);  // y_i conj(x_j)
    __syncthreads();
    if (t == 0) {
      double nrm = 0;
      for (int k = 0; k < nn; k++) nrm += A[k].x * A[k].x + A[k].y * A[k].y;
      nrm = sqrt(nrm);
      int sq = 0;
      while (nrm > 0.25 && sq < 60) {
        nrm *= 0.5;
        sq++;
      }
      s_sq = sq;
    }
    __syncthreads();
    const int sq = s_sq;
    const double sc = ldexp(1.0, -sq);
    A[t] = make_double2(A[t].x * sc, A[t].y * sc);
    E[t] = make_double2(E[t].x * sc, E[t].y * sc);
    T[t] = Ex[t] = make_double2(i == j ? 1.0 : 0.0, 0.0);
    S[t] = P[t] = make_double2(0, 0);
    __syncthreads();
    for (int k = 1; k <= EXPF_TAYLOR; k++) {
      double2 ta = make_double2(0, 0), sa = make_double2(0, 0);
      for (int l = 0; l < n; l++) {
        const double2 tl = T[i * n + l];
        cmac(ta, tl, A[l * n + j]);
        cmac(sa, tl, E[l * n + j]);
        cmac(sa, S[i * n + l], A[l * n + j]);
      }
      __syncthreads();
      T[t] = make_double2(ta.x / k, ta.y / k);
      S[t] = make_double2(sa.x / k, sa.y / k);
      Ex[t] = cadd(Ex[t], T[t]);
      P[t] = cadd(P[t], S[t]);
      __syncthreads();
    }
    for (int q = 0; q < sq; q++) {
      double2 ea = make_double2(0, 0), pa = make_double2(0, 0);
      for (int l = 0; l < n; l++) {
        const double2 el = Ex[i * n + l];
        cmac(ea, el, Ex[l * n + j]);
        cmac(pa, el, P[l * n + j]);
        cmac(pa, P[i * n + l], Ex[l * n + j]);
      }
      __syncthreads();
      Ex[t] = ea;
      P[t] = pa;
      __syncthreads();
    }
  }
  // the sigma insertions of the linear term (g5_sigma, fmat_create) with P in
  // place of Y X^+: sum_c f_qc (P[(s_c,i),(c,j)] + conj(P[(c,j),(s_c,i)]))
  for (int o = t; o < 6 * N * N; o += blockDim.x) {
    const int q = o / (N * N), ii = (o / N) % N, jj = o % N;
    double2 s = make_double2(0, 0);
    for (int c = 0; c < 4; c++) {
      const int sc = c_sig_src[q][c];
      const double2 *P = (c >> 1) ? P1 : P0;
      const double2 a = P[((sc & 1) * N + ii) * n + (c & 1) * N + jj];
      const double2 bb = P[((c & 1) * N + jj) * n + (sc & 1) * N + ii];
      const double2 w = make_double2(a.x + bb.x, a.y - bb.y);
      s.x += c_sig_fr[q][c] * w.x - c_sig_fi[q][c] * w.y;
      s.y += c_sig_fr[q][c] * w.y + c_sig_fi[q][c] * w.x;
    }
    if (REAL) s.y = 0.0;
    double2 &out = clf[((long)q * N * N + ii * N + jj) * lp + d];
    out.x += residue * s.x;
    out.y += residue * s.y;
  }
}

template <int N, bool REAL>
static int launch_force_expclover(double2 *clf, const double2 *cl, const double2 *X, const double2 *Y, Geo g,
                                  double sigma, double residue) {
  constexpr size_t smem = expf_smem<N>();
  if (smem > 48 * 1024)
    HR_CUDA(cudaFuncSetAttribute(k_force_expclover_fermion<N, REAL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  k_force_expclover_fermion<N, REAL><<<(unsigned)(2L * g.ld), 4 * N * N, smem, L.stream>>>(clf, cl, X, Y, g, sigma,
                                                                                          residue);
  HR_LAUNCH_CHECK();
  return 0;
}

// force_clover_core (force_fermion_core.c:282-379): one thread per (site, mu)
template <int N, bool REAL>
__global__ void k_force_clover_core(double *fsum, const void *U, const double2 *clf, Geo g, ProjTab P, double coeff) {
  long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int mu = blockIdx.y;
  if (d >= 2L * g.ld) return;
  int p = d >= g.ld ? 1 : 0;
  if (d - p * g.ld >= g.VH) return;
  int t, x, y, z;
  dev_coords(g, (int)d, t, x, y, z);
  const long lp = 2L * g.ld;
  for (int nu = 0; nu < 4; nu++) {
    if (nu == mu) continue;
    int c[4] = {t, x, y, z};
    long o1 = nbr_index(g, t, x, y, z, mu, +1);
    long o2 = nbr_index(g, t, x, y, z, nu, +1);
    long o3 = nbr_index(g, t, x, y, z, nu, -1);
    int cm[4] = {c[0], c[1], c[2], c[3]};
    int L4[4] = {g.T, g.X, g.Y, g.Z};
    cm[nu] = (cm[nu] - 1 + L4[nu]) % L4[nu];
    long o4 = nbr_index(g, cm[0], cm[1], cm[2], cm[3], mu, +1);
    int cp[4] = {c[0], c[1], c[2], c[3]};
    cp[nu] = (cp[nu] + 1) % L4[nu];
    long o5 = nbr_index(g, cp[0], cp[1], cp[2], cp[3], mu, +1);
    int num, sign;
    if (mu < nu) { num = nu * (nu - 1) / 2 + mu; sign = +1; }
    else { num = mu * (mu - 1) / 2 + nu; sign = -1; }
    CMat<N> W0, W1, W2, W3, W4, W5, W6, W7, W8, s1, s2, s3, fm, Z, a;
    auto zload = [&](CMat<N> &m, long s) {
      for (int k = 0; k < N * N; k++) m.c[k] = clf[((long)num * N * N + k) * lp + s];
    };
    // W0 = U(o3,mu)^+, W1 = U(o3,nu), W2 = U(o1,nu), W3 = U(o2,mu)^+, W4 = U(x,nu)^+, W5 = U(o4,nu)^+
    for (int k = 0; k < N * N; k++) W0.c[k] = make_double2(0, 0);
    {
      CMat<N> tmpm;
      mload<N, REAL>(tmpm, U, mu, o3, lp);
      for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) W0.c[i * N + j] = make_double2(tmpm.c[j * N + i].x, -tmpm.c[j * N + i].y);
      mload<N, REAL>(W1, U, nu, o3, lp);
      mload<N, REAL>(W2, U, nu, o1, lp);
      mload<N, REAL>(tmpm, U, mu, o2, lp);
      for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) W3.c[i * N + j] = make_double2(tmpm.c[j * N + i].x, -tmpm.c[j * N + i].y);
      mload<N, REAL>(tmpm, U, nu, d, lp);
      for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) W4.c[i * N + j] = make_double2(tmpm.c[j * N + i].x, -tmpm.c[j * N + i].y);
      mload<N, REAL>(tmpm, U, nu, o4, lp);
      for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) W5.c[i * N + j] = make_double2(tmpm.c[j * N + i].x, -tmpm.c[j * N + i].y);
    }
    mmul<N, false, false>(W6, W0, W1);
    mmul<N, false, false>(W7, W2, W3);
    mmul<N, false, false>(s1, W5, W6);
    mmul<N, false, false>(W8, W7, W4);
    for (int k = 0; k < N * N; k++) W8.c[k] = csub(W8.c[k], s1.c[k]);
    zload(Z, d);
    mmul<N, false, false>(fm, W8, Z);
    zload(Z, o1);
    mmul<N, false, false>(s1, Z, W8);
    madd(fm, s1);
    zload(Z, o3);
    mmul<N, false, false>(s1, W0, Z);
    mmul<N, false, false>(s2, s1, W1);
    zload(Z, o4);
    mmul<N, false, false>(s3, Z, W6);
    madd(s2, s3);
    mmul<N, false, false>(s1, W5, s2);
    for (int k = 0; k < N * N; k++) fm.c[k] = csub(fm.c[k], s1.c[k]);
    zload(Z, o5);
    mmul<N, false, false>(s1, W2, Z);
    mmul<N, false, false>(s2, s1, W3);
    zload(Z, o2);
    mmul<N, false, false>(s3, W7, Z);
    madd(s2, s3);
    mmul<N, false, false>(s1, s2, W4);
    madd(fm, s1);
    mload<N, REAL>(a, U, mu, d, lp);
    mmul<N, false, false>(s1, a, fm);
    double2 m[N * N];
    for (int k = 0; k < N * N; k++) m[k] = REAL ? make_double2(s1.c[k].x, 0.0) : s1.c[k];
    project_add<N>(m, P, fsum, lp, mu, d, sign * coeff);
  }
}

// _compute_clover_force (clover_tools.c:208-298) on odd sites from the packed inverse
template <int N, bool REAL>
__global__ void k_force_logdet(double2 *clf, const double *idg, const double2 *iod, Geo g, double coeff) {
  int cb = blockIdx.x * blockDim.x + threadIdx.x;
  if (cb >= g.VH) return;
  const long lp = 2L * g.ld, d = (long)g.ld + cb;  // odd sites
  const int n = 2 * N, no = N * (2 * N - 1);
  auto Ael = [&](int b, int i, int j) -> double2 {  // coeff * (D^-1)_ij of block b
    double2 v;
    if (i == j) v = make_double2(idg[((long)b * n + i) * lp + d], 0.0);
    else if (i > j) v = iod[((long)b * no + i * (i - 1) / 2 + j) * lp + d];
    else {
      double2 w = iod[((long)b * no + j * (j - 1) / 2 + i) * lp + d];
      v = make_double2(w.x, -w.y);
    }
    return make_double2(coeff * v.x, coeff * v.y);
  };
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++) {
      int ij = i * N + j;
      double2 a21 = Ael(0, i + N, j), a12c = Ael(0, j + N, i), a43 = Ael(1, i + N, j), a34c = Ael(1, j + N, i);
      double2 a12 = make_double2(a12c.x, -a12c.y), a34 = make_double2(a34c.x, -a34c.y);
      // the inverse is Hermitian, so conj(A[j][i]) = A[i][j] on both branches of the reference
      double2 a11 = Ael(0, i, j), a22 = Ael(0, i + N, j + N), a33 = Ael(1, i, j), a44 = Ael(1, i + N, j + N);
      double2 *f = clf + (long)ij * lp + d;
      const long qs = (long)N * N * lp;
      if (REAL) {
        f[0 * qs].x += a12.y + a21.y - a34.y - a43.y;
        f[1 * qs].x += a12.x - a21.x + a43.x - a34.x;
        f[2 * qs].x += a22.y - a11.y + a44.y - a33.y;
        f[3 * qs].x += a11.y - a22.y + a44.y - a33.y;
        f[4 * qs].x += a12.x - a21.x + a34.x - a43.x;
        f[5 * qs].x -= a12.y + a21.y + a34.y + a43.y;
      } else {
        double2 s;
        // -= i (a12 + a21 - a34 - a43)
        s = make_double2(a12.x + a21.x - a34.x - a43.x, a12.y + a21.y - a34.y - a43.y);
        f[0 * qs].x += s.y; f[0 * qs].y -= s.x;
        s = make_double2(a12.x - a21.x + a43.x - a34.x, a12.y - a21.y + a43.y - a34.y);
        f[1 * qs].x += s.x; f[1 * qs].y += s.y;
        s = make_double2(a22.x - a11.x + a44.x - a33.x, a22.y - a11.y + a44.y - a33.y);
        f[2 * qs].x += s.y; f[2 * qs].y -= s.x;
        s = make_double2(a11.x - a22.x + a44.x - a33.x, a11.y - a22.y + a44.y - a33.y);
        f[3 * qs].x += s.y; f[3 * qs].y -= s.x;
        s = make_double2(a12.x - a21.x + a34.x - a43.x, a12.y - a21.y + a34.y - a43.y);
        f[4 * qs].x += s.x; f[4 * qs].y += s.y;
        // += i (a12 + a21 + a34 + a43)
        s = make_double2(a12.x + a21.x + a34.x + a43.x, a12.y + a21.y + a34.y + a43.y);
        f[5 * qs].x -= s.y; f[5 * qs].y += s.x;
      }
    }
}

template <int N, bool REAL, int E, int FR = 0>
static void launch_force_w3(double *fsum, const void *U, const double2 *X, const double2 *Y, Geo g, int dimg,
                            double coeff, size_t smem, bool pf, int st = 0) {
  const unsigned grid = 4 * nb(2L * g.ld, 64);
  if constexpr (!REAL && FR == 0) {
    if (st != 0) {
      // the staged link (and spinors) after the generator sums
      smem += sizeof(double2) * N * N * 64 + (st == 2 ? sizeof(double2) * 4 * 4 * N * 32 : 0);
      if (st == 1) {
        cudaFuncSetAttribute(k_force_hop_w3<N, REAL, E, false, 0, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        k_force_hop_w3<N, REAL, E, false, 0, 1><<<grid, 128, smem, L.stream>>>(fsum, U, X, Y, g, dimg, coeff);
      } else {
        cudaFuncSetAttribute(k_force_hop_w3<N, REAL, E, false, 0, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        k_force_hop_w3<N, REAL, E, false, 0, 2><<<grid, 128, smem, L.stream>>>(fsum, U, X, Y, g, dimg, coeff);
      }
      return;
    }
  }
  if constexpr (FR != 0) {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(k_force_hop_w3<N, REAL, E, false, FR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_force_hop_w3<N, REAL, E, false, FR><<<grid, 128, smem, L.stream>>>(fsum, U, X, Y, g, dimg, coeff, L.Ug,
                                                                           L.recon12 == 4);
  } else if (pf) {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(k_force_hop_w3<N, REAL, E, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_force_hop_w3<N, REAL, E, true><<<grid, 128, smem, L.stream>>>(fsum, U, X, Y, g, dimg, coeff);
  } else {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(k_force_hop_w3<N, REAL, E, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_force_hop_w3<N, REAL, E, false><<<grid, 128, smem, L.stream>>>(fsum, U, X, Y, g, dimg, coeff);
  }
}

// variant 1: one lane per link (k_force_hop_w); 2: two lanes per link in two
// warps with the constant table (k_force_hop_w3); 3: 2 with the L2 prefetches;
// 4: 2 with the NF = 6 two-index links built from the fundamental ones (link
// modes 3 and 4; elsewhere variant 2); 5: 2 with the link staged in shared
// memory by cp.async (the default for complex links); 6: 5 with the spinor at
// x staged too (5 and 6: complex links; real ones run 2).  Variants 2-6 need
// the padded table (ft_E > 0); without it variant 1 runs.
template <int N, bool REAL>
static void launch_force_w(double *fsum, const void *U, const double2 *X, const double2 *Y, Geo g, ProjTabK P,
                           double coeff, size_t smem, int variant) {
  if constexpr ((!REAL && N <= 6) || (REAL && N == 3)) {
    if (variant >= 2 && ft_E > 0) {
      if constexpr (N == 6 && !REAL) {
        if (variant == 4 && L.recon_allow && L.recon12 >= 3 && L.Ug) {
          const bool sym = L.repr == HRGPU_SYM;
          if (ft_E == 2) {
            if (sym) launch_force_w3<N, REAL, 2, 1>(fsum, U, X, Y, g, P.dimg, coeff, smem, false);
            else launch_force_w3<N, REAL, 2, 2>(fsum, U, X, Y, g, P.dimg, coeff, smem, false);
          } else if (ft_E == 3) {
            if (sym) launch_force_w3<N, REAL, 3, 1>(fsum, U, X, Y, g, P.dimg, coeff, smem, false);
            else launch_force_w3<N, REAL, 3, 2>(fsum, U, X, Y, g, P.dimg, coeff, smem, false);
          } else {
            if (sym) launch_force_w3<N, REAL, 5, 1>(fsum, U, X, Y, g, P.dimg, coeff, smem, false);
            else launch_force_w3<N, REAL, 5, 2>(fsum, U, X, Y, g, P.dimg, coeff, smem, false);
          }
          return;
        }
      }
      const bool pf = variant == 3;
      const int st = variant == 5 ? 1 : variant == 6 ? 2 : 0;
      if (ft_E == 2) launch_force_w3<N, REAL, 2>(fsum, U, X, Y, g, P.dimg, coeff, smem, pf, st);
      else if (ft_E == 3) launch_force_w3<N, REAL, 3>(fsum, U, X, Y, g, P.dimg, coeff, smem, pf, st);
      else launch_force_w3<N, REAL, 5>(fsum, U, X, Y, g, P.dimg, coeff, smem, pf, st);
    } else {
      if (smem > 48 * 1024)
        cudaFuncSetAttribute(k_force_hop_w<N, REAL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      k_force_hop_w<N, REAL><<<dim3(nb(2L * g.ld), 4), 128, smem, L.stream>>>(fsum, U, X, Y, g, P, coeff);
    }
  }
}

static ProjTab proj() {
  ProjTab P;
  P.off = L.d_proj_off;
  P.k = L.d_proj_k;
  P.c = L.d_proj_c;
  P.dimg = L.dimg;
  return P;
}

static int ensure_force() {
  if (!L.force_sum) {
    size_t b = sizeof(double) * 4 * L.dimg * 2 * L.ld;
    HR_CUDA(cudaMalloc(&L.force_sum, b));
    HR_CUDA(cudaMemsetAsync(L.force_sum, 0, b, L.stream));
  }
  return 0;
}

int links_out(void *host, const void *dev, int nel, int elem_bytes, int ndir);

}  // namespace hrgpu

namespace hrgpu {

// the clover part of fermion_force_end (force_fermion_core.c:964-984), into force_sum
int fermion_force_finish(double dt) {
  if (!L.clover) return 0;
  if (int rc = check_gauge(HRGPU_DOUBLE)) return rc;
  const double coeff = dt * (L.repr_norm2 / L.fund_norm2) * (1. / 8.) * L.csw;
  Geo g = make_geo();
  const long n = 2L * L.ld;
  HR_NF_DISPATCH(L.real, L.nf, (k_force_clover_core<N_, R_><<<dim3(nb(n, 64), 4), 64, 0, L.stream>>>(L.force_sum, L.U, L.cl_force, g, proj(), coeff)));
  HR_LAUNCH_CHECK();
  return 0;
}

}  // namespace hrgpu

using namespace hrgpu;

extern "C" {

int hrgpu_fermion_force_begin(void) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "fermion_force_begin: lattice not initialised");
  if (int rc = ensure_force()) return rc;
  HR_CUDA(cudaMemsetAsync(L.force_sum, 0, sizeof(double) * 4 * L.dimg * 2 * L.ld, L.stream));
  if (L.clover && L.cl_force)
    HR_CUDA(cudaMemsetAsync(L.cl_force, 0, sizeof(double2) * 6 * L.nf * L.nf * 2 * L.ld, L.stream));
  return 0;
}

int hrgpu_force_fermion_core(void *Xs, void *Ys, int auto_fill_odd, double dt, double residue) {
  if (int rc = check_gauge(HRGPU_DOUBLE)) return rc;
  HR_REQUIRE(Xs && Ys && Xs != Ys, HRGPU_E_ARG, "force_fermion_core: bad fields");
  if (int rc = ensure_force()) return rc;
  const size_t half = (size_t)4 * L.nf * L.ld;
  double2 *X = (double2 *)Xs, *Y = (double2 *)Ys;
  if (auto_fill_odd) {
    const double mass = static_mass();
    if (L.clover) {
      if (int rc = clover_prepare(mass, HRGPU_DOUBLE)) return rc;
      const double *ddg, *idg;
      const double2 *dod, *iod;
      clover_blocks<double>(&ddg, &dod, &idg, &iod);
      if (int rc = hop<double>(HRGPU_ODD, X + half, X, EP_CLOV_INV, -0.5, nullptr, 0.0, 0, nullptr, idg, iod)) return rc;
      if (int rc = hop<double>(HRGPU_ODD, Y + half, Y, EP_CLOV_INV, -0.5, nullptr, 0.0, 0, nullptr, idg, iod)) return rc;
    } else {
      if (int rc = hop<double>(HRGPU_ODD, X + half, X, EP_AXPY, -0.5, nullptr, 0.0, 0, nullptr, nullptr, nullptr)) return rc;
      if (int rc = hop<double>(HRGPU_ODD, Y + half, Y, EP_AXPY, -0.5, nullptr, 0.0, 0, nullptr, nullptr, nullptr)) return rc;
    }
  }
  // UPDATE_EO sign (force_fermion_core.c:825)
  const double coeff = -residue * dt * (L.repr_norm2 / L.fund_norm2);
  Geo g = make_geo();
  const long n = 2L * L.ld;
  if (L.clover && L.expclover) {
    HR_NF_DISPATCH(L.real, L.nf, (launch_force_expclover<N_, R_>(L.cl_force, L.cl_term, X, Y, g, 4.0 + static_mass(), residue)));
  } else if (L.clover) {
    HR_NF_DISPATCH(L.real, L.nf, (k_force_clover_fermion<N_, R_><<<dim3(nb(n), 6), 128, 0, L.stream>>>(L.cl_force, X, Y, g, residue)));
    HR_LAUNCH_CHECK();
  }
  if ((!L.real && L.nf <= 6) || (L.real && L.nf == 3)) {
    ProjTabK P;
    P.off = L.d_projk_off;
    P.A = L.d_projk_A;
    P.c = L.d_projk_c;
    P.dimg = L.dimg;
    const size_t smem = sizeof(double) * 128 * L.dimg;
    if (int rc = force_table_upload()) return rc;
    const int variant = L.force_variant ? L.force_variant : (L.real ? 2 : 5);
    HR_NF_DISPATCH(L.real, L.nf, (launch_force_w<N_, R_>(L.force_sum, L.U, X, Y, g, P, coeff, smem, variant)));
  } else {
    HR_NF_DISPATCH(L.real, L.nf, (k_force_hop<N_, R_><<<dim3(nb(n), 4), 128, 0, L.stream>>>(L.force_sum, L.U, X, Y, g, proj(), coeff)));
  }
  HR_LAUNCH_CHECK();
  return 0;
}

int hrgpu_set_force_variant(int variant) {
  HR_REQUIRE(variant >= 0 && variant <= 6, HRGPU_E_ARG, "set_force_variant: variant must be 0..6");
  L.force_variant = variant;
  return 0;
}

int hrgpu_force_clover_logdet(double mass, double residue) {
  HR_REQUIRE(L.ready && L.clover, HRGPU_E_STATE, "force_clover_logdet: no clover term");
  // the exponential clover blocks are traceless: det D_oo does not depend on the
  // links and there is no log-det force (the reference has the function for
  // WITH_CLOVER only, force_fermion_core.c:776-782)
  if (L.expclover) return 0;
  if (int rc = clover_prepare(mass, HRGPU_DOUBLE)) return rc;
  Geo g = make_geo();
  HR_NF_DISPATCH(L.real, L.nf, (k_force_logdet<N_, R_><<<nb(L.VH), 128, 0, L.stream>>>(L.cl_force, L.cl_idg, L.cl_iod, g, residue)));
  HR_LAUNCH_CHECK();
  return 0;
}

int hrgpu_fermion_force_end(double dt, double *force_host) {
  HR_REQUIRE(L.ready && L.force_sum, HRGPU_E_STATE, "fermion_force_end: no force accumulated");
  HR_REQUIRE(force_host, HRGPU_E_ARG, "fermion_force_end: NULL force field");
  if (int rc = fermion_force_finish(dt)) return rc;
  const size_t m = (size_t)L.V * 4 * L.dimg;
  double *tmp = new double[m];
  int rc = links_out(tmp, L.force_sum, L.dimg, 8, 4);
  if (rc == 0)
    for (size_t i = 0; i < m; i++) force_host[i] += tmp[i];
  delete[] tmp;
  return rc;
}

// cl_force (the six sigma-insertion matrices per site that force_fermion_core's
// clover part accumulates) in HiRep's layout [V][6][NF*NF] complex
int hrgpu_clover_force_get(void *host) {
  HR_REQUIRE(L.ready && L.clover && L.cl_force, HRGPU_E_STATE, "clover_force_get: no clover force accumulated");
  HR_REQUIRE(host, HRGPU_E_ARG, "clover_force_get: NULL output");
  return links_out(host, L.cl_force, L.nf * L.nf, 16, 6);
}

int hrgpu_force_sum_get(double *host) {
  HR_REQUIRE(L.ready && L.force_sum, HRGPU_E_STATE, "force_sum_get: no force accumulated");
  return links_out(host, L.force_sum, L.dimg, 8, 4);
}

}  // extern "C"
