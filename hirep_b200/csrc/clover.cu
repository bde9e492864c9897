// clover.cu -- clover term on the device (LibHR/Update/clover_tools.c).
//
// The clover term A (four NF x NF blocks s0..s3 per site, clover_tools.c:161-206)
// is built from the four-leaf loops.  For the operators it is repacked as two
// Hermitian 2NF x 2NF blocks per site,
//   block 0 = [[s0, s1], [s1^+, -s0]] acting on spin (0,1)
//   block 1 = [[s2, s3], [s3^+, -s2]] acting on spin (2,3)     (Dphi.c:1113-1131)
// stored as packed lower triangles (real diagonal, complex strict lower part).
// D = (4+m) + A is kept packed, and so is D^-1, computed in FP64 from HiRep's
// LDL factorisation (clover_tools.c:97-159) followed by forward/back
// substitution of unit vectors (as in _compute_clover_force, :208-250).  The
// operators then apply D or D^-1 as a dense Hermitian mat-vec fused into the
// hopping kernel's epilogue instead of a per-site triangular solve.
#include "dirac.cuh"

namespace hrgpu {

static inline unsigned nb(long n, int t = 128) { return (unsigned)((n + t - 1) / t); }

// four-leaf loop (clover_tools.c:59-95)
template <int N, bool REAL>
__device__ void clover_loop_dev(CMat<N> &u, const void *U, const Geo &g, long lp, int t, int x, int y, int z, int mu,
                                int nu) {
  CMat<N> a, b, s1, s2, s3;
  long id = ((t + x + y + z) & 1) * g.ld + coords_to_cb(g, t, x, y, z);
  // leaf 1
  long o1 = nbr_index(g, t, x, y, z, mu, +1), o2 = nbr_index(g, t, x, y, z, nu, +1);
  mload<N, REAL>(a, U, mu, id, lp); mload<N, REAL>(b, U, nu, o1, lp); mmul<N, false, false>(s1, a, b);
  mload<N, REAL>(a, U, nu, id, lp); mload<N, REAL>(b, U, mu, o2, lp); mmul<N, false, false>(s2, a, b);
  mmul<N, false, true>(u, s1, s2);
  // leaf 2: o1 = x-mu, o2 = x-mu+nu
  int tt = t, xx = x, yy = y, zz = z;
  {
    int c[4] = {t, x, y, z};
    c[mu] = (c[mu] - 1 + (mu == 0 ? g.T : mu == 1 ? g.X : mu == 2 ? g.Y : g.Z)) % (mu == 0 ? g.T : mu == 1 ? g.X : mu == 2 ? g.Y : g.Z);
    tt = c[0]; xx = c[1]; yy = c[2]; zz = c[3];
  }
  o1 = nbr_index(g, t, x, y, z, mu, -1);
  o2 = nbr_index(g, tt, xx, yy, zz, nu, +1);
  mload<N, REAL>(a, U, nu, o1, lp); mload<N, REAL>(b, U, mu, o2, lp); mmul<N, false, false>(s1, a, b);
  mload<N, REAL>(a, U, nu, id, lp); mmul<N, false, true>(s2, a, s1);
  mload<N, REAL>(a, U, mu, o1, lp); mmul<N, false, false>(s3, s2, a);
  madd(u, s3);
  // leaf 3: o1 = x-mu, o2 = x-nu, o3 = x-mu-nu
  long o3 = nbr_index(g, tt, xx, yy, zz, nu, -1);
  o2 = nbr_index(g, t, x, y, z, nu, -1);
  mload<N, REAL>(a, U, nu, o3, lp); mload<N, REAL>(b, U, mu, o1, lp); mmul<N, false, false>(s1, a, b);
  mload<N, REAL>(a, U, mu, o3, lp); mmul<N, true, false>(s2, s1, a);
  mload<N, REAL>(a, U, nu, o2, lp); mmul<N, false, false>(s3, s2, a);
  madd(u, s3);
  // leaf 4: o1 = x-nu, o2 = x-nu+mu
  {
    int c[4] = {t, x, y, z};
    c[nu] = (c[nu] - 1 + (nu == 0 ? g.T : nu == 1 ? g.X : nu == 2 ? g.Y : g.Z)) % (nu == 0 ? g.T : nu == 1 ? g.X : nu == 2 ? g.Y : g.Z);
    tt = c[0]; xx = c[1]; yy = c[2]; zz = c[3];
  }
  o1 = nbr_index(g, t, x, y, z, nu, -1);
  o2 = nbr_index(g, tt, xx, yy, zz, mu, +1);
  mload<N, REAL>(a, U, nu, o1, lp); mload<N, REAL>(b, U, mu, o1, lp); mmul<N, true, false>(s1, a, b);
  mload<N, REAL>(a, U, nu, o2, lp); mload<N, REAL>(b, U, mu, id, lp); mmul<N, false, true>(s2, a, b);
  mmul<N, false, false>(s3, s1, s2);
  madd(u, s3);
}

// compute_clover_term (clover_tools.c:161-206), one thread per site with the six
// loops in registers: the form for NF <= 4, where they fit
template <int N, bool REAL>
__global__ void k_clover_term(double2 *cl, const void *U, Geo g, double csw) {
  long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= 2L * g.ld) return;
  int p = d >= g.ld ? 1 : 0;
  if (d - p * g.ld >= g.VH) return;
  int t, x, y, z;
  dev_coords(g, (int)d, t, x, y, z);
  const long lp = 2L * g.ld;
  CMat<N> tmp[6];
  clover_loop_dev<N, REAL>(tmp[0], U, g, lp, t, x, y, z, 0, 1);
  clover_loop_dev<N, REAL>(tmp[1], U, g, lp, t, x, y, z, 0, 2);
  clover_loop_dev<N, REAL>(tmp[2], U, g, lp, t, x, y, z, 0, 3);
  clover_loop_dev<N, REAL>(tmp[3], U, g, lp, t, x, y, z, 1, 2);
  clover_loop_dev<N, REAL>(tmp[4], U, g, lp, t, x, y, z, 1, 3);
  clover_loop_dev<N, REAL>(tmp[5], U, g, lp, t, x, y, z, 2, 3);
  const double c = -csw / 16.0;
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++) {
      int ij = i * N + j, ji = j * N + i;
      double2 at, bt, ct, dt;
      if (REAL) {
        // real loops: at = i(t2_ji - t2_ij), bt = i(t3_ij - t3_ji), ct = t1_ji - t1_ij + i(t0_ji - t0_ij),
        // dt = t4_ij - t4_ji + i(t5_ji - t5_ij)
        at = make_double2(0.0, tmp[2].c[ji].x - tmp[2].c[ij].x);
        bt = make_double2(0.0, tmp[3].c[ij].x - tmp[3].c[ji].x);
        ct = make_double2(tmp[1].c[ji].x - tmp[1].c[ij].x, tmp[0].c[ji].x - tmp[0].c[ij].x);
        dt = make_double2(tmp[4].c[ij].x - tmp[4].c[ji].x, tmp[5].c[ji].x - tmp[5].c[ij].x);
      } else {
        double2 q;
        // at = i (conj(t2_ji) - t2_ij)
        q = make_double2(tmp[2].c[ji].x - tmp[2].c[ij].x, -tmp[2].c[ji].y - tmp[2].c[ij].y);
        at = make_double2(-q.y, q.x);
        q = make_double2(tmp[3].c[ij].x - tmp[3].c[ji].x, -tmp[3].c[ij].y - tmp[3].c[ji].y);
        bt = make_double2(-q.y, q.x);
        // ct = i (conj(t0_ji) - t0_ij) - t1_ij + conj(t1_ji)
        q = make_double2(tmp[0].c[ji].x - tmp[0].c[ij].x, -tmp[0].c[ji].y - tmp[0].c[ij].y);
        ct = make_double2(-q.y - tmp[1].c[ij].x + tmp[1].c[ji].x, q.x - tmp[1].c[ij].y - tmp[1].c[ji].y);
        // dt = t4_ij - conj(t4_ji) + i (conj(t5_ji) - t5_ij)
        q = make_double2(tmp[5].c[ji].x - tmp[5].c[ij].x, -tmp[5].c[ji].y - tmp[5].c[ij].y);
        dt = make_double2(tmp[4].c[ij].x - tmp[4].c[ji].x - q.y, tmp[4].c[ij].y + tmp[4].c[ji].y + q.x);
      }
      double2 bc = make_double2(bt.x, -bt.y);  // conj(bt)
      cl[((long)0 * N * N + ij) * lp + d] = make_double2(c * (at.x - bc.x), c * (at.y - bc.y));
      cl[((long)1 * N * N + ij) * lp + d] = make_double2(c * (ct.x - dt.x), c * (ct.y - dt.y));
      cl[((long)2 * N * N + ij) * lp + d] = make_double2(-c * (at.x + bc.x), -c * (at.y + bc.y));
      cl[((long)3 * N * N + ij) * lp + d] = make_double2(-c * (ct.x + dt.x), -c * (ct.y + dt.y));
    }
}

// compute_clover_term for NF >= 5, one thread per (site, plane):
// the thread forms plane q's four-leaf loop (the sum of the four plaquettes of
// clover_tools.c:59-95) row by row, each row r as a row vector carried through
// each leaf's four links, e_r U1 U2 U3 U4 (with daggers as the leaf has them),
// reading the link elements from L1/L2, so no NF x NF temporaries are held.
// The lanes of a warp are consecutive sites with the same plane, so each
// link-element load is one contiguous run.  Blocks (in two launches)
// hold the planes that one pair of output blocks needs: (0,3) and (1,2) give
// s0 and s2, (0,1) (0,2) (1,3) (2,3) give s1 and s3; the rows meet in shared
// memory and are combined, c = -csw/16 times the reference's combinations of
// the loops and their conjugate transposes.  The products are associated row
// first instead of pairwise, so the blocks agree with the reference to
// rounding.  (One thread per site holding the six loops and a loop's
// temporaries, 7 KB of local memory at NF = 6, took 58 ms at 24^3x48.)
template <int N>
struct CTSites {
  static constexpr int v = N <= 6 ? 32 : (N <= 10 ? 16 : 8);  // sites per block
};

template <int N, bool REAL>
__device__ __forceinline__ double2 lnk(const void *U, int mu, long d, int k, long lp) {
  if (REAL) return make_double2(__ldg((const double *)U + ((long)mu * N * N + k) * lp + d), 0.0);
  return __ldg((const double2 *)U + ((long)mu * N * N + k) * lp + d);
}

// v = row r of the link (mu, d), or of its dagger
template <int N, bool REAL, bool DAG>
__device__ __forceinline__ void vrow(double2 (&v)[N], const void *U, int mu, long d, long lp, int r) {
#pragma unroll
  for (int j = 0; j < N; j++) {
    const double2 m = DAG ? lnk<N, REAL>(U, mu, d, j * N + r, lp) : lnk<N, REAL>(U, mu, d, r * N + j, lp);
    v[j] = DAG ? make_double2(m.x, -m.y) : m;
  }
}

// v <- v M with M the link (mu, d) or its dagger
template <int N, bool REAL, bool DAG>
__device__ __forceinline__ void vmul(double2 (&v)[N], const void *U, int mu, long d, long lp) {
  double2 w[N];
#pragma unroll
  for (int j = 0; j < N; j++) w[j] = make_double2(0.0, 0.0);
#pragma unroll
  for (int k = 0; k < N; k++) {
#pragma unroll
    for (int j = 0; j < N; j++) {
      if (DAG) cmacc(w[j], lnk<N, REAL>(U, mu, d, j * N + k, lp), v[k]);  // conj(M_jk) v_k
      else cmac(w[j], v[k], lnk<N, REAL>(U, mu, d, k * N + j, lp));
    }
  }
#pragma unroll
  for (int j = 0; j < N; j++) v[j] = w[j];
}

__device__ __forceinline__ long site_shift(const Geo &g, int t, int x, int y, int z, int mu, int a, int nu, int b) {
  int c[4] = {t, x, y, z};
  const int Ls[4] = {g.T, g.X, g.Y, g.Z};
  c[mu] = (c[mu] + a + Ls[mu]) % Ls[mu];
  c[nu] = (c[nu] + b + Ls[nu]) % Ls[nu];
  return (long)((c[0] + c[1] + c[2] + c[3]) & 1) * g.ld + coords_to_cb(g, c[0], c[1], c[2], c[3]);
}

// GROUP 0: planes 2, 3 -> blocks 0, 2; GROUP 1: planes 0, 1, 4, 5 -> blocks 1, 3
template <int N, bool REAL, int GROUP>
__global__ void __launch_bounds__(CTSites<N>::v * (GROUP ? 4 : 2)) k_clover_term_r(double2 *cl, const void *U, Geo g,
                                                                                 double csw) {
  constexpr int SB = CTSites<N>::v, NP = GROUP ? 4 : 2;
  extern __shared__ double2 ct_sm[];  // [NP][N rows][N][SB]
  const int tid = threadIdx.x, sl = tid % SB, pl = tid / SB;
  const int q = GROUP ? (pl < 2 ? pl : pl + 2) : 2 + pl;  // HiRep's plane index
  const long lp = 2L * g.ld;
  auto site_ok = [&](long d) {
    const int p = d >= g.ld ? 1 : 0;
    return d < 2L * g.ld && d - p * g.ld < g.VH;
  };
  const long d0 = (long)blockIdx.x * SB + sl;
  int t = 0, x = 0, y = 0, z = 0;
  if (site_ok(d0)) dev_coords(g, (int)d0, t, x, y, z);
  for (int r = 0; r < N; r++) {  // the rows of this thread's loop, one after the other
    const long d = d0;
    double2 acc[N], v[N];
#pragma unroll
    for (int j = 0; j < N; j++) acc[j] = make_double2(0.0, 0.0);
    if (site_ok(d)) {
      // planes in HiRep's order: (0,1) (0,2) (0,3) (1,2) (1,3) (2,3)
      const int mu = q < 3 ? 0 : (q < 5 ? 1 : 2), nu = q < 3 ? q + 1 : (q < 5 ? q - 1 : 3);
      const long x0 = site_shift(g, t, x, y, z, mu, 0, nu, 0);
      const long xpm = site_shift(g, t, x, y, z, mu, 1, nu, 0), xpn = site_shift(g, t, x, y, z, mu, 0, nu, 1);
      const long xmm = site_shift(g, t, x, y, z, mu, -1, nu, 0), xmn = site_shift(g, t, x, y, z, mu, 0, nu, -1);
      const long xmmpn = site_shift(g, t, x, y, z, mu, -1, nu, 1), xmmmn = site_shift(g, t, x, y, z, mu, -1, nu, -1);
      const long xpmmn = site_shift(g, t, x, y, z, mu, 1, nu, -1);
      // leaf 1: U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+
      vrow<N, REAL, false>(v, U, mu, x0, lp, r);
      vmul<N, REAL, false>(v, U, nu, xpm, lp);
      vmul<N, REAL, true>(v, U, mu, xpn, lp);
      vmul<N, REAL, true>(v, U, nu, x0, lp);
#pragma unroll
      for (int j = 0; j < N; j++) acc[j] = cadd(acc[j], v[j]);
      // leaf 2: U_nu(x) U_mu(x-mu+nu)^+ U_nu(x-mu)^+ U_mu(x-mu)
      vrow<N, REAL, false>(v, U, nu, x0, lp, r);
      vmul<N, REAL, true>(v, U, mu, xmmpn, lp);
      vmul<N, REAL, true>(v, U, nu, xmm, lp);
      vmul<N, REAL, false>(v, U, mu, xmm, lp);
#pragma unroll
      for (int j = 0; j < N; j++) acc[j] = cadd(acc[j], v[j]);
      // leaf 3: U_mu(x-mu)^+ U_nu(x-mu-nu)^+ U_mu(x-mu-nu) U_nu(x-nu)
      vrow<N, REAL, true>(v, U, mu, xmm, lp, r);
      vmul<N, REAL, true>(v, U, nu, xmmmn, lp);
      vmul<N, REAL, false>(v, U, mu, xmmmn, lp);
      vmul<N, REAL, false>(v, U, nu, xmn, lp);
#pragma unroll
      for (int j = 0; j < N; j++) acc[j] = cadd(acc[j], v[j]);
      // leaf 4: U_nu(x-nu)^+ U_mu(x-nu) U_nu(x-nu+mu) U_mu(x)^+
      vrow<N, REAL, true>(v, U, nu, xmn, lp, r);
      vmul<N, REAL, false>(v, U, mu, xmn, lp);
      vmul<N, REAL, false>(v, U, nu, xpmmn, lp);
      vmul<N, REAL, true>(v, U, mu, x0, lp);
#pragma unroll
      for (int j = 0; j < N; j++) acc[j] = cadd(acc[j], v[j]);
    }
#pragma unroll
    for (int j = 0; j < N; j++) ct_sm[(((long)pl * N + r) * N + j) * SB + sl] = acc[j];
  }
  __syncthreads();
  const double c = -csw / 16.0;
  for (int o = tid; o < SB * N * N; o += SB * NP) {
    const int s2 = o % SB, ij = o / SB, i = ij / N, j = ij % N, ji = j * N + i;
    const long d = (long)blockIdx.x * SB + s2;
    if (!site_ok(d)) continue;
    // loop of plane slot p, element e (row e / N, column e % N)
    auto T = [&](int p, int e) { return ct_sm[((long)p * N * N + e) * SB + s2]; };
    if (GROUP == 0) {  // slots 0, 1 = planes 2, 3
      double2 at, bt;
      if (REAL) {
        at = make_double2(0.0, T(0, ji).x - T(0, ij).x);
        bt = make_double2(0.0, T(1, ij).x - T(1, ji).x);
      } else {
        double2 qq = make_double2(T(0, ji).x - T(0, ij).x, -T(0, ji).y - T(0, ij).y);
        at = make_double2(-qq.y, qq.x);
        qq = make_double2(T(1, ij).x - T(1, ji).x, -T(1, ij).y - T(1, ji).y);
        bt = make_double2(-qq.y, qq.x);
      }
      const double2 bc = make_double2(bt.x, -bt.y);
      cl[((long)0 * N * N + ij) * lp + d] = make_double2(c * (at.x - bc.x), c * (at.y - bc.y));
      cl[((long)2 * N * N + ij) * lp + d] = make_double2(-c * (at.x + bc.x), -c * (at.y + bc.y));
    } else {  // slots 0, 1, 2, 3 = planes 0, 1, 4, 5
      double2 ct, dt;
      if (REAL) {
        ct = make_double2(T(1, ji).x - T(1, ij).x, T(0, ji).x - T(0, ij).x);
        dt = make_double2(T(2, ij).x - T(2, ji).x, T(3, ji).x - T(3, ij).x);
      } else {
        double2 qq = make_double2(T(0, ji).x - T(0, ij).x, -T(0, ji).y - T(0, ij).y);
        ct = make_double2(-qq.y - T(1, ij).x + T(1, ji).x, qq.x - T(1, ij).y - T(1, ji).y);
        qq = make_double2(T(3, ji).x - T(3, ij).x, -T(3, ji).y - T(3, ij).y);
        dt = make_double2(T(2, ij).x - T(2, ji).x - qq.y, T(2, ij).y + T(2, ji).y + qq.x);
      }
      cl[((long)1 * N * N + ij) * lp + d] = make_double2(c * (ct.x - dt.x), c * (ct.y - dt.y));
      cl[((long)3 * N * N + ij) * lp + d] = make_double2(-c * (ct.x + dt.x), -c * (ct.y + dt.y));
    }
  }
}

template <int N, bool REAL>
static void launch_clover_term(double2 *cl, const void *U, Geo g, double csw) {
  constexpr int SB = CTSites<N>::v;
  const size_t smem0 = sizeof(double2) * SB * 2 * N * N, smem1 = 2 * smem0;
  if (smem0 > 48 * 1024)
    cudaFuncSetAttribute(k_clover_term_r<N, REAL, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem0);
  if (smem1 > 48 * 1024)
    cudaFuncSetAttribute(k_clover_term_r<N, REAL, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1);
  const unsigned grid = nb(2L * g.ld, SB);
  k_clover_term_r<N, REAL, 0><<<grid, SB * 2, smem0, L.stream>>>(cl, U, g, csw);
  k_clover_term_r<N, REAL, 1><<<grid, SB * 4, smem1, L.stream>>>(cl, U, g, csw);
}

// measured (compute_clover_term, FP64): 16^3x32 SU(3) 0.39 ms one thread per
// site against 0.80 ms per (site, plane); 16^4 SU(4) antisymmetric 6.4 against
// 3.9 ms; 24^3x48 SU(3) symmetric 57.8 against 48.2 ms
template <int N, bool REAL>
static void launch_clover(double2 *cl, const void *U, Geo g, double csw) {
  if constexpr (N <= 4) {
    k_clover_term<N, REAL><<<nb(2L * g.ld), 128, 0, L.stream>>>(cl, U, g, csw);
  } else {
    launch_clover_term<N, REAL>(cl, U, g, csw);
  }
}

template <int N>
__global__ void k_clover_pack_diag(const double2 *cl, double sigma, double *dg, double2 *od, Geo g) {
  long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= 2L * g.ld) return;
  const long lp = 2L * g.ld;
  const int n = 2 * N;
  for (int b = 0; b < 2; b++) {
    for (int i = 0; i < n; i++) dg[((long)b * n + i) * lp + d] = hblock<N>(cl, b, i, i, lp, d, sigma).x;
    for (int i = 1; i < n; i++)
      for (int j = 0; j < i; j++)
        od[((long)b * N * (2 * N - 1) + i * (i - 1) / 2 + j) * lp + d] = hblock<N>(cl, b, i, j, lp, d, sigma);
  }
}

// LDL (clover_tools.c:97-114) and explicit inverse, packed; ldet: the product
// of the LDL diagonals of both blocks (det D_oo, for clover_la_logdet)
template <int N>
__global__ void k_clover_pack_inv(const double2 *cl, double sigma, double *dg, double2 *od, double *ldet, Geo g) {
  long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= 2L * g.ld) return;
  int p = d >= g.ld ? 1 : 0;
  const long lp = 2L * g.ld;
  constexpr int n = 2 * N;
  if (d - p * g.ld >= g.VH) {
    for (int b = 0; b < 2; b++) {
      for (int i = 0; i < n; i++) dg[((long)b * n + i) * lp + d] = 0.0;
      for (int k = 0; k < N * (2 * N - 1); k++) od[((long)b * N * (2 * N - 1) + k) * lp + d] = make_double2(0.0, 0.0);
    }
    ldet[d] = 1.0;
    return;
  }
  double prod = 1.0;
  double2 A[n * (n + 1) / 2];
  double2 col[n];
#define CP(i, j) A[(i) * ((i) + 1) / 2 + (j)]
  for (int b = 0; b < 2; b++) {
    for (int i = 0; i < n; i++)
      for (int j = 0; j <= i; j++) CP(i, j) = hblock<N>(cl, b, i, j, lp, d, sigma);
    for (int i = 0; i < n; i++) {
      for (int k = 0; k < i; k++) {
        double2 a = CP(i, k);
        double w = (a.x * a.x + a.y * a.y) * CP(k, k).x;
        CP(i, i).x -= w;  // conj(a) a D_k is real
      }
      for (int j = i + 1; j < n; j++) {
        for (int k = 0; k < i; k++) {
          double2 a = CP(i, k), c = CP(j, k);
          // conj(a) * c * D_k
          double2 q = make_double2((a.x * c.x + a.y * c.y) * CP(k, k).x, (a.x * c.y - a.y * c.x) * CP(k, k).x);
          CP(j, i) = csub(CP(j, i), q);
        }
        double di = CP(i, i).x;
        CP(j, i) = make_double2(CP(j, i).x / di, CP(j, i).y / di);
      }
    }
    for (int i = 0; i < n; i++) prod *= CP(i, i).x;
    for (int c = 0; c < n; c++) {
      for (int i = 0; i < n; i++) col[i] = make_double2(i == c ? 1.0 : 0.0, 0.0);
      for (int i = c; i < n; i++)
        for (int k = 0; k < i; k++) {
          double2 l = CP(i, k), v = col[k];
          col[i] = make_double2(col[i].x - (l.x * v.x - l.y * v.y), col[i].y - (l.x * v.y + l.y * v.x));
        }
      for (int i = n - 1; i >= c; i--) {
        double di = CP(i, i).x;
        col[i] = make_double2(col[i].x / di, col[i].y / di);
        for (int k = i + 1; k < n; k++) {
          double2 l = CP(k, i), v = col[k];  // conj(l) * v
          col[i] = make_double2(col[i].x - (l.x * v.x + l.y * v.y), col[i].y - (l.x * v.y - l.y * v.x));
        }
      }
      dg[((long)b * n + c) * lp + d] = col[c].x;
      for (int i = c + 1; i < n; i++) od[((long)b * N * (2 * N - 1) + i * (i - 1) / 2 + c) * lp + d] = col[i];
    }
  }
  ldet[d] = prod;
#undef CP
}

// exponential clover (Dphi.c:1292-1482, LibHR/Utils/clover_exp.c): per chiral
// block A, D = sigma exp(A / sigma) and D^-1 = exp(-A / sigma) / sigma, both
// Hermitian and packed like the blocks above.  The exponential is scaling and
// squaring of the Taylor series to order 20 in FP64 (the reference's series are
// exact to rounding as well).  One block of (2NF)^2 threads per site, one
// matrix element per thread, the matrices in shared memory (this runs once per
// mass).
template <int N>
__global__ void __launch_bounds__(4 * N * N) k_clover_pack_exp(const double2 *cl, double sigma, double *dg, double2 *od, double *idg, double2 *iod,
                                  Geo g) {
  constexpr int n = 2 * N, NO = N * (2 * N - 1);
  __shared__ double2 A[n * n], T[n * n], E[n * n];
  __shared__ int s_sq;
  const long d = blockIdx.x;
  const int p = d >= g.ld ? 1 : 0;
  const long lp = 2L * g.ld;
  const int t = threadIdx.x, i = t / n, j = t % n;
  if (d - p * g.ld >= g.VH) {  // padding sites
    for (int b = 0; b < 2; b++) {
      if (i == j) dg[((long)b * n + i) * lp + d] = idg[((long)b * n + i) * lp + d] = 0.0;
      if (i > j) {
        const long k = ((long)b * NO + i * (i - 1) / 2 + j) * lp + d;
        od[k] = iod[k] = make_double2(0, 0);
      }
    }
    return;
  }
  for (int b = 0; b < 2; b++)
    for (int sgn = 0; sgn < 2; sgn++) {
      const double c = (sgn ? -1.0 : 1.0) / sigma;
      double2 v = (i >= j) ? hblock<N>(cl, b, i, j, lp, d, 0.0) : hblock<N>(cl, b, j, i, lp, d, 0.0);
      if (i < j) v.y = -v.y;
      A[t] = make_double2(c * v.x, c * v.y);
      __syncthreads();
      if (t == 0) {
        double nrm = 0;
        for (int k = 0; k < n * n; k++) nrm += A[k].x * A[k].x + A[k].y * A[k].y;
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
      E[t] = T[t] = make_double2(i == j ? 1.0 : 0.0, 0.0);
      __syncthreads();
      for (int k = 1; k <= 20; k++) {  // T <- T A / k, E += T
        double2 acc = make_double2(0, 0);
        for (int l = 0; l < n; l++) cmac(acc, T[i * n + l], A[l * n + j]);
        __syncthreads();
        T[t] = make_double2(acc.x / k, acc.y / k);
        E[t] = cadd(E[t], T[t]);
        __syncthreads();
      }
      for (int q = 0; q < sq; q++) {  // E <- E E
        double2 acc = make_double2(0, 0);
        for (int l = 0; l < n; l++) cmac(acc, E[i * n + l], E[l * n + j]);
        __syncthreads();
        E[t] = acc;
        __syncthreads();
      }
      const double scale = sgn ? 1.0 / sigma : sigma;
      double *pdg = sgn ? idg : dg;
      double2 *pod = sgn ? iod : od;
      if (i == j) pdg[((long)b * n + i) * lp + d] = scale * E[t].x;
      if (i > j) pod[((long)b * NO + i * (i - 1) / 2 + j) * lp + d] = make_double2(scale * E[t].x, scale * E[t].y);
      __syncthreads();
    }
}

template <typename DST, typename SRC>
__global__ void k_cvt(DST *dst, const SRC *src, long n) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (DST)src[i];
}

// standalone Cphi_diag / Cphi_diag_inv on one parity (aliasing allowed)
template <int N, typename R>
__global__ void k_clover_apply(typename C2<R>::T *out, const typename C2<R>::T *in, const R *dg,
                               const typename C2<R>::T *od, int p, Geo g) {
  typedef typename C2<R>::T V;
  int cb = blockIdx.x * blockDim.x + threadIdx.x;
  if (cb >= g.VH) return;
  const long ld = g.ld, lp = 2L * g.ld, site = (long)p * g.ld + cb;
  V x[2 * N], y[2 * N];
  V res[4 * N];
  for (int b = 0; b < 2; b++) {
    for (int i = 0; i < 2 * N; i++) x[i] = in[(long)(2 * b * N + i) * ld + cb];
    herm_apply<N>(y, x, dg + (long)b * 2 * N * lp, od + (long)b * N * (2 * N - 1) * lp, lp, site, N);
    for (int i = 0; i < 2 * N; i++) res[2 * b * N + i] = y[i];
  }
  for (int k = 0; k < 4 * N; k++) out[(long)k * ld + cb] = res[k];
}

}  // namespace hrgpu

using namespace hrgpu;

namespace hrgpu {

static int alloc_clover() {
  const long lp = 2L * L.ld;
  const int n = 2 * L.nf, no = L.nf * (2 * L.nf - 1), n2 = L.nf * L.nf;
  if (!L.cl_term) {
    HR_CUDA(cudaMalloc(&L.cl_term, sizeof(double2) * 4 * n2 * lp));
    HR_CUDA(cudaMemsetAsync(L.cl_term, 0, sizeof(double2) * 4 * n2 * lp, L.stream));
    HR_CUDA(cudaMalloc(&L.cl_dg, sizeof(double) * 2 * n * lp));
    HR_CUDA(cudaMalloc(&L.cl_od, sizeof(double2) * 2 * no * lp));
    HR_CUDA(cudaMalloc(&L.cl_idg, sizeof(double) * 2 * n * lp));
    HR_CUDA(cudaMalloc(&L.cl_iod, sizeof(double2) * 2 * no * lp));
    HR_CUDA(cudaMalloc(&L.cl_dg_f, sizeof(float) * 2 * n * lp));
    HR_CUDA(cudaMalloc(&L.cl_od_f, sizeof(float2) * 2 * no * lp));
    HR_CUDA(cudaMalloc(&L.cl_idg_f, sizeof(float) * 2 * n * lp));
    HR_CUDA(cudaMalloc(&L.cl_iod_f, sizeof(float2) * 2 * no * lp));
    HR_CUDA(cudaMalloc(&L.cl_force, sizeof(double2) * 6 * n2 * lp));
    HR_CUDA(cudaMalloc(&L.cl_ldet, sizeof(double) * lp));
    HR_CUDA(cudaMemsetAsync(L.cl_force, 0, sizeof(double2) * 6 * n2 * lp, L.stream));
  }
  return 0;
}

int compute_clover_term_dev() {
  HR_REQUIRE(L.clover, HRGPU_E_STATE, "compute_clover_term: clover not initialised");
  if (int rc = check_gauge(HRGPU_DOUBLE)) return rc;
  Geo g = make_geo();
  HR_NF_DISPATCH(L.real, L.nf, (launch_clover<N_, R_>(L.cl_term, L.U, g, L.csw)));
  HR_LAUNCH_CHECK();
  L.sigma = 0xF00F;
  L.sigma_diag = 0xF00F;
  L.sigma_flt = 0xF00F;
  return 0;
}

int clover_prepare(double mass, int prec) {
  const double sigma = 4.0 + mass;
  Geo g = make_geo();
  long n = 2L * L.ld;
  const long lp = 2L * L.ld;
  if (L.expclover && (L.sigma_diag != sigma || L.sigma != sigma)) {
    HR_NFC_DISPATCH(L.nf, (k_clover_pack_exp<N_><<<(unsigned)n, 4 * N_ * N_, 0, L.stream>>>(L.cl_term, sigma, L.cl_dg, L.cl_od, L.cl_idg, L.cl_iod, g)));
    HR_LAUNCH_CHECK();
    L.sigma_diag = L.sigma = sigma;
    L.clover_gen[HRGPU_DOUBLE]++;
  }
  if (L.sigma_diag != sigma) {
    HR_NFC_DISPATCH(L.nf, (k_clover_pack_diag<N_><<<nb(n), 128, 0, L.stream>>>(L.cl_term, sigma, L.cl_dg, L.cl_od, g)));
    HR_LAUNCH_CHECK();
    L.sigma_diag = sigma;
    L.clover_gen[HRGPU_DOUBLE]++;
  }
  if (L.sigma != sigma) {
    HR_NFC_DISPATCH(L.nf, (k_clover_pack_inv<N_><<<nb(n, 64), 64, 0, L.stream>>>(L.cl_term, sigma, L.cl_idg, L.cl_iod, L.cl_ldet, g)));
    HR_LAUNCH_CHECK();
    L.sigma = sigma;
    L.clover_gen[HRGPU_DOUBLE]++;
  }
  if (prec == HRGPU_FLOAT && L.sigma_flt != sigma) {
    const long nd = 2L * 2 * L.nf * lp, no = 2L * L.nf * (2 * L.nf - 1) * lp * 2;
    k_cvt<float, double><<<nb(nd, 256), 256, 0, L.stream>>>(L.cl_dg_f, L.cl_dg, nd);
    k_cvt<float, double><<<nb(no, 256), 256, 0, L.stream>>>((float *)L.cl_od_f, (const double *)L.cl_od, no);
    k_cvt<float, double><<<nb(nd, 256), 256, 0, L.stream>>>(L.cl_idg_f, L.cl_idg, nd);
    k_cvt<float, double><<<nb(no, 256), 256, 0, L.stream>>>((float *)L.cl_iod_f, (const double *)L.cl_iod, no);
    HR_LAUNCH_CHECK();
    L.sigma_flt = sigma;
    L.clover_gen[HRGPU_FLOAT]++;
  }
  return 0;
}

template <>
void clover_blocks<double>(const double **ddg, const double2 **dod, const double **idg, const double2 **iod) {
  *ddg = L.cl_dg; *dod = L.cl_od; *idg = L.cl_idg; *iod = L.cl_iod;
}
template <>
void clover_blocks<float>(const float **ddg, const float2 **dod, const float **idg, const float2 **iod) {
  *ddg = L.cl_dg_f; *dod = L.cl_od_f; *idg = L.cl_idg_f; *iod = L.cl_iod_f;
}

// which: 0 = D = (4+m)+A, 1 = D^-1
int clover_apply(int which, double mass, void *out, const void *in, int par) {
  HR_REQUIRE(L.ready && L.clover, HRGPU_E_STATE, "Cphi_diag: no clover term");
  HR_REQUIRE(out && in && par >= 0 && par <= 2, HRGPU_E_ARG, "Cphi_diag: bad arguments");
  if (int rc = clover_prepare(mass, HRGPU_DOUBLE)) return rc;
  Geo g = make_geo();
  const double *dg = which ? L.cl_idg : L.cl_dg;
  const double2 *od = which ? L.cl_iod : L.cl_od;
  for (int p = 0; p < 2; p++) {
    if (par != HRGPU_FULL && par != p) continue;
    size_t off = par == HRGPU_FULL ? (size_t)p * 4 * L.nf * L.ld : 0;
    double2 *o = (double2 *)out + off;
    const double2 *i = (const double2 *)in + off;
    HR_NFC_DISPATCH(L.nf, (k_clover_apply<N_, double><<<nb(L.VH), 128, 0, L.stream>>>(o, i, dg, od, p, g)));
    HR_LAUNCH_CHECK();
  }
  return 0;
}

int links_out(void *host, const void *dev, int nel, int elem_bytes, int ndir);

}  // namespace hrgpu

extern "C" {

int hrgpu_clover_init(double csw) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "hrgpu_clover_init: lattice not initialised");
  if (int rc = alloc_clover()) return rc;
  L.clover = true;
  L.expclover = false;
  L.csw = csw;
  L.sigma = L.sigma_diag = L.sigma_flt = 0xF00F;
  if (L.have_gauge) return compute_clover_term_dev();
  return 0;
}

int hrgpu_expclover_init(double csw) {
  if (int rc = hrgpu_clover_init(csw)) return rc;
  L.expclover = true;
  return 0;
}

int hrgpu_compute_clover_term(void) { return compute_clover_term_dev(); }

int hrgpu_compute_ldl_decomp(double sigma) {
  HR_REQUIRE(L.ready && L.clover, HRGPU_E_STATE, "hrgpu_compute_ldl_decomp: no clover term");
  return clover_prepare(sigma - 4.0, HRGPU_DOUBLE);
}

int hrgpu_clover_term_get(void *cl_host) {
  HR_REQUIRE(L.ready && L.clover, HRGPU_E_STATE, "hrgpu_clover_term_get: no clover term");
  return links_out(cl_host, L.cl_term, L.nf * L.nf, 16, 4);
}

int hrgpu_Cphi_diag(double mass, void *out, const void *in, int par) { return clover_apply(0, mass, out, in, par); }
int hrgpu_Cphi_diag_inv(double mass, void *out, const void *in, int par) { return clover_apply(1, mass, out, in, par); }

}  // extern "C"
