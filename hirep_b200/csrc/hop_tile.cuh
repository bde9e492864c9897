// hop_tile.cuh -- the hopping kernel on many fields at once (batches).
//
// Batch layout: tiles of TILE_F = 4 fields, and inside a tile blocks of
// TILE_S = 8 sites holding all 4NF components of those sites:
//   element (component c, checkerboard site n, field f) at
//     (((f/4) * ld/8 + n/8) * 4NF + c) * 32 + (n%8) * 4 + f%4
// so the components of one (site, field) sit at a fixed stride of 32 elements:
// one base address per site and immediate offsets for every load.  A thread
// computes one (site, field); a warp holds the 8 sites of a block x the 4
// fields of a tile, so each component load of the warp is one contiguous run
// of 256 bytes (FP32) or 512 bytes (FP64).
//
// Links and clover blocks are read from copies in an array-of-structures-of-
// arrays layout with blocks of TILE_S = 8 sites:
//   links   [parity][site block][mu][NF*NF element][8]
//   clover  [parity][site block][chiral block][packed element][8]
// so the element offsets are compile-time constants, and the 8 sites of a
// warp read one contiguous run per element (64 bytes for FP32 complex).
// The copies are made from the single-field arrays when those change.
#pragma once
#include "hop.cuh"

namespace hrgpu {

constexpr int TILE_F = 4;  // fields per tile
constexpr int TILE_S = 8;  // sites per block of the link and clover copies
constexpr int HOPT_THREADS = 128;

template <typename R>
struct TileArgs {
  const void *in;   // batch at the input parity
  void *out;        // batch at the output parity
  const void *aux;  // batch at the output parity (EP_AXPY, EP_CLOV)
  const void *U;    // link copy [2][ld/8][4][NF*NF][8]
  const R *cdg;     // clover copy, diagonal  [2][ld/8][2][2NF][8]
  const typename C2<R>::T *cod;  // clover copy, off-diagonal [2][ld/8][2][NF(2NF-1)][8]
  const int *stop;  // when non-null and *stop != 0 the launch does nothing
  R cacc, caux;
  int outp, g5, nb;
  Geo g;
};

// Packed FP32 arithmetic (fma.rn.f32x2: two FP32 FMAs in one instruction).
// A complex product u h is (Re u, Re u) (Re h, Im h) + (Im u, Im u) (-Im h, Re h);
// summing P = sum (Re u, Re u) h and Q = sum (Im u, Im u) h separately, the row
// of U h is (P.x - Q.y, P.y + Q.x) and that of U^+ h (P.x + Q.y, P.y - Q.x):
// two packed FMAs per link element and half spinor instead of four.
__device__ __forceinline__ unsigned long long pk2(float x, float y) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(x), "f"(y));
  return r;
}
__device__ __forceinline__ float2 upk2(unsigned long long r) {
  float2 v;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
  return v;
}
__device__ __forceinline__ unsigned long long ffma2(unsigned long long a, unsigned long long b, unsigned long long c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// c0 = U h0, c1 = U h1 (DAG: U^+) for complex FP32 links, packed FMAs
template <int NA, bool DAG>
__device__ __forceinline__ void link_mul2_f2(float2 *c0, float2 *c1, const float2 *h0, const float2 *h1, const float2 *U,
                                             long plane) {
  const unsigned long long pol = l2_evict_first();
  unsigned long long g0[NA], g1[NA];
#pragma unroll
  for (int j = 0; j < NA; j++) {
    g0[j] = pk2(h0[j].x, h0[j].y);
    g1[j] = pk2(h1[j].x, h1[j].y);
  }
#pragma unroll
  for (int i = 0; i < NA; i++) {
    unsigned long long p0 = 0ull, q0 = 0ull, p1 = 0ull, q1 = 0ull;
#pragma unroll
    for (int j = 0; j < NA; j++) {
      const float2 u = ld_ef1(U + (long)(DAG ? j * NA + i : i * NA + j) * plane, pol);
      const unsigned long long ur = pk2(u.x, u.x), ui = pk2(u.y, u.y);
      p0 = ffma2(ur, g0[j], p0);
      q0 = ffma2(ui, g0[j], q0);
      p1 = ffma2(ur, g1[j], p1);
      q1 = ffma2(ui, g1[j], q1);
    }
    const float2 P0 = upk2(p0), Q0 = upk2(q0), P1 = upk2(p1), Q1 = upk2(q1);
    if (!DAG) {
      c0[i] = make_float2(P0.x - Q0.y, P0.y + Q0.x);
      c1[i] = make_float2(P1.x - Q1.y, P1.y + Q1.x);
    } else {
      c0[i] = make_float2(P0.x + Q0.y, P0.y - Q0.x);
      c1[i] = make_float2(P1.x + Q1.y, P1.y - Q1.x);
    }
  }
}

// one (site cb, field f) of the hop with the fused epilogues of k_hop.  The
// eight directions are unrolled so that the loads of a direction are issued
// together (a loop over directions, one direction's loads live at a time and
// twice the resident warps, measured 1.65x slower at NF=6).
template <int NFT, bool REAL, typename R, int EP, bool F2 = false>
__device__ __forceinline__ void hopt_site(const TileArgs<R> &a, const int cb, const int tile, const int lane) {
  typedef typename C2<R>::T V;
  typedef typename LinkE<REAL, R>::T E;
  constexpr int NA = NFT;
  constexpr int nf = NFT;
  constexpr int NS = 4 * NFT;          // components per site
  constexpr int NL = NFT * NFT;        // link elements
  constexpr long LSTEP = TILE_S;       // element stride inside a block of the copies
  const Geo &g = a.g;
  const int outp = a.outp, inp = outp ^ 1;
  const long nblk = g.ld / TILE_S;
  int t, x, y, z;
  cb_to_coords(g, cb, outp, t, x, y, z);
  const long tblk = (long)tile * nblk;  // first site block of this tile
  constexpr int CSTEP = TILE_S * TILE_F;  // component stride in a batch
  const V *in = (const V *)a.in;
  const E *U = (const E *)a.U;
  auto sbase = [&](const V *p, int n) {
    return p + ((tblk + (n >> 3)) * NS) * CSTEP + (n & 7) * TILE_F + lane;
  };
  auto ubase = [&](int p, int n, int mu) {
    return U + (((long)p * nblk + (n >> 3)) * 4 + mu) * NL * LSTEP + (n & 7);
  };
  V r0[NA], r1[NA], r2[NA], r3[NA];
#pragma unroll
  for (int i = 0; i < NA; i++) r0[i] = r1[i] = r2[i] = r3[i] = cmk<V>(0.0, 0.0);
  // forward (bw = 0): (1 - gamma_mu) U(x,mu) psi(x+mu);
  // backward (bw = 1): (1 + gamma_mu) U(x-mu,mu)^+ psi(x-mu)
  auto step = [&](const int mu, const int bw) {
    int tt = t, xx = x, yy = y, zz = z;
    if (mu == 0) tt = bw ? ((t == 0) ? g.T - 1 : t - 1) : ((t + 1 == g.T) ? 0 : t + 1);
    if (mu == 1) xx = bw ? ((x == 0) ? g.X - 1 : x - 1) : ((x + 1 == g.X) ? 0 : x + 1);
    if (mu == 2) yy = bw ? ((y == 0) ? g.Y - 1 : y - 1) : ((y + 1 == g.Y) ? 0 : y + 1);
    if (mu == 3) zz = bw ? ((z == 0) ? g.Z - 1 : z - 1) : ((z + 1 == g.Z) ? 0 : z + 1);
    const int cn = coords_to_cb(g, tt, xx, yy, zz);
    const V *s = sbase(in, cn);
    V h0[NA], h1[NA], c0[NA], c1[NA];
#pragma unroll
    for (int i = 0; i < NA; i++) {
      V s0 = ld_c(s + (0 * nf + i) * CSTEP), s1 = ld_c(s + (1 * nf + i) * CSTEP);
      V s2 = ld_c(s + (2 * nf + i) * CSTEP), s3 = ld_c(s + (3 * nf + i) * CSTEP);
      if (!bw) {
        if (mu == 0) { h0[i] = cadd(s0, s2); h1[i] = cadd(s1, s3); }
        if (mu == 1) { h0[i] = caddi(s0, s3); h1[i] = caddi(s1, s2); }
        if (mu == 2) { h0[i] = cadd(s0, s3); h1[i] = csub(s1, s2); }
        if (mu == 3) { h0[i] = caddi(s0, s2); h1[i] = csubi(s1, s3); }
      } else {
        if (mu == 0) { h0[i] = csub(s0, s2); h1[i] = csub(s1, s3); }
        if (mu == 1) { h0[i] = csubi(s0, s3); h1[i] = csubi(s1, s2); }
        if (mu == 2) { h0[i] = csub(s0, s3); h1[i] = cadd(s1, s2); }
        if (mu == 3) { h0[i] = csubi(s0, s2); h1[i] = caddi(s1, s3); }
      }
    }
    if constexpr (F2) {
      if (!bw) link_mul2_f2<NA, false>(c0, c1, h0, h1, ubase(outp, cb, mu), LSTEP);
      else link_mul2_f2<NA, true>(c0, c1, h0, h1, ubase(inp, cn, mu), LSTEP);
    } else if (!bw) {
      const E *Ub = ubase(outp, cb, mu);
      link_mul<NA, false, 2>(c0, h0, Ub, LSTEP, 0L, nf);
      link_mul<NA, false, 2>(c1, h1, Ub, LSTEP, 0L, nf);
    } else {
      const E *Ub = ubase(inp, cn, mu);
      link_mul<NA, true, 2>(c0, h0, Ub, LSTEP, 0L, nf);
      link_mul<NA, true, 2>(c1, h1, Ub, LSTEP, 0L, nf);
    }
#pragma unroll
    for (int i = 0; i < NA; i++) {
      r0[i] = cadd(r0[i], c0[i]);
      r1[i] = cadd(r1[i], c1[i]);
      if (!bw) {
        if (mu == 0) { r2[i] = cadd(r2[i], c0[i]); r3[i] = cadd(r3[i], c1[i]); }
        if (mu == 1) { r3[i] = csubi(r3[i], c0[i]); r2[i] = csubi(r2[i], c1[i]); }
        if (mu == 2) { r3[i] = cadd(r3[i], c0[i]); r2[i] = csub(r2[i], c1[i]); }
        if (mu == 3) { r2[i] = csubi(r2[i], c0[i]); r3[i] = caddi(r3[i], c1[i]); }
      } else {
        if (mu == 0) { r2[i] = csub(r2[i], c0[i]); r3[i] = csub(r3[i], c1[i]); }
        if (mu == 1) { r3[i] = caddi(r3[i], c0[i]); r2[i] = caddi(r2[i], c1[i]); }
        if (mu == 2) { r3[i] = csub(r3[i], c0[i]); r2[i] = cadd(r2[i], c1[i]); }
        if (mu == 3) { r2[i] = caddi(r2[i], c0[i]); r3[i] = csubi(r3[i], c1[i]); }
      }
    }
  };
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    step(mu, 0);
    step(mu, 1);
  }
  // ---- epilogue
  const R ca = a.cacc;
  V *out = (V *)a.out + ((tblk + (cb >> 3)) * NS) * CSTEP + (cb & 7) * TILE_F + lane;
  if (EP == EP_AXPY) {
    const R cx = a.caux;
    const bool use_aux = a.aux != nullptr && cx != (R)0;
    const V *aux = use_aux ? sbase((const V *)a.aux, cb) : nullptr;
#pragma unroll
    for (int i = 0; i < NA; i++) {
      V q0 = cscale(ca, r0[i]), q1 = cscale(ca, r1[i]), q2 = cscale(ca, r2[i]), q3 = cscale(ca, r3[i]);
      if (use_aux) {
        rmac(q0, cx, ld_c(aux + (0 * nf + i) * CSTEP));
        rmac(q1, cx, ld_c(aux + (1 * nf + i) * CSTEP));
        rmac(q2, cx, ld_c(aux + (2 * nf + i) * CSTEP));
        rmac(q3, cx, ld_c(aux + (3 * nf + i) * CSTEP));
      }
      r0[i] = q0; r1[i] = q1; r2[i] = q2; r3[i] = q3;
    }
  } else {
    // clover block b acts on spins (2b, 2b+1); packed as in clover_epilogue
    constexpr int N2 = 2 * NFT, NO = NFT * (2 * NFT - 1);
    const long blk = (long)outp * nblk + (cb >> 3);
    const V *aux = (EP == EP_CLOV) ? sbase((const V *)a.aux, cb) : nullptr;
#pragma unroll
    for (int b = 0; b < 2; b++) {
      V(&ra)[NA] = b ? r2 : r0;
      V(&rb)[NA] = b ? r3 : r1;
      V xin[2 * NA], yout[2 * NA];
#pragma unroll
      for (int i = 0; i < NA; i++) {
        if (EP == EP_CLOV_INV) {
          xin[i] = cscale(ca, ra[i]);
          xin[nf + i] = cscale(ca, rb[i]);
        } else {
          xin[i] = ld_c(aux + ((2 * b) * nf + i) * CSTEP);
          xin[nf + i] = ld_c(aux + ((2 * b + 1) * nf + i) * CSTEP);
        }
      }
      const R *dg = a.cdg + ((blk * 2 + b) * N2) * LSTEP + (cb & 7);
      const V *od = a.cod + ((blk * 2 + b) * NO) * LSTEP + (cb & 7);
      herm_apply<NA, 2>(yout, xin, dg, od, LSTEP, 0L, nf);
#pragma unroll
      for (int i = 0; i < NA; i++) {
        if (EP == EP_CLOV_INV) {
          ra[i] = yout[i];
          rb[i] = yout[nf + i];
        } else {
          ra[i] = cadd(cscale(ca, ra[i]), yout[i]);
          rb[i] = cadd(cscale(ca, rb[i]), yout[nf + i]);
        }
      }
    }
  }
  const R sg = a.g5 ? (R)-1 : (R)1;
#pragma unroll
  for (int i = 0; i < NA; i++) {
    out[(0 * nf + i) * CSTEP] = r0[i];
    out[(1 * nf + i) * CSTEP] = r1[i];
    out[(2 * nf + i) * CSTEP] = cscale(sg, r2[i]);
    out[(3 * nf + i) * CSTEP] = cscale(sg, r3[i]);
  }
}

// A warp is 8 consecutive sites x the 4 fields of one tile; the warps of all
// tiles of the same 8 sites are adjacent, so the links and clover blocks of
// those sites are read from DRAM once and then hit in L1/L2 for the other tiles.
template <int NFT, bool REAL, typename R, int EP, int MINB, bool F2 = false>
__global__ void __launch_bounds__(HOPT_THREADS, MINB) k_hopt(TileArgs<R> a) {
  if (a.stop && *a.stop) return;
  const long flat = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = (int)(flat & (TILE_F - 1));
  const int s8 = (int)((flat >> 2) & (TILE_S - 1));
  const long w = flat >> 5;  // (site group, tile) pair of this warp
  const int ntile = (a.nb + TILE_F - 1) / TILE_F;
  const long group = w / ntile;
  const int tile = (int)(w - group * ntile);
  const long cbl = group * TILE_S + s8;
  if (cbl >= a.g.VH || tile * TILE_F + lane >= a.nb) return;
  hopt_site<NFT, REAL, R, EP, F2>(a, (int)cbl, tile, lane);
}

// ---------------------------------------------------------------------------
// the copies in blocks of 8 sites
// ---------------------------------------------------------------------------
// links: src [4][nel][2ld] (site d = p*ld + cb) -> dst [2][ld/8][4][nel][8]
template <typename E>
__global__ void k_tile_links(E *dst, const E *src, int nel, int ld) {
  const long n = 2L * ld * 4 * nel;
  const long nblk = ld / TILE_S;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    // i runs over the destination in order: s8 fastest
    const int s8 = (int)(i % TILE_S);
    long r = i / TILE_S;
    const int e = (int)(r % nel);
    r /= nel;
    const int mu = (int)(r % 4);
    r /= 4;
    const long blk = r % nblk;
    const int p = (int)(r / nblk);
    const long d = (long)p * ld + blk * TILE_S + s8;
    dst[i] = src[((long)mu * nel + e) * 2 * ld + d];
  }
}

// packed clover blocks: src [2 blocks][k][2ld] -> dst [2 parities][ld/8][2 blocks][k][8]
template <typename E>
__global__ void k_tile_clover(E *dst, const E *src, int kn, int ld) {
  const long n = 2L * ld * 2 * kn;
  const long nblk = ld / TILE_S;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int s8 = (int)(i % TILE_S);
    long r = i / TILE_S;
    const int k = (int)(r % kn);
    r /= kn;
    const int b = (int)(r % 2);
    r /= 2;
    const long blk = r % nblk;
    const int p = (int)(r / nblk);
    const long d = (long)p * ld + blk * TILE_S + s8;
    dst[i] = src[((long)b * kn + k) * 2 * ld + d];
  }
}

}  // namespace hrgpu
