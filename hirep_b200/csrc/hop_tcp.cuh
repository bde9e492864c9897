// hop_tcp.cuh -- the tensor-core batched hop with the neighbours prefetched:
// batch variant 4 (FP32, complex NF = 6, nb <= 16).
//
// The per-site GEMM is the one of hop_tc.cuh (rows = output spin x field,
// the eight directions' links stacked along K, complex made real, three TF32
// products for FP32 accuracy).  What differs is the flow, built so that the
// loads, the row building and the MMAs of different sites overlap:
//   * one persistent CTA per SM, two warpgroups; warpgroup g takes every other
//     site of the CTA's list and owns half of the tensor memory (its A rows,
//     hi and lo, 192 columns, and its 16-column accumulator);
//   * the raw data of a site -- the neighbour spinors of its nb fields in the
//     eight directions and its eight links -- are copied global -> shared
//     with cp.async two sites ahead, into a two-slot ring per warpgroup, so a
//     warpgroup builds its rows from shared memory while the copies of its
//     next sites are in flight;
//   * each thread builds its row (spin s, field f) for all eight directions
//     and writes it to tensor memory (tcgen05.st); the links are staged into
//     the B operand in shared memory; one elected thread issues the 36 MMAs of
//     the site and waits on their mbarrier (bounded) while the other warpgroup
//     keeps building; then the warpgroup reads its accumulator and runs the
//     epilogue of k_hopt.
// Warpgroups synchronise with named barriers (ids 1, 2), never with each
// other.  A wait that gives up sets the launch's error word, both warpgroups
// stop taking sites, and the CTA frees its tensor memory.  No multicast.
#pragma once
#include "hop_async.cuh"
#include "hop_tc.cuh"

namespace hrgpu {

constexpr int TCP_THREADS = 256;  // two warpgroups
constexpr int TCP_NBMAX = 16;     // fields of the raw-data slots

template <int NFT>
struct TcpLayout {
  static constexpr int NF = NFT, NF2 = 2 * NFT, NS = 4 * NFT, NL = NFT * NFT;
  static constexpr int K = 8 * NF2;                        // both rounds of hop_tc at once
  static constexpr int RAW = 8 * NS * TCP_NBMAX;           // float2 of neighbour spinors per slot
  static constexpr int LNK = 8 * NL;                       // float2 of links per slot
  static constexpr int SLOT = RAW + LNK;                   // float2 per slot
  static constexpr int BSZ = 16 * K;                       // floats of one B copy (hi or lo)
  static constexpr int XCH = 4 * 32 * NF;                  // float2 of the clover exchange
  // per warpgroup: 2 slots (float2), B hi + lo (float), exchange (float2)
  static constexpr size_t WG_BYTES = 2 * SLOT * 8 + 2 * BSZ * 4 + XCH * 8;
  static constexpr size_t SMEM = 2 * WG_BYTES;
  static constexpr int COL_A = 0, COL_ALO = K, WG_COLS = 2 * K, COL_D = 2 * WG_COLS;  // + 16 g
};

__device__ __forceinline__ void wg_bar(int g) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(128) : "memory");
}

// the neighbour site of cb (output parity outp) in direction d = 2 mu + bw
__device__ __forceinline__ int tcp_nbr(const Geo &g, int t, int x, int y, int z, int d) {
  const int mu = d >> 1, bw = d & 1;
  if (mu == 0) t = bw ? ((t == 0) ? g.T - 1 : t - 1) : ((t + 1 == g.T) ? 0 : t + 1);
  if (mu == 1) x = bw ? ((x == 0) ? g.X - 1 : x - 1) : ((x + 1 == g.X) ? 0 : x + 1);
  if (mu == 2) y = bw ? ((y == 0) ? g.Y - 1 : y - 1) : ((y + 1 == g.Y) ? 0 : y + 1);
  if (mu == 3) z = bw ? ((z == 0) ? g.Z - 1 : z - 1) : ((z + 1 == g.Z) ? 0 : z + 1);
  return coords_to_cb(g, t, x, y, z);
}

// copies of one site's raw data into a slot, by the 128 threads of a warpgroup
template <int NFT>
__device__ __forceinline__ void tcp_fetch(const TileArgs<float> &a, int cb, float2 *slot, int lt) {
  typedef TcpLayout<NFT> Y;
  constexpr int CSTEP = TILE_S * TILE_F;
  const Geo &g = a.g;
  const int outp = a.outp, inp = outp ^ 1;
  const long nblk = g.ld / TILE_S;
  int t, x, y, z;
  cb_to_coords(g, cb, outp, t, x, y, z);
  const int ntile = (a.nb + TILE_F - 1) / TILE_F;
  const float2 *in = (const float2 *)a.in, *U = (const float2 *)a.U;
  // spinors: (direction d, component c, tile T, half h) -> 16 B = fields 4T + 2h, 4T + 2h + 1
  const int nsp = 8 * Y::NS * ntile * 2;
  for (int q = lt; q < nsp; q += 128) {
    const int h = q & 1, T = (q >> 1) % ntile, dc = (q >> 1) / ntile, c = dc % Y::NS, d = dc / Y::NS;
    const int cn = tcp_nbr(g, t, x, y, z, d);
    const float2 *src = in + (((long)T * nblk + (cn >> 3)) * Y::NS + c) * CSTEP + (cn & 7) * TILE_F + 2 * h;
    cp_async16(slot + (d * Y::NS + c) * TCP_NBMAX + 4 * T + 2 * h, src);
  }
  // links: (direction d, element e), 8 B each (elements of a site are 8 float2 apart)
  float2 *lk = slot + Y::RAW;
  for (int q = lt; q < Y::LNK; q += 128) {
    const int e = q % Y::NL, d = q / Y::NL, mu = d >> 1, bw = d & 1;
    long base;
    if (!bw) {
      base = (((long)outp * nblk + (cb >> 3)) * 4 + mu) * Y::NL * TILE_S + (cb & 7);
    } else {
      const int cn = tcp_nbr(g, t, x, y, z, d);
      base = (((long)inp * nblk + (cn >> 3)) * 4 + mu) * Y::NL * TILE_S + (cn & 7);
    }
    cp_async8(lk + q, U + base + (long)e * TILE_S);
  }
}

template <int NFT, int EP>
__global__ void __launch_bounds__(TCP_THREADS, 1) k_hopt_tcp(TileArgs<float> a, unsigned *err) {
  typedef TcpLayout<NFT> Y;
  constexpr int NF = NFT, NF2 = Y::NF2, NS = Y::NS, K = Y::K;
  constexpr uint32_t SBO = (K / 4) * 128, LBO = 128;
  constexpr int CSTEP = TILE_S * TILE_F;
  constexpr long LSTEP = TILE_S;
  static_assert(NF2 % 4 == 0 && 2 * Y::WG_COLS + 32 <= 512, "tensor-core hop (prefetched): NF");
  extern __shared__ __align__(128) unsigned char smem_tcp[];
  __shared__ __align__(8) unsigned long long bar[2];
  __shared__ uint32_t taddr_s;
  __shared__ int s_fail[2];  // per warpgroup: written by its MMA thread before a barrier of that warpgroup

  const int tid = threadIdx.x, g = tid >> 7, lt = tid & 127, w = lt >> 5, lane = lt & 31;
  const int s = w, f = lane;  // this thread's row: spin s of field f (TMEM lane 32 w + lane)
  unsigned char *mine = smem_tcp + g * Y::WG_BYTES;
  float2 *slots = (float2 *)mine;                                  // 2 x SLOT
  float *sBhi = (float *)(mine + 2 * Y::SLOT * 8), *sBlo = sBhi + Y::BSZ;
  float2 *xch = (float2 *)(sBlo + Y::BSZ);
  const Geo &gg = a.g;
  const int outp = a.outp;
  const long nblk = gg.ld / TILE_S;
  const bool live = f < a.nb;

  for (int i = lt; i < 2 * Y::BSZ; i += 128) sBhi[i] = 0.f;  // padding rows n >= 2NF stay zero
  if (tid < 2) s_fail[tid] = 0;
  if (tid < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(tc_smem(&taddr_s))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int q = 0; q < 2; q++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&bar[q])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tm = taddr_s;
  const uint32_t rowA = tm + ((uint32_t)(w * 32) << 16) + g * Y::WG_COLS;  // this thread's lanes, its A columns
  const uint32_t colD = Y::COL_D + 16 * g;
  const uint32_t rowD = tm + ((uint32_t)(w * 32) << 16) + colD;
  const uint32_t bar_a = tc_smem(&bar[g]);
  uint32_t parity = 0;
  bool pending = false;
  const bool stopped = a.stop && *a.stop;

  // this warpgroup's sites: k-th is blockIdx.x + gridDim.x (2k + g)
  auto site = [&](int k) { return (int)blockIdx.x + (int)gridDim.x * (2 * k + g); };
  if (!stopped) {
    for (int k = 0; k < 2; k++) {  // prologue: two sites ahead
      if (site(k) < gg.VH) tcp_fetch<NFT>(a, site(k), slots + k * Y::SLOT, lt);
      cp_async_commit();
    }
  }
  for (int k = 0; !stopped; k++) {
    const int cb = site(k);
    if (cb >= gg.VH) break;
    float2 *slot = slots + (k & 1) * Y::SLOT;
    cp_async_wait<1>();
    wg_bar(g);
    int tt, xx, yy, zz;
    cb_to_coords(gg, cb, outp, tt, xx, yy, zz);
    // ---- B: the eight links (threads 0 .. 8NF-1 of the warpgroup)
    if (lt < 8 * NF) {
      const int d = lt / NF, i = lt % NF, bw = d & 1;
      const float2 *lk = slot + Y::RAW + d * Y::NL;
#pragma unroll
      for (int j = 0; j < NF; j++) {
        float2 u = bw ? lk[j * NF + i] : lk[i * NF + j];
        if (bw) u.y = -u.y;
        const float vals[4] = {u.x, -u.y, u.y, u.x};
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int n = (q < 2) ? i : NF + i, kk = d * NF2 + (q & 1) * NF + j;
          const int off = (n >> 3) * (SBO / 4) + (kk >> 2) * (LBO / 4) + (n & 7) * 4 + (kk & 3);
          const float hi = tf32_rn(vals[q]);
          sBhi[off] = hi;
          sBlo[off] = tf32_rn(vals[q] - hi);
        }
      }
    }
    // ---- A: this thread's row for the eight directions (all lanes store: tcgen05.st is warp-collective)
#pragma unroll
    for (int d = 0; d < 8; d++) {
      const TcSpin S = tc_spin(d >> 1, d & 1);
      const int kq = (s == 0) ? 0 : (s == 1) ? 1 : (s == 2) ? S.k2 : S.k3;
      const int beta = (s < 2) ? 0 : (s == 2) ? S.beta2 : S.beta3;
      const int pk = S.p[kq], ak = S.alpha[kq];
      float hv[NF2], lv[NF2];
#pragma unroll
      for (int j = 0; j < NF; j++) {
        float2 v = make_float2(0.f, 0.f);
        if (live) {
          const float2 a0 = slot[(d * NS + kq * NF + j) * TCP_NBMAX + f];
          const float2 a1 = slot[(d * NS + pk * NF + j) * TCP_NBMAX + f];
          v = cphase(cadd(a0, cphase(a1, ak)), beta);
        }
        hv[j] = tf32_rn(v.x);
        lv[j] = tf32_rn(v.x - hv[j]);
        hv[NF + j] = tf32_rn(v.y);
        lv[NF + j] = tf32_rn(v.y - hv[NF + j]);
      }
#pragma unroll
      for (int c = 0; c < NF2; c += 4) {
        tc_st4(rowA + Y::COL_A + d * NF2 + c, hv[c], hv[c + 1], hv[c + 2], hv[c + 3]);
        tc_st4(rowA + Y::COL_ALO + d * NF2 + c, lv[c], lv[c + 1], lv[c + 2], lv[c + 3]);
      }
    }
    wg_bar(g);  // the slot has been read: refill it with the site two ahead
    if (site(k + 2) < gg.VH) tcp_fetch<NFT>(a, site(k + 2), slot, lt);
    cp_async_commit();
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    wg_bar(g);
    if (lt == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      constexpr uint32_t ID = tc_idesc_tf32(128, 16);
      const uint32_t bh = tc_smem(sBhi), bl = tc_smem(sBlo), a0 = tm + g * Y::WG_COLS;
#pragma unroll
      for (int ks = 0; ks < K / 8; ks++) {
        const uint64_t dbh = tc_sdesc(bh + ks * 2 * LBO, LBO, SBO), dbl = tc_sdesc(bl + ks * 2 * LBO, LBO, SBO);
        const uint32_t ahi = a0 + Y::COL_A + ks * 8, alo = a0 + Y::COL_ALO + ks * 8, acc0 = ks > 0 ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.u32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n}\n" ::"r"(
                tm + colD),
            "r"(ahi), "l"(dbh), "r"(ID), "r"(acc0)
            : "memory");
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.u32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n}\n" ::"r"(
                tm + colD),
            "r"(ahi), "l"(dbl), "r"(ID), "r"(1u)
            : "memory");
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.u32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n}\n" ::"r"(
                tm + colD),
            "r"(alo), "l"(dbh), "r"(ID), "r"(1u)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_a)
                   : "memory");
      pending = true;
      const bool ok = tc_wait(bar_a, parity);
      if (ok) pending = false;
      else s_fail[g] = 1;
    }
    parity ^= 1u;
    wg_bar(g);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (s_fail[g]) break;  // uniform over the warpgroup: read after the barrier that follows the only write
    // ---- the accumulator row and the epilogue (as hopt_site)
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(rowD)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    float2 R[NF];
#pragma unroll
    for (int i = 0; i < NF; i++) R[i] = make_float2(__uint_as_float(r[i]), __uint_as_float(r[NF + i]));
    const float ca = a.cacc;
    float2 *outb = (float2 *)a.out + (((long)(f >> 2) * nblk + (cb >> 3)) * NS) * CSTEP + (cb & 7) * TILE_F + (f & 3);
    const float2 *auxb =
        a.aux ? (const float2 *)a.aux + (((long)(f >> 2) * nblk + (cb >> 3)) * NS) * CSTEP + (cb & 7) * TILE_F + (f & 3)
              : nullptr;
    if (EP == EP_AXPY) {
      if (live) {
        const float cx = a.caux;
        const bool use_aux = auxb != nullptr && cx != 0.f;
        const float sg = (a.g5 && s >= 2) ? -1.f : 1.f;
#pragma unroll
        for (int i = 0; i < NF; i++) {
          float2 q = cscale(ca, R[i]);
          if (use_aux) rmac(q, cx, ld_c(auxb + (s * NF + i) * CSTEP));
          outb[(s * NF + i) * CSTEP] = cscale(sg, q);
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < NF; i++) xch[(s * 32 + f) * NF + i] = R[i];
      wg_bar(g);
      if (w < 2 && live) {
        constexpr int N2 = 2 * NFT, NO = NFT * (2 * NFT - 1);
        const int b = w;
        const long blk = (long)outp * nblk + (cb >> 3);
        float2 xin[2 * NF], yout[2 * NF];
#pragma unroll
        for (int i = 0; i < NF; i++) {
          if (EP == EP_CLOV_INV) {
            xin[i] = cscale(ca, xch[((2 * b) * 32 + f) * NF + i]);
            xin[NF + i] = cscale(ca, xch[((2 * b + 1) * 32 + f) * NF + i]);
          } else {
            xin[i] = ld_c(auxb + ((2 * b) * NF + i) * CSTEP);
            xin[NF + i] = ld_c(auxb + ((2 * b + 1) * NF + i) * CSTEP);
          }
        }
        const float *dg = a.cdg + ((blk * 2 + b) * N2) * LSTEP + (cb & 7);
        const float2 *od = a.cod + ((blk * 2 + b) * NO) * LSTEP + (cb & 7);
        herm_apply<NF>(yout, xin, dg, od, LSTEP, 0L, NF);
        const float sgb = (a.g5 && b == 1) ? -1.f : 1.f;
#pragma unroll
        for (int i = 0; i < NF; i++) {
          float2 o0, o1;
          if (EP == EP_CLOV_INV) {
            o0 = yout[i];
            o1 = yout[NF + i];
          } else {
            o0 = cadd(cscale(ca, xch[((2 * b) * 32 + f) * NF + i]), yout[i]);
            o1 = cadd(cscale(ca, xch[((2 * b + 1) * 32 + f) * NF + i]), yout[NF + i]);
          }
          outb[((2 * b) * NF + i) * CSTEP] = cscale(sgb, o0);
          outb[((2 * b + 1) * NF + i) * CSTEP] = cscale(sgb, o1);
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  }
  cp_async_wait<0>();  // no copy lands in shared memory after the CTA is gone
  if (lt == 0 && pending) tc_wait(bar_a, parity ^ 1u);  // one more bounded chance for a commit that timed out
  if (lt == 0 && s_fail[g] && err) atomicOr(err, 1u);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (tid < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tm) : "memory");
}

}  // namespace hrgpu
