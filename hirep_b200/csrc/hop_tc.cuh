// hop_tc.cuh -- the batched hop with the link products on the 5th-generation
// tensor cores (tcgen05.mma, kind::tf32, FP32 accumulate in tensor memory).
//
// One output site at a time per CTA (a persistent grid walks the sites).  The
// site's hop over nb <= 32 fields is one small GEMM per site:
//   R^T (rows = output spin s x field f, columns = colour i, complex)
//     = sum over the 8 directions d of V_d^T U_d^T ,
// where V_d holds, for every (s, f), the spin-projected half spinor of the
// neighbour in direction d with the reconstruction phase of spin s already
// applied (v = beta_s (psi_k + alpha_k psi_p) -- phases commute with the
// colour product, so r_s = sum_d U_d v_{s,d}).  The 8 directions stack along
// K.  Complex arithmetic is made real: A (128 x K) holds [Re v | Im v] per
// direction, B (K x 16) the links as [[Re U^T, Im U^T], [-Im U^T, Re U^T]]
// blocks, and the 12 (NF = 6) real output columns come out as Re R, Im R.
//
// Operands: A lives in tensor memory, one lane per row (s, f): the thread of
// lane f in warp s computes its own row and writes it with tcgen05.st, so no
// shared-memory staging of the spinors is needed.  B (the links, 16 rows) is
// staged by the threads in shared memory in the canonical K-major layout
// without swizzle (core matrices of 8 rows x 16 bytes; LBO = 128 B between
// core matrices along K, SBO between 8-row groups).  FP32 accuracy from TF32
// inputs takes three products, A_hi B_hi + A_hi B_lo + A_lo B_hi, with
// x = hi + lo split by round-to-nearest TF32 conversions (the lo x lo term is
// below 2^-22).  The 8 directions go in two rounds of 4 (K = 48 per round at
// NF = 6), so a CTA needs 2 x 48 + 16 = 112 of its 128 tensor-memory columns
// and four CTAs fit an SM.  A round: rows and links written, one thread issues
// 18 MMAs and commits them to an mbarrier; every thread waits on it (bounded)
// before the next writes.  After the second round each thread reads its row of
// the accumulator (tcgen05.ld) and runs the epilogue of k_hopt (scale, the
// aux term, the clover blocks through a shared-memory exchange, gamma_5).
//
// Waits are bounded: a wait that gives up sets the launch's error word, the
// CTA stops taking sites, waits (bounded) for its last commit and frees its
// tensor memory.  Only this GPU's own memory is read; there is no multicast.
// FP32 only, complex NF = 6 (the two-index representations of SU(3) and
// SU(4)), nb <= 32.
#pragma once
#include "hop_tile.cuh"

namespace hrgpu {

constexpr int TC_THREADS = 128;
constexpr int TC_DIRS = 4;  // directions per MMA round

__device__ __forceinline__ uint32_t tc_smem(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: no swizzle, K-major, version 1 (sm_100)
__device__ __forceinline__ uint64_t tc_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor of kind::tf32: D in F32, A and B TF32, both K-major
__host__ __device__ constexpr uint32_t tc_idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ float tf32_rn(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity) {
  for (int it = 0; it < (1 << 22); it++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tc_st4(uint32_t taddr, float a, float b, float c, float d) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr), "r"(__float_as_uint(a)),
               "r"(__float_as_uint(b)), "r"(__float_as_uint(c)), "r"(__float_as_uint(d))
               : "memory");
}

// multiply a complex number by one of 1, i, -1, -i (q = 0..3)
__device__ __forceinline__ float2 cphase(float2 v, int q) {
  if (q == 0) return v;
  if (q == 1) return make_float2(-v.y, v.x);
  if (q == 2) return make_float2(-v.x, -v.y);
  return make_float2(v.y, -v.x);
}

// Spin structure of direction (mu, bw): the two half spinors are
// h_k = psi_k + alpha_k psi_{p_k} (k = 0, 1), and the lower output spins take
// r2 += beta2 c_{k2}, r3 += beta3 c_{k3} (the reconstruction of hopt_site).
// Phases as quarter turns: 0 = 1, 1 = i, 2 = -1, 3 = -i.
struct TcSpin {
  int p[2], alpha[2], k2, beta2, k3, beta3;
};
__device__ __forceinline__ TcSpin tc_spin(int mu, int bw) {
  TcSpin r;
  const int fw_p[4][2] = {{2, 3}, {3, 2}, {3, 2}, {2, 3}};
  const int fw_a[4][2] = {{0, 0}, {1, 1}, {0, 2}, {1, 3}};
  // (k2, beta2, k3, beta3) forward and backward
  const int fw_r[4][4] = {{0, 0, 1, 0}, {1, 3, 0, 3}, {1, 2, 0, 0}, {0, 3, 1, 1}};
  const int bw_r[4][4] = {{0, 2, 1, 2}, {1, 1, 0, 1}, {1, 0, 0, 2}, {0, 1, 1, 3}};
  r.p[0] = fw_p[mu][0];
  r.p[1] = fw_p[mu][1];
  r.alpha[0] = bw ? (fw_a[mu][0] + 2) & 3 : fw_a[mu][0];
  r.alpha[1] = bw ? (fw_a[mu][1] + 2) & 3 : fw_a[mu][1];
  const int(&q)[4] = bw ? bw_r[mu] : fw_r[mu];
  r.k2 = q[0];
  r.beta2 = q[1];
  r.k3 = q[2];
  r.beta3 = q[3];
  return r;
}

template <int NFT, int EP>
__global__ void __launch_bounds__(TC_THREADS) k_hopt_tc(TileArgs<float> a, unsigned *err) {
  constexpr int NF = NFT, NF2 = 2 * NFT, NS = 4 * NFT, NL = NFT * NFT;
  constexpr int KR = TC_DIRS * NF2;  // K of one round
  static_assert(KR % 8 == 0 && NF2 <= 16 && 2 * KR + 16 <= 128, "tensor-core hop: NF");
  constexpr int COL_AHI = 0, COL_ALO = KR, COL_D = 2 * KR, TCOLS = 128;
  constexpr uint32_t SBO = (KR / 4) * 128, LBO = 128;
  constexpr int CSTEP = TILE_S * TILE_F;
  constexpr long LSTEP = TILE_S;
  extern __shared__ __align__(128) unsigned char smem_tc[];
  float *sBhi = (float *)smem_tc, *sBlo = sBhi + 16 * KR;  // B (16 x KR) hi / lo, core-matrix layout
  float2 *xch = (float2 *)(sBlo + 16 * KR);                  // [4 spins][32 fields][NF] clover exchange
  __shared__ __align__(8) unsigned long long bar;
  __shared__ uint32_t taddr_s;
  __shared__ int s_fail;

  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  const int s = w, f = lane;  // this thread's row of A and of the accumulator: spin s of field f
  const Geo &g = a.g;
  const int outp = a.outp, inp = outp ^ 1;
  const long nblk = g.ld / TILE_S;
  const bool live = f < a.nb;
  const float2 *in = (const float2 *)a.in;
  const float2 *U = (const float2 *)a.U;

  for (int i = t; i < 2 * 16 * KR; i += TC_THREADS) sBhi[i] = 0.f;  // padding rows n >= 2NF stay zero
  if (t == 0) s_fail = 0;
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem(&taddr_s)),
                 "r"(TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tm = taddr_s;
  const uint32_t row = tm + ((uint32_t)(w * 32) << 16);  // this warp's 32 lanes
  const uint32_t bar_a = tc_smem(&bar);
  uint32_t parity = 0;
  bool pending = false;  // a commit not yet waited for
  const bool stopped = a.stop && *a.stop;

  for (int cb = blockIdx.x; !stopped && cb < g.VH; cb += gridDim.x) {
    int tt, xx, yy, zz;
    cb_to_coords(g, cb, outp, tt, xx, yy, zz);
#pragma unroll
    for (int round = 0; round < 2; round++) {
      // ---- B: the links of this round's four directions (threads 0 .. 4NF-1)
      if (t < TC_DIRS * NF) {
        const int dl = t / NF, i = t % NF, dd = round * TC_DIRS + dl, mu = dd >> 1, bw = dd & 1;
        const float2 *Ub;
        if (!bw) {
          Ub = U + (((long)outp * nblk + (cb >> 3)) * 4 + mu) * NL * LSTEP + (cb & 7);
        } else {
          int t2 = tt, x2 = xx, y2 = yy, z2 = zz;
          if (mu == 0) t2 = (tt == 0) ? g.T - 1 : tt - 1;
          if (mu == 1) x2 = (xx == 0) ? g.X - 1 : xx - 1;
          if (mu == 2) y2 = (yy == 0) ? g.Y - 1 : yy - 1;
          if (mu == 3) z2 = (zz == 0) ? g.Z - 1 : zz - 1;
          const int cn = coords_to_cb(g, t2, x2, y2, z2);
          Ub = U + (((long)inp * nblk + (cn >> 3)) * 4 + mu) * NL * LSTEP + (cn & 7);
        }
#pragma unroll
        for (int j = 0; j < NF; j++) {
          // row i of the direction's matrix: U(x,mu) forward, U(x-mu,mu)^+ backward
          float2 u = bw ? ld_c(Ub + (long)(j * NF + i) * LSTEP) : ld_c(Ub + (long)(i * NF + j) * LSTEP);
          if (bw) u.y = -u.y;
          // B[n][k], k = dl*2NF + c*NF + j: n = i (Re out), n = NF + i (Im out)
          const float vals[4] = {u.x, -u.y, u.y, u.x};  // (n=i,c=0) (n=i,c=1) (n=NF+i,c=0) (n=NF+i,c=1)
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const int n = (q < 2) ? i : NF + i, k = dl * NF2 + (q & 1) * NF + j;
            const int off = (n >> 3) * (SBO / 4) + (k >> 2) * (LBO / 4) + (n & 7) * 4 + (k & 3);
            const float hi = tf32_rn(vals[q]);
            sBhi[off] = hi;
            sBlo[off] = tf32_rn(vals[q] - hi);
          }
        }
      }
      // ---- A: this thread's row (s, f) for the round's four directions; tcgen05.st
      // is warp-collective, so the lanes of absent fields store zeros
      {
#pragma unroll
        for (int dl = 0; dl < TC_DIRS; dl++) {
          const int dd = round * TC_DIRS + dl, mu = dd >> 1, bw = dd & 1;
          int t2 = tt, x2 = xx, y2 = yy, z2 = zz;
          if (mu == 0) t2 = bw ? ((tt == 0) ? g.T - 1 : tt - 1) : ((tt + 1 == g.T) ? 0 : tt + 1);
          if (mu == 1) x2 = bw ? ((xx == 0) ? g.X - 1 : xx - 1) : ((xx + 1 == g.X) ? 0 : xx + 1);
          if (mu == 2) y2 = bw ? ((yy == 0) ? g.Y - 1 : yy - 1) : ((yy + 1 == g.Y) ? 0 : yy + 1);
          if (mu == 3) z2 = bw ? ((zz == 0) ? g.Z - 1 : zz - 1) : ((zz + 1 == g.Z) ? 0 : zz + 1);
          const int cn = coords_to_cb(g, t2, x2, y2, z2);
          const float2 *sp = in + (((long)(f >> 2) * nblk + (cn >> 3)) * NS) * CSTEP + (cn & 7) * TILE_F + (f & 3);
          const TcSpin S = tc_spin(mu, bw);
          const int k = (s == 0) ? 0 : (s == 1) ? 1 : (s == 2) ? S.k2 : S.k3;
          const int beta = (s < 2) ? 0 : (s == 2) ? S.beta2 : S.beta3;
          const int pk = S.p[k], ak = S.alpha[k];
          float re[NF], im[NF];
#pragma unroll
          for (int j = 0; j < NF; j++) {
            float2 v = make_float2(0.f, 0.f);
            if (live) {
              const float2 a0 = ld_c(sp + (k * NF + j) * CSTEP), a1 = ld_c(sp + (pk * NF + j) * CSTEP);
              v = cphase(cadd(a0, cphase(a1, ak)), beta);
            }
            re[j] = v.x;
            im[j] = v.y;
          }
          float hv[NF2], lv[NF2];
#pragma unroll
          for (int j = 0; j < NF; j++) {
            hv[j] = tf32_rn(re[j]);
            lv[j] = tf32_rn(re[j] - hv[j]);
            hv[NF + j] = tf32_rn(im[j]);
            lv[NF + j] = tf32_rn(im[j] - hv[NF + j]);
          }
#pragma unroll
          for (int c = 0; c < NF2; c += 4) {
            tc_st4(row + COL_AHI + dl * NF2 + c, hv[c], hv[c + 1], hv[c + 2], hv[c + 3]);
            tc_st4(row + COL_ALO + dl * NF2 + c, lv[c], lv[c + 1], lv[c + 2], lv[c + 3]);
          }
        }
      }
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      if (t == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        constexpr uint32_t ID = tc_idesc_tf32(128, 16);
        const uint32_t bh = tc_smem(sBhi), bl = tc_smem(sBlo);
#pragma unroll
        for (int ks = 0; ks < KR / 8; ks++) {
          const uint64_t dbh = tc_sdesc(bh + ks * 2 * LBO, LBO, SBO), dbl = tc_sdesc(bl + ks * 2 * LBO, LBO, SBO);
          const uint32_t ahi = tm + COL_AHI + ks * 8, alo = tm + COL_ALO + ks * 8;
          const uint32_t acc0 = (round > 0 || ks > 0) ? 1u : 0u;
          asm volatile(
              "{\n .reg .pred p;\n setp.ne.u32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n}\n" ::"r"(
                  tm + COL_D),
              "r"(ahi), "l"(dbh), "r"(ID), "r"(acc0)
              : "memory");
          asm volatile(
              "{\n .reg .pred p;\n setp.ne.u32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n}\n" ::"r"(
                  tm + COL_D),
              "r"(ahi), "l"(dbl), "r"(ID), "r"(1u)
              : "memory");
          asm volatile(
              "{\n .reg .pred p;\n setp.ne.u32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n}\n" ::"r"(
                  tm + COL_D),
              "r"(alo), "l"(dbh), "r"(ID), "r"(1u)
              : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_a)
                     : "memory");
      }
      pending = true;
      const bool ok = tc_wait(bar_a, parity);
      parity ^= 1u;
      if (!ok) atomicExch(&s_fail, 1);
      else pending = false;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      __syncthreads();  // every thread saw the MMAs complete (or the failure) before anyone rewrites A or B
      if (s_fail) break;
    }
    if (s_fail) break;
    // ---- the accumulator row: Re R_i in columns 0..NF-1, Im R_i in NF..2NF-1
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(row + COL_D)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    float2 R[NF];
#pragma unroll
    for (int i = 0; i < NF; i++) R[i] = make_float2(__uint_as_float(r[i]), __uint_as_float(r[NF + i]));
    // ---- epilogue (as hopt_site)
    const float ca = a.cacc;
    float2 *outb = (float2 *)a.out + (((long)(f >> 2) * nblk + (cb >> 3)) * NS) * CSTEP + (cb & 7) * TILE_F + (f & 3);
    const float2 *auxb =
        a.aux ? (const float2 *)a.aux + (((long)(f >> 2) * nblk + (cb >> 3)) * NS) * CSTEP + (cb & 7) * TILE_F + (f & 3)
              : nullptr;
    const float sg = (a.g5 && s >= 2) ? -1.f : 1.f;
    if (EP == EP_AXPY) {
      if (live) {
        const float cx = a.caux;
        const bool use_aux = auxb != nullptr && cx != 0.f;
#pragma unroll
        for (int i = 0; i < NF; i++) {
          float2 q = cscale(ca, R[i]);
          if (use_aux) rmac(q, cx, ld_c(auxb + (s * NF + i) * CSTEP));
          outb[(s * NF + i) * CSTEP] = cscale(sg, q);
        }
      }
    } else {
      // clover block b acts on spins (2b, 2b+1): gather them through shared memory
#pragma unroll
      for (int i = 0; i < NF; i++) xch[(s * 32 + f) * NF + i] = R[i];
      __syncthreads();
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
    __syncthreads();  // the accumulator and the exchange are rewritten by the next site
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (s_fail) {
    if (t == 0 && err) atomicOr(err, 1u);
    if (pending) tc_wait(bar_a, parity ^ 1u);  // give the last commit one more bounded chance
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (w == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(TCOLS) : "memory");
}

// shared memory of one CTA: B hi/lo and the clover exchange, padded so that at
// most four CTAs share an SM (their tensor memory: 4 x 128 columns)
template <int NFT>
constexpr size_t tc_smem_bytes() {
  return 50 * 1024;
}

}  // namespace hrgpu
