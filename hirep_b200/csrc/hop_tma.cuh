// hop_tma.cuh -- the hopping kernel with its time halo staged by the TMA unit.
//
// A block is 128 consecutive checkerboard sites of the output parity, all in
// one time slab (the device layout puts t slowest, and the variant runs only
// where a slab holds a whole number of blocks).  Their t+1 and t-1 neighbours
// are then two contiguous runs of 128 sites of the input field in every
// component plane: thread 0 copies those 2 x 4NF runs into shared memory with
// untiled bulk copies (cp.async.bulk, completion counted in bytes on an
// mbarrier), while every thread computes the x, y and z directions from global
// memory; the t direction comes last, from shared memory.  Each wait on the
// mbarrier is bounded: a thread that gives up reads its t neighbours from
// global memory instead (the same values), and the block waits again, bounded,
// before it exits so that no copy lands in released shared memory; if that
// last wait gives up, the block sets bit 0 of the launch's error word, which
// the launcher turns into an error status.  No multicast: every copy reads
// this GPU's own memory into this block.  Measured slower than variant 0 in
// every case, the variant is not among the autotuner's candidates; it runs
// only when pinned with hrgpu_set_hop_variant(5).
#pragma once
#include "hop_async.cuh"

namespace hrgpu {

template <int NFT, typename R>
struct TmaLayout {
  typedef typename C2<R>::T V;
  static constexpr int NC = 4 * NFT;  // spinor components
  static constexpr unsigned RUN = HOP_THREADS * sizeof(V);  // bytes of one run
  static constexpr int SMEM = 2 * NC * (int)RUN;
};

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// global -> shared bulk copy of `bytes` (a multiple of 16, both addresses 16-byte
// aligned), completion reported to the mbarrier at shared address bar
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               :
               : "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

template <int NFT, bool REAL, typename R, int EP>
__global__ void __launch_bounds__(HOP_THREADS) k_hop_tma(HopArgs<R> a) {
  typedef TmaLayout<NFT, R> LAY;
  typedef typename LAY::V V;
  extern __shared__ __align__(16) unsigned char smem_halo[];
  __shared__ __align__(8) unsigned long long bar;
  V *sup = (V *)smem_halo, *sdn = sup + LAY::NC * HOP_THREADS;
  const unsigned bar_a = smem_u32(&bar);
  pdl_enter();
  if (a.stop && *a.stop) return;
  const Geo &g = a.g;
  const int S = g.Xh * g.Y * g.Z;                    // sites of one parity in a time slab
  const int cb0 = a.cb0 + blockIdx.x * HOP_THREADS;  // the block's first site
  const int t = cb0 / S;
  const int up0 = (t + 1 == g.T) ? cb0 - (g.T - 1) * S : cb0 + S;  // its t+1 neighbours
  const int dn0 = (t == 0) ? cb0 + (g.T - 1) * S : cb0 - S;        // its t-1 neighbours
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(2u * LAY::NC * LAY::RUN)
                 : "memory");
    const V *in = (const V *)a.in;
    for (int c = 0; c < LAY::NC; c++) {
      bulk_g2s(sup + c * HOP_THREADS, in + (long)c * g.ld + up0, LAY::RUN, bar_a);
      bulk_g2s(sdn + c * HOP_THREADS, in + (long)c * g.ld + dn0, LAY::RUN, bar_a);
    }
  }
  const double nrm = hop_site<NFT, REAL, R, EP, typename LinkE<REAL, R>::T, true>(
      a, cb0 + threadIdx.x, sup + threadIdx.x, sdn + threadIdx.x, bar_a);
  if (a.red) block_partial<R>(nrm, a.red);
  // at once when the copies were seen; bounded otherwise.  A block that gives
  // up here may leave copies in flight into shared memory the next resident
  // block reuses, so the launch is reported as failed (the launcher reads the
  // word back after every launch of this variant)
  if (!tma_wait(bar_a) && a.err) atomicOr(a.err, 1u);
}

}  // namespace hrgpu
