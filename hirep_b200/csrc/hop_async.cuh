// hop_async.cuh -- pipelined variant of the hopping kernel.
//
// One thread per site.  The neighbour spinor and the link of direction d+1 are
// copied global -> shared with cp.async while direction d is computed, so every
// thread keeps one direction's data (21 x 16 B for NF = 3) in flight without
// holding it in registers.  Shared memory is laid out [stage][element][thread]
// so the copies of consecutive threads land in consecutive words.  Each thread
// reads back only what it copied itself, so cp.async.wait_group is the only
// synchronisation.  Built for the small representations only (the per-thread
// staging grows with NF^2).
#pragma once
#include "hop.cuh"

namespace hrgpu {

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
// one element of BYTES (16: double complex, 8: float complex or double, 4: float)
template <int BYTES>
__device__ __forceinline__ void cp_async(void *smem, const void *gmem) {
  static_assert(BYTES == 16 || BYTES == 8 || BYTES == 4, "cp.async copies 4, 8 or 16 bytes");
  if (BYTES == 16) cp_async16(smem, gmem);
  else if (BYTES == 8) cp_async8(smem, gmem);
  else cp_async4(smem, gmem);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <int NA, bool REAL, typename R>
struct AsyncLayout {
  typedef typename C2<R>::T V;
  typedef typename LinkE<REAL, R>::T E;
  static constexpr int NS = 4 * NA;   // spinor elements per direction
  static constexpr int NL = NA * NA;  // link elements per direction
  static constexpr int STAGE_BYTES = HOP_THREADS * (NS * (int)sizeof(V) + NL * (int)sizeof(E));
  static constexpr int SMEM = 2 * STAGE_BYTES;
};

template <int N, bool RL>
struct AsyncOK {
  static constexpr bool v = RL ? (N == 3) : (N <= 4);
};

template <int NFT, bool REAL, typename R, int EP>
__global__ void __launch_bounds__(HOP_THREADS) k_hop_async(HopArgs<R> a) {
  typedef typename C2<R>::T V;
  typedef typename LinkE<REAL, R>::T E;
  typedef AsyncLayout<NFT, REAL, R> LAY;
  constexpr int NA = NFT;
  const int nf = NFT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Geo g = a.g;
  pdl_enter();
  if (a.stop && *a.stop) return;
  const int tid = threadIdx.x;
  const int cs = a.cb0 + blockIdx.x * blockDim.x + tid;
  const bool active = cs < a.cb1;
  const int cb = active ? cs : a.cb1 - 1;
  const int outp = a.outp, inp = outp ^ 1;
  int t, x, y, z;
  cb_to_coords(g, cb, outp, t, x, y, z);
  const long ld = g.ld, lplane = 2L * g.ld;
  const V *in = (const V *)a.in;
  const E *U = (const E *)a.U;
  const long nf2 = (long)nf * nf;
  const long so = (long)outp * ld + cb;
  auto sp_slot = [&](int st, int e) -> V * {
    return (V *)(smem_raw + (size_t)st * LAY::STAGE_BYTES) + (size_t)e * HOP_THREADS + tid;
  };
  auto ln_slot = [&](int st, int e) -> E * {
    return (E *)(smem_raw + (size_t)st * LAY::STAGE_BYTES + (size_t)HOP_THREADS * LAY::NS * sizeof(V)) +
           (size_t)e * HOP_THREADS + tid;
  };
  // direction d = 2 mu + (backward): neighbour checkerboard index and link site
  auto issue = [&](int d) {
    const int mu = d >> 1, bw = d & 1, s = bw ? -1 : 1;
    int tt = t, xx = x, yy = y, zz = z;
    if (mu == 0) tt = (t + s + g.T) % g.T;
    if (mu == 1) xx = (x + s + g.X) % g.X;
    if (mu == 2) yy = (y + s + g.Y) % g.Y;
    if (mu == 3) zz = (z + s + g.Z) % g.Z;
    const int cn = coords_to_cb(g, tt, xx, yy, zz);
    const long sl = bw ? (long)inp * ld + cn : so;
    const int st = d & 1;
#pragma unroll
    for (int e = 0; e < LAY::NS; e++) cp_async<sizeof(V)>(sp_slot(st, e), in + (long)e * ld + cn);
    const E *Umu = U + (long)mu * nf2 * lplane + sl;
#pragma unroll
    for (int e = 0; e < LAY::NL; e++) cp_async<sizeof(E)>(ln_slot(st, e), Umu + (long)e * lplane);
    cp_async_commit();
  };
  V r0[NA], r1[NA], r2[NA], r3[NA];
#pragma unroll
  for (int i = 0; i < NA; i++) r0[i] = r1[i] = r2[i] = r3[i] = cmk<V>(0.0, 0.0);
  issue(0);
#pragma unroll
  for (int d = 0; d < 8; d++) {
    if (d + 1 < 8) {
      issue(d + 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    const int st = d & 1, mu = d >> 1, bw = d & 1;
    V h0[NA], h1[NA], c0[NA], c1[NA];
#pragma unroll
    for (int i = 0; i < NA; i++) {
      V s0 = *sp_slot(st, 0 * nf + i), s1 = *sp_slot(st, 1 * nf + i);
      V s2 = *sp_slot(st, 2 * nf + i), s3 = *sp_slot(st, 3 * nf + i);
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
#pragma unroll
    for (int i = 0; i < NA; i++) {
      V q0 = cmk<V>(0.0, 0.0), q1 = cmk<V>(0.0, 0.0);
#pragma unroll
      for (int j = 0; j < NA; j++) {
        if (!bw) {
          E u = *ln_slot(st, i * nf + j);
          if constexpr (REAL) { rmac(q0, u, h0[j]); rmac(q1, u, h1[j]); }
          else { cmac(q0, u, h0[j]); cmac(q1, u, h1[j]); }
        } else {
          E u = *ln_slot(st, j * nf + i);
          if constexpr (REAL) { rmac(q0, u, h0[j]); rmac(q1, u, h1[j]); }
          else { cmacc(q0, u, h0[j]); cmacc(q1, u, h1[j]); }
        }
      }
      c0[i] = q0;
      c1[i] = q1;
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
  }
  V *out = (V *)a.out + cb;
  const R ca = a.cacc;
  if (EP == EP_AXPY) {
    const V *aux = (const V *)a.aux + cb;
    const R cx = a.caux;
#pragma unroll
    for (int i = 0; i < NA; i++) {
      V q0 = cscale(ca, r0[i]), q1 = cscale(ca, r1[i]), q2 = cscale(ca, r2[i]), q3 = cscale(ca, r3[i]);
      if (aux != nullptr && cx != (R)0) {
        rmac(q0, cx, ld_c(aux + (long)(0 * nf + i) * ld));
        rmac(q1, cx, ld_c(aux + (long)(1 * nf + i) * ld));
        rmac(q2, cx, ld_c(aux + (long)(2 * nf + i) * ld));
        rmac(q3, cx, ld_c(aux + (long)(3 * nf + i) * ld));
      }
      r0[i] = q0; r1[i] = q1; r2[i] = q2; r3[i] = q3;
    }
  } else {
    clover_epilogue<NA, EP>(r0, r1, a, ca, cb, 0, cb, ld);
    clover_epilogue<NA, EP>(r2, r3, a, ca, cb, 1, cb, ld);
  }
  const R sg = a.g5 ? (R)-1 : (R)1;
  double nrm = 0.0;
#pragma unroll
  for (int i = 0; i < NA; i++) {
    V o2 = cscale(sg, r2[i]), o3 = cscale(sg, r3[i]);
    if (active) {
      out[(long)(0 * nf + i) * ld] = r0[i];
      out[(long)(1 * nf + i) * ld] = r1[i];
      out[(long)(2 * nf + i) * ld] = o2;
      out[(long)(3 * nf + i) * ld] = o3;
    }
    nrm += (double)r0[i].x * r0[i].x + (double)r0[i].y * r0[i].y + (double)r1[i].x * r1[i].x +
           (double)r1[i].y * r1[i].y + (double)o2.x * o2.x + (double)o2.y * o2.y + (double)o3.x * o3.x +
           (double)o3.y * o3.y;
  }
  if (a.red) {
    if (!active) nrm = 0.0;
    block_partial<R>(nrm, a.red);
  }
}

}  // namespace hrgpu
