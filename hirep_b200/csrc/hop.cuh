// hop.cuh -- the even-odd Wilson hopping kernel (HiRep's Dphi_, LibHR/Update/Dphi.c:193-374)
// with fused epilogues for the preconditioned and clover operators.
//
// One thread per output site of one parity.  Per direction the thread loads the
// neighbour spinor from structure-of-arrays planes (consecutive threads read
// consecutive 16-byte complex numbers), spin-projects it to two NF-vectors,
// multiplies by U or U^+ streamed element by element from the link planes, and
// accumulates the four spin components of the result in registers.  Neighbours
// are computed from the coordinates (no index tables are read).
//
// Epilogues (all written with the -1/2 of Dphi_ folded into `cacc`):
//   EP_AXPY      out = cacc*acc + caux*aux          (Dphi, eopre second hop)
//   EP_CLOV_INV  out = Hinv (cacc*acc)              (Cphi_eopre first hop: D_oo^-1 D_oe)
//   EP_CLOV      out = cacc*acc + Hdiag*aux         (Cphi, Cphi_eopre second hop)
// then optionally gamma_5, and optionally a per-block partial of |out|^2.
#pragma once
#include <cuda_bf16.h>

#include <type_traits>

#include "hrgpu_internal.cuh"

namespace hrgpu {

enum { EP_AXPY = 0, EP_CLOV_INV = 1, EP_CLOV = 2 };
constexpr int HOP_THREADS = 128;

template <typename R>
struct HopArgs {
  const void *in;    // input parity field, planes [4NF][ld]
  void *out;         // output parity field
  const void *U;     // links [4][NF*NF][2ld]
  const void *aux;   // field at the output sites (EP_AXPY, EP_CLOV)
  const R *cdg;      // packed clover diag [2][2NF][2ld] (Hdiag or Hinv)
  const typename C2<R>::T *cod;  // packed clover off-diagonal [2][NF(2NF-1)][2ld]
  double *red;       // block partials of |out|^2 (or nullptr)
  const int *stop;   // inverter state: when non-null and *stop != 0 the launch does nothing
  unsigned *err;     // device error word (variant 5: bit 0 = a bounded wait gave up), or nullptr
  R cacc, caux;
  int outp;
  int g5;
  int nf;
  int cb0, cb1;      // output sites cb0 <= cb < cb1 of parity outp
  int recon;         // Lattice::recon12 at launch: 2 (4) puts the antiperiodic sign on rebuilt rows (links)
  const void *Ug;    // fundamental links [4][NG*NG][2ld], element type of R (two-index links built on the fly, recon 3, 4)
  Geo g;
};

template <bool REAL, typename R>
struct LinkE {
  typedef typename C2<R>::T T;
};
template <typename R>
struct LinkE<true, R> {
  typedef R T;
};

template <typename V> __device__ __forceinline__ V ld_c(const V *p) { return __ldg(p); }
__device__ __forceinline__ double ld_c(const double *p) { return __ldg(p); }
__device__ __forceinline__ float ld_c(const float *p) { return __ldg(p); }

// read-only loads that do not allocate in L1: a single-field hop reads each
// link once, so its links pass L1 by and leave it to the neighbour spinors
__device__ __forceinline__ double2 ld_u(const double2 *p) {
  double2 v;
  asm("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}
__device__ __forceinline__ float2 ld_u(const float2 *p) {
  float2 v;
  asm("ld.global.nc.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
  return v;
}
__device__ __forceinline__ double ld_u(const double *p) {
  double v;
  asm("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ float ld_u(const float *p) {
  float v;
  asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}

// read-once data (the clover blocks of a single-field hop): no L1 allocation
// and first out of L2, so that the links and spinors the next hop reads stay
__device__ __forceinline__ unsigned long long l2_evict_first() {
  unsigned long long pol;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ double2 ld_ef(const double2 *p, unsigned long long pol) {
  double2 v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float2 ld_ef(const float2 *p, unsigned long long pol) {
  float2 v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_ef(const double *p, unsigned long long pol) {
  double v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float ld_ef(const float *p, unsigned long long pol) {
  float v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
// the same policy in L2 with the line kept in L1 (data that other warps of
// the SM read again soon: the batched kernel's links and clover blocks)
__device__ __forceinline__ double2 ld_ef1(const double2 *p, unsigned long long pol) {
  double2 v;
  asm("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float2 ld_ef1(const float2 *p, unsigned long long pol) {
  float2 v;
  asm("ld.global.nc.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_ef1(const double *p, unsigned long long pol) {
  double v;
  asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float ld_ef1(const float *p, unsigned long long pol) {
  float v;
  asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
// load policy LP: 0 read-only (ld_c), 1 ld_ef, 2 ld_ef1
template <int LP, typename T>
__device__ __forceinline__ T ld_p(const T *p, unsigned long long pol) {
  if constexpr (LP == 1) return ld_ef(p, pol);
  else if constexpr (LP == 2) return ld_ef1(p, pol);
  else return ld_c(p);
}

// chi = U h (DAG=false) or U^+ h (DAG=true); U element (i,j) at U[(i*nf+j)*plane + site]
template <int NA> struct Unroll { static constexpr int v = NA <= 12 ? NA : 1; };

// LP: load policy of the link elements (ld_p)
template <int NA, bool DAG, int LP = 0, typename V>
__device__ __forceinline__ void link_mul(V *chi, const V *h, const V *U, long plane, long site, int nf) {
  const unsigned long long pol = LP ? l2_evict_first() : 0ull;
#pragma unroll
  for (int i = 0; i < NA; i++) {
    if (i >= nf) break;
    V a = cmk<V>(0.0, 0.0);
#pragma unroll (Unroll<NA>::v)
    for (int j = 0; j < NA; j++) {
      if (j >= nf) break;
      if (!DAG) {
        V u = ld_p<LP>(U + (long)(i * nf + j) * plane + site, pol);
        cmac(a, u, h[j]);
      } else {
        V u = ld_p<LP>(U + (long)(j * nf + i) * plane + site, pol);
        cmacc(a, u, h[j]);
      }
    }
    chi[i] = a;
  }
}

template <int NA, bool DAG, int LP = 0, typename V, typename R>
__device__ __forceinline__ void link_mul(V *chi, const V *h, const R *U, long plane, long site, int nf) {
  const unsigned long long pol = LP ? l2_evict_first() : 0ull;
#pragma unroll
  for (int i = 0; i < NA; i++) {
    if (i >= nf) break;
    V a = cmk<V>(0.0, 0.0);
#pragma unroll (Unroll<NA>::v)
    for (int j = 0; j < NA; j++) {
      if (j >= nf) break;
      R u = ld_p<LP>(U + (long)(DAG ? j * nf + i : i * nf + j) * plane + site, pol);
      rmac(a, u, h[j]);
    }
    chi[i] = a;
  }
}

// links stored in BF16 (the FP32 operator's optional storage): the products are FP32
template <int NA, bool DAG>
__device__ __forceinline__ void link_mul(float2 *chi, const float2 *h, const __nv_bfloat162 *U, long plane, long site,
                                         int nf) {
#pragma unroll
  for (int i = 0; i < NA; i++) {
    if (i >= nf) break;
    float2 a = make_float2(0.f, 0.f);
#pragma unroll (Unroll<NA>::v)
    for (int j = 0; j < NA; j++) {
      if (j >= nf) break;
      if (!DAG) {
        float2 u = __bfloat1622float2(__ldg(U + (long)(i * nf + j) * plane + site));
        cmac(a, u, h[j]);
      } else {
        float2 u = __bfloat1622float2(__ldg(U + (long)(j * nf + i) * plane + site));
        cmacc(a, u, h[j]);
      }
    }
    chi[i] = a;
  }
}

template <int NA, bool DAG>
__device__ __forceinline__ void link_mul(float2 *chi, const float2 *h, const __nv_bfloat16 *U, long plane, long site,
                                         int nf) {
#pragma unroll
  for (int i = 0; i < NA; i++) {
    if (i >= nf) break;
    float2 a = make_float2(0.f, 0.f);
#pragma unroll (Unroll<NA>::v)
    for (int j = 0; j < NA; j++) {
      if (j >= nf) break;
      float u = __bfloat162float(DAG ? __ldg(U + (long)(j * nf + i) * plane + site) : __ldg(U + (long)(i * nf + j) * plane + site));
      rmac(a, u, h[j]);
    }
    chi[i] = a;
  }
}

// c0 = W h0 and c1 = W h1 with W = U (DAG=false) or U^+ (DAG=true) of one link.
// R12 (complex NF = 3 links stored in the operator's own precision, in the
// kernels instantiated for reconstruction): only rows 0 and 1 are loaded and
// row 2 is rebuilt as sg conj(r0 x r1) (su3_row2), a third less link traffic;
// otherwise the full link is read.  The link loads do not allocate in L1
// (ld_u): a single-field hop reads each link once.
// The real form (R12R: SU(2) adjoint links, SO(3)) rebuilds row 2 as sg (r0 x r1).
template <int NA, bool DAG, bool R12, bool R12R = false, typename V, typename E, typename R>
__device__ __forceinline__ void link_mul2(V *c0, V *c1, const V *h0, const V *h1, const E *U, long plane, long site,
                                          int nf, R sg) {
  if constexpr (R12R) {
    R u[9];
#pragma unroll
    for (int e = 0; e < 6; e++) u[e] = ld_u(U + (long)e * plane + site);
    so3_row2(u, sg);
#pragma unroll
    for (int i = 0; i < 3; i++) {
      V a0 = cmk<V>(0.0, 0.0), a1 = cmk<V>(0.0, 0.0);
#pragma unroll
      for (int j = 0; j < 3; j++) {
        const R w = DAG ? u[3 * j + i] : u[3 * i + j];
        rmac(a0, w, h0[j]);
        rmac(a1, w, h1[j]);
      }
      c0[i] = a0;
      c1[i] = a1;
    }
    return;
  }
  if constexpr (R12) {
    {
      V u[9];
#pragma unroll
      for (int e = 0; e < 6; e++) u[e] = ld_u(U + (long)e * plane + site);
      su3_row2(u, sg);
#pragma unroll
      for (int i = 0; i < 3; i++) {
        V a0 = cmk<V>(0.0, 0.0), a1 = cmk<V>(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < 3; j++) {
          if (!DAG) {
            cmac(a0, u[3 * i + j], h0[j]);
            cmac(a1, u[3 * i + j], h1[j]);
          } else {
            cmacc(a0, u[3 * j + i], h0[j]);
            cmacc(a1, u[3 * j + i], h1[j]);
          }
        }
        c0[i] = a0;
        c1[i] = a1;
      }
      return;
    }
  }
  if constexpr (std::is_same<E, __nv_bfloat162>::value || std::is_same<E, __nv_bfloat16>::value) {
    link_mul<NA, DAG>(c0, h0, U, plane, site, nf);  // BF16 storage
    link_mul<NA, DAG>(c1, h1, U, plane, site, nf);
  } else {
    // the full link, each element loaded once for both half spinors
#pragma unroll
    for (int i = 0; i < NA; i++) {
      if (i >= nf) break;
      V a0 = cmk<V>(0.0, 0.0), a1 = cmk<V>(0.0, 0.0);
#pragma unroll (Unroll<NA>::v)
      for (int j = 0; j < NA; j++) {
        if (j >= nf) break;
        const E u = ld_u(U + (long)(DAG ? j * nf + i : i * nf + j) * plane + site);
        if constexpr (sizeof(E) == sizeof(V)) {
          if (!DAG) {
            cmac(a0, u, h0[j]);
            cmac(a1, u, h1[j]);
          } else {
            cmacc(a0, u, h0[j]);
            cmacc(a1, u, h1[j]);
          }
        } else {
          rmac(a0, u, h0[j]);
          rmac(a1, u, h1[j]);
        }
      }
      c0[i] = a0;
      c1[i] = a1;
    }
  }
}

// BF16 storage type of a link element
template <bool REAL>
struct LinkBF16 {
  typedef __nv_bfloat162 T;
};
template <>
struct LinkBF16<true> {
  typedef __nv_bfloat16 T;
};

// y = H x for one packed Hermitian 2NF x 2NF block (diag real, strict lower complex)
// LP: load policy of the blocks (ld_p; 1 for a single-field hop, which reads them once)
template <int NA, int LP = 0, typename V, typename R>
__device__ __forceinline__ void herm_apply(V *y, const V *x, const R *dg, const V *od, long plane, long site, int nf) {
  const int n = 2 * nf;
  const unsigned long long pol = LP ? l2_evict_first() : 0ull;
#pragma unroll
  for (int i = 0; i < 2 * NA; i++) {
    if (i >= n) break;
    R d = ld_p<LP>(dg + (long)i * plane + site, pol);
    y[i] = cscale(d, x[i]);
  }
#pragma unroll (Unroll<2 * NA>::v)
  for (int i = 1; i < 2 * NA; i++) {
    if (i >= n) break;
#pragma unroll (Unroll<2 * NA>::v)
    for (int j = 0; j < 2 * NA; j++) {
      if (j >= i) break;
      V l = ld_p<LP>(od + (long)(i * (i - 1) / 2 + j) * plane + site, pol);
      cmac(y[i], l, x[j]);   // y_i += L_ij x_j
      cmacc(y[j], l, x[i]);  // y_j += conj(L_ij) x_i
    }
  }
}

template <typename R>
__device__ __forceinline__ void block_partial(double v, double *red) {
  __shared__ double sh[HOP_THREADS / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) s += sh[k];
    red[blockIdx.x] = s;
  }
}

// clover epilogue on one chiral block: (ra, rb) are the spin pair of block b
// sofs / cs: offset of this site's first element and component stride in the
// spinor fields (cb and ld for a single field)
template <int NA, int EP, typename V, typename R>
__device__ __forceinline__ void clover_epilogue(V (&ra)[NA], V (&rb)[NA], const HopArgs<R> &a, R ca, int cb, int b,
                                                long sofs, long cs) {
  const Geo &g = a.g;
  const int nf = NA;
  const long lp = 2L * g.ld, site = (long)a.outp * g.ld + cb;
  const int n2 = 2 * nf, no = nf * (2 * nf - 1);
  V xin[2 * NA], yout[2 * NA];
  if (EP == EP_CLOV_INV) {
#pragma unroll
    for (int i = 0; i < NA; i++) {
      xin[i] = cscale(ca, ra[i]);
      xin[nf + i] = cscale(ca, rb[i]);
    }
  } else {
    const V *aux = (const V *)a.aux + sofs;
#pragma unroll
    for (int i = 0; i < NA; i++) {
      xin[i] = ld_c(aux + (long)((2 * b) * nf + i) * cs);
      xin[nf + i] = ld_c(aux + (long)((2 * b + 1) * nf + i) * cs);
    }
  }
  herm_apply<NA, 1>(yout, xin, a.cdg + (long)b * n2 * lp, a.cod + (long)b * no * lp, lp, site, nf);
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

// the t+-1 neighbours staged in shared memory by k_hop_tma: wait (bounded) for
// the bulk copies on the block's mbarrier; false if they did not land in time
__device__ __forceinline__ bool tma_wait(unsigned bar) {
  for (int it = 0; it < (1 << 22); it++) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(0u)
        : "memory");
    if (done) return true;
  }
  return false;
}

template <typename V>
__device__ __forceinline__ V ld_sel(const V *p, bool smem) {
  return smem ? *p : ld_c(p);
}

// The two-index representations with NF = 6 built on the fly from the
// fundamental link u: FR = 1 the symmetric one of SU(3), FR = 2 the
// antisymmetric one of SU(4).  Element (C, A) of the represented link is the
// one k_represent writes (the same products and factors, and the boundary
// sign sg): the columns A and the rows C run over the index pairs (a >= b)
// and (e <= c) in k_represent's order.  Reading NG^2 instead of 36 complex
// numbers per link (9 or 16) trades 2.3-4x fewer link bytes for two complex
// products per element.
template <int FR>
struct TwoIdx {
  static constexpr int NG = FR == 1 ? 3 : 4;
  // basis element k = 0..5 is the index pair (lo(k), hi(k)): rows C = (e, c) =
  // (lo, hi), columns A = (a, b) = (hi, lo); symmetric (0,0) (0,1) (1,1) (0,2)
  // (1,2) (2,2), antisymmetric (0,1) (0,2) (1,2) (0,3) (1,3) (2,3)
  __host__ __device__ static constexpr int lo(int k) { return (k == 2 || k == 4) ? 1 : (k == 5 ? 2 : 0); }
  __host__ __device__ static constexpr int hi(int k) { return (k == 0 ? 0 : (k <= 2 ? 1 : 2)) + (FR == 2 ? 1 : 0); }
};

template <int FR, typename V>
__device__ __forceinline__ V two_idx_elem(const V (&u)[TwoIdx<FR>::NG * TwoIdx<FR>::NG], int C, int A,
                                          decltype(V::x) sg) {
  typedef decltype(V::x) R;
  constexpr int N = TwoIdx<FR>::NG;
  const int e = TwoIdx<FR>::lo(C), c = TwoIdx<FR>::hi(C), a = TwoIdx<FR>::hi(A), b = TwoIdx<FR>::lo(A);
  auto mk = [](R x, R y) {
    V r;
    r.x = x;
    r.y = y;
    return r;
  };
  auto cm = [&](V p, V q) { return mk(p.x * q.x - p.y * q.y, p.x * q.y + p.y * q.x); };
  if (FR == 1) {
    // the factors sqrt(2) and 1/sqrt(2) as constants (k_represent divides by
    // sqrt(2): the elements may differ from the stored ones in the last bit)
    constexpr R st = (R)1.4142135623730951, ist = (R)0.7071067811865476;
    const bool diag = a == b;
    const V mf = diag ? cm(u[e * N + a], u[c * N + a]) : cadd(cm(u[e * N + a], u[c * N + b]), cm(u[e * N + b], u[c * N + a]));
    V w;
    if (e < c) w = diag ? mk(mf.x * st, mf.y * st) : mf;
    else w = diag ? mf : mk(mf.x * ist, mf.y * ist);
    return mk(sg * w.x, sg * w.y);
  } else {
    const V mf = csub(cm(u[e * N + a], u[c * N + b]), cm(u[e * N + b], u[c * N + a]));
    return mk(-sg * mf.x, -sg * mf.y);
  }
}

// c0 = U^R h0, c1 = U^R h1 (DAG: U^R+) with U^R built from the fundamental link
// at `site` of the planes Ug (plane stride `plane`)
template <int FR, bool DAG, typename V>
__device__ __forceinline__ void two_idx_mul2(V *c0, V *c1, const V *h0, const V *h1, const V *Ug, long plane, long site,
                                             decltype(V::x) sg) {
  constexpr int N = TwoIdx<FR>::NG;
  V u[N * N];
#pragma unroll
  for (int k = 0; k < N * N; k++) u[k] = ld_u(Ug + (long)k * plane + site);
#pragma unroll
  for (int i = 0; i < 6; i++) {
    V a0 = cmk<V>(0.0, 0.0), a1 = cmk<V>(0.0, 0.0);
#pragma unroll
    for (int j = 0; j < 6; j++) {
      if (!DAG) {
        const V v = two_idx_elem<FR>(u, i, j, sg);
        cmac(a0, v, h0[j]);
        cmac(a1, v, h1[j]);
      } else {
        const V v = two_idx_elem<FR>(u, j, i, sg);
        cmacc(a0, v, h0[j]);
        cmacc(a1, v, h1[j]);
      }
    }
    c0[i] = a0;
    c1[i] = a1;
  }
}

// one output site (checkerboard index cb < VH) of the hop; returns |out|^2 when a.red is set
// LE: the storage type of a link element (BF16 for the FP32 operator's optional link copy)
// TSM: the t+1 / t-1 neighbours come from shared memory (tsu, tsd: this thread's
// element of component 0, components HOP_THREADS apart) once the bulk copies on
// the mbarrier at shared address bar have landed; the t direction is then
// visited last, after x, y, z, to give the copies time
template <int NFT, bool REAL, typename R, int EP, typename LE = typename LinkE<REAL, R>::T, bool TSM = false,
          bool RC = false, int FR = 0>
__device__ __forceinline__ double hop_site(const HopArgs<R> &a, const int cb, const typename C2<R>::T *tsu = nullptr,
                                           const typename C2<R>::T *tsd = nullptr, unsigned bar = 0) {
  typedef typename C2<R>::T V;
  typedef LE E;
  constexpr int NA = NFT;
  constexpr bool R12 = RC && NFT == 3 && !REAL && std::is_same<LE, V>::value;
  constexpr bool R12R = RC && NFT == 3 && REAL && std::is_same<LE, R>::value;
  const int nf = NFT;
  const Geo g = a.g;
  double nrm = 0.0;
  {
    const int outp = a.outp, inp = outp ^ 1;
    int t, x, y, z;
    cb_to_coords(g, cb, outp, t, x, y, z);
    const long ld = g.ld, lplane = 2L * g.ld;
    const V *in = (const V *)a.in;
    const E *U = (const E *)a.U;
    const long nf2 = (long)nf * nf;
    V r0[NA], r1[NA], r2[NA], r3[NA], h0[NA], h1[NA], c0[NA], c1[NA];
#pragma unroll
    for (int i = 0; i < NA; i++) r0[i] = r1[i] = r2[i] = r3[i] = cmk<V>(0.0, 0.0);
    const long so = (long)outp * g.ld + cb;  // this site in the link planes
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int mu = TSM ? ((k + 1) & 3) : k;
      const bool use_sm = TSM && mu == 0 && tma_wait(bar);
      int tp = t, xp = x, yp = y, zp = z, tm = t, xm = x, ym = y, zm = z;
      if (mu == 0) { tp = (t + 1 == g.T) ? 0 : t + 1; tm = (t == 0) ? g.T - 1 : t - 1; }
      if (mu == 1) { xp = (x + 1 == g.X) ? 0 : x + 1; xm = (x == 0) ? g.X - 1 : x - 1; }
      if (mu == 2) { yp = (y + 1 == g.Y) ? 0 : y + 1; ym = (y == 0) ? g.Y - 1 : y - 1; }
      if (mu == 3) { zp = (z + 1 == g.Z) ? 0 : z + 1; zm = (z == 0) ? g.Z - 1 : z - 1; }
      const int cup = coords_to_cb(g, tp, xp, yp, zp);
      const int cdn = coords_to_cb(g, tm, xm, ym, zm);
      const E *Umu = U + (long)mu * nf2 * lplane;
      // ---- forward: (1 - gamma_mu) U(x,mu) psi(x+mu)
      {
        const V *s = use_sm ? tsu : in + cup;
        const long st = use_sm ? (long)HOP_THREADS : ld;
#pragma unroll
        for (int i = 0; i < NA; i++) {
          if (i >= nf) break;
          V s0 = ld_sel(s + (long)(0 * nf + i) * st, use_sm), s1 = ld_sel(s + (long)(1 * nf + i) * st, use_sm);
          V s2 = ld_sel(s + (long)(2 * nf + i) * st, use_sm), s3 = ld_sel(s + (long)(3 * nf + i) * st, use_sm);
          if (mu == 0) { h0[i] = cadd(s0, s2); h1[i] = cadd(s1, s3); }
          if (mu == 1) { h0[i] = caddi(s0, s3); h1[i] = caddi(s1, s2); }
          if (mu == 2) { h0[i] = cadd(s0, s3); h1[i] = csub(s1, s2); }
          if (mu == 3) { h0[i] = caddi(s0, s2); h1[i] = csubi(s1, s3); }
        }
        if constexpr (FR != 0) {
          const R sgr = (a.recon == 4 && mu == 0 && t == 0) ? (R)-1 : (R)1;
          two_idx_mul2<FR, false>(c0, c1, h0, h1,
                                  (const V *)a.Ug + (long)mu * TwoIdx<FR>::NG * TwoIdx<FR>::NG * lplane, lplane, so,
                                  sgr);
        } else {
          const R sgf = (a.recon == 2 && mu == 0 && t == 0) ? (R)-1 : (R)1;
          link_mul2<NA, false, R12, R12R>(c0, c1, h0, h1, Umu, lplane, so, nf, sgf);
        }
#pragma unroll
        for (int i = 0; i < NA; i++) {
          if (i >= nf) break;
          r0[i] = cadd(r0[i], c0[i]);
          r1[i] = cadd(r1[i], c1[i]);
          if (mu == 0) { r2[i] = cadd(r2[i], c0[i]); r3[i] = cadd(r3[i], c1[i]); }
          if (mu == 1) { r3[i] = csubi(r3[i], c0[i]); r2[i] = csubi(r2[i], c1[i]); }
          if (mu == 2) { r3[i] = cadd(r3[i], c0[i]); r2[i] = csub(r2[i], c1[i]); }
          if (mu == 3) { r2[i] = csubi(r2[i], c0[i]); r3[i] = caddi(r3[i], c1[i]); }
        }
      }
      // ---- backward: (1 + gamma_mu) U(x-mu,mu)^+ psi(x-mu)
      {
        const V *s = use_sm ? tsd : in + cdn;
        const long st = use_sm ? (long)HOP_THREADS : ld;
#pragma unroll
        for (int i = 0; i < NA; i++) {
          if (i >= nf) break;
          V s0 = ld_sel(s + (long)(0 * nf + i) * st, use_sm), s1 = ld_sel(s + (long)(1 * nf + i) * st, use_sm);
          V s2 = ld_sel(s + (long)(2 * nf + i) * st, use_sm), s3 = ld_sel(s + (long)(3 * nf + i) * st, use_sm);
          if (mu == 0) { h0[i] = csub(s0, s2); h1[i] = csub(s1, s3); }
          if (mu == 1) { h0[i] = csubi(s0, s3); h1[i] = csubi(s1, s2); }
          if (mu == 2) { h0[i] = csub(s0, s3); h1[i] = cadd(s1, s2); }
          if (mu == 3) { h0[i] = csubi(s0, s2); h1[i] = caddi(s1, s3); }
        }
        const long sn = (long)inp * g.ld + cdn;
        if constexpr (FR != 0) {
          const R sgr = (a.recon == 4 && mu == 0 && tm == 0) ? (R)-1 : (R)1;
          two_idx_mul2<FR, true>(c0, c1, h0, h1,
                                 (const V *)a.Ug + (long)mu * TwoIdx<FR>::NG * TwoIdx<FR>::NG * lplane, lplane, sn,
                                 sgr);
        } else {
          const R sgb = (a.recon == 2 && mu == 0 && tm == 0) ? (R)-1 : (R)1;
          link_mul2<NA, true, R12, R12R>(c0, c1, h0, h1, Umu, lplane, sn, nf, sgb);
        }
#pragma unroll
        for (int i = 0; i < NA; i++) {
          if (i >= nf) break;
          r0[i] = cadd(r0[i], c0[i]);
          r1[i] = cadd(r1[i], c1[i]);
          if (mu == 0) { r2[i] = csub(r2[i], c0[i]); r3[i] = csub(r3[i], c1[i]); }
          if (mu == 1) { r3[i] = caddi(r3[i], c0[i]); r2[i] = caddi(r2[i], c1[i]); }
          if (mu == 2) { r3[i] = csub(r3[i], c0[i]); r2[i] = cadd(r2[i], c1[i]); }
          if (mu == 3) { r2[i] = caddi(r2[i], c0[i]); r3[i] = csubi(r3[i], c1[i]); }
        }
      }
    }
    // ---- epilogue
    V *out = (V *)a.out + cb;
    const R ca = a.cacc;
    if (EP == EP_AXPY) {
      const V *aux = (const V *)a.aux + cb;
      const R cx = a.caux;
#pragma unroll
      for (int i = 0; i < NA; i++) {
        if (i >= nf) break;
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
      // clover blocks: block 0 acts on spin (0,1), block 1 on spin (2,3)
      clover_epilogue<NA, EP>(r0, r1, a, ca, cb, 0, cb, ld);
      clover_epilogue<NA, EP>(r2, r3, a, ca, cb, 1, cb, ld);
    }
    const R sg = a.g5 ? (R)-1 : (R)1;
#pragma unroll
    for (int i = 0; i < NA; i++) {
      if (i >= nf) break;
      V o2 = cscale(sg, r2[i]), o3 = cscale(sg, r3[i]);
      out[(long)(0 * nf + i) * ld] = r0[i];
      out[(long)(1 * nf + i) * ld] = r1[i];
      out[(long)(2 * nf + i) * ld] = o2;
      out[(long)(3 * nf + i) * ld] = o3;
      if (a.red) {
        nrm += (double)r0[i].x * r0[i].x + (double)r0[i].y * r0[i].y + (double)r1[i].x * r1[i].x +
               (double)r1[i].y * r1[i].y + (double)o2.x * o2.x + (double)o2.y * o2.y + (double)o3.x * o3.x +
               (double)o3.y * o3.y;
      }
    }
  }
  return nrm;
}

// threads per output site of a single-field hop variant: 2 for the spin-split
// variants 1 and 3, 1 for the others (0, 2, 4 and 5)
__host__ __device__ constexpr int hop_threads_per_site(int variant) { return (variant == 1 || variant == 3) ? 2 : 1; }

// Programmatic dependent launch: let the next kernel of the stream be scheduled
// as soon as every block of this one has started (its blocks then fill the SMs
// that this launch's last, partial wave leaves idle), and wait for the previous
// kernel and its memory before touching global memory.  Both are no-ops for a
// launch without the programmatic-serialization attribute.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// RC: rebuild row 2 of the 3x3 links (instantiated for NF = 3 only); FR: build
// the NF = 6 two-index links from the fundamental ones (see TwoIdx)
template <int NFT, bool REAL, typename R, int EP, int MINB, typename LE = typename LinkE<REAL, R>::T, bool RC = false,
          int FR = 0>
__global__ void __launch_bounds__(HOP_THREADS, MINB) k_hop(HopArgs<R> a) {
  pdl_enter();
  if (a.stop && *a.stop) return;
  const int cb = a.cb0 + blockIdx.x * blockDim.x + threadIdx.x;
  double nrm = 0.0;
  if (cb < a.cb1) nrm = hop_site<NFT, REAL, R, EP, LE, false, RC, FR>(a, cb);
  if (a.red) block_partial<R>(nrm, a.red);
}

// ---------------------------------------------------------------------------
// Spin-split variant: two threads per site.  Thread h (0 or 1) carries the
// half-spinor projection that starts from spin component h: for direction mu
// and sign s it forms hv = psi_h + f * psi_t (t the partner component of
// (1 -/+ gamma_mu), f = +-1 or +-i), multiplies by U or U^+, adds the product
// to output spin h, and adds conj(f) times it to a partial sum of output spin t.
// The partial sums of spins 2 and 3 of the two threads are combined with one
// lane shuffle at the end.  Each thread holds a third of the accumulators of
// k_hop, so the register count (and with it the number of resident warps that
// keep loads in flight) improves; links are loaded by both threads of a pair at
// the same address (one transaction).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int partner_of(int mu, int h) { return (mu == 0 || mu == 3) ? 2 + h : 3 - h; }

template <typename V>
__device__ __forceinline__ V shfl_pair(V v) {
  V r;
  r.x = __shfl_xor_sync(0xffffffffu, v.x, 1);
  r.y = __shfl_xor_sync(0xffffffffu, v.y, 1);
  return r;
}

// z * v for z in {+1, -1, +i, -i}: (re, im) selector
template <typename V>
__device__ __forceinline__ V mul_unit(V v, int re, int im) {
  V r;
  if (im == 0) { r.x = re * v.x; r.y = re * v.y; }
  else { r.x = -im * v.y; r.y = im * v.x; }
  return r;
}

// one thread (half h of the pair) of site cb; inactive threads compute but do
// not write (their partner needs the shuffles)
template <int NFT, bool REAL, typename R, int EP, typename LE = typename LinkE<REAL, R>::T>
__device__ __forceinline__ double hop2_site(const HopArgs<R> &a, const int cb, const int h, const bool active) {
  typedef typename C2<R>::T V;
  typedef LE E;
  constexpr int NA = NFT;
  const int nf = NFT;
  const Geo g = a.g;
  const int outp = a.outp, inp = outp ^ 1;
  int t, x, y, z;
  cb_to_coords(g, cb, outp, t, x, y, z);
  const long ld = g.ld, lplane = 2L * g.ld;
  const V *in = (const V *)a.in;
  const E *U = (const E *)a.U;
  const long nf2 = (long)nf * nf;
  V rm[NA], p2[NA], p3[NA], hv[NA], ch[NA];
#pragma unroll
  for (int i = 0; i < NA; i++) rm[i] = p2[i] = p3[i] = cmk<V>(0.0, 0.0);
  const long so = (long)outp * g.ld + cb;
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    int tp = t, xp = x, yp = y, zp = z, tm = t, xm = x, ym = y, zm = z;
    if (mu == 0) { tp = (t + 1 == g.T) ? 0 : t + 1; tm = (t == 0) ? g.T - 1 : t - 1; }
    if (mu == 1) { xp = (x + 1 == g.X) ? 0 : x + 1; xm = (x == 0) ? g.X - 1 : x - 1; }
    if (mu == 2) { yp = (y + 1 == g.Y) ? 0 : y + 1; ym = (y == 0) ? g.Y - 1 : y - 1; }
    if (mu == 3) { zp = (z + 1 == g.Z) ? 0 : z + 1; zm = (z == 0) ? g.Z - 1 : z - 1; }
    const E *Umu = U + (long)mu * nf2 * lplane;
    const int pt = partner_of(mu, h);
    // projection factor f for sign +: mu0: 1; mu1: i; mu2: (h ? -1 : 1); mu3: (h ? -i : i)
    const int fre = (mu == 0) ? 1 : (mu == 2) ? (h ? -1 : 1) : 0;
    const int fim = (mu == 1) ? 1 : (mu == 3) ? (h ? -1 : 1) : 0;
#pragma unroll
    for (int sgn = 0; sgn < 2; sgn++) {  // 0: forward, 1: backward
      const int s = sgn ? -1 : 1;
      const int cn = sgn ? coords_to_cb(g, tm, xm, ym, zm) : coords_to_cb(g, tp, xp, yp, zp);
      const V *sp = in + cn;
#pragma unroll
      for (int i = 0; i < NA; i++) {
        V a0 = ld_c(sp + (long)(h * nf + i) * ld);
        V a1 = ld_c(sp + (long)(pt * nf + i) * ld);
        hv[i] = cadd(a0, mul_unit(a1, s * fre, s * fim));
      }
      if (sgn == 0) link_mul<NA, false>(ch, hv, Umu, lplane, so, nf);
      else link_mul<NA, true>(ch, hv, Umu, lplane, (long)inp * g.ld + cn, nf);
      // reconstruction: output spin h += chi, output spin pt += conj(f) chi
#pragma unroll
      for (int i = 0; i < NA; i++) {
        rm[i] = cadd(rm[i], ch[i]);
        V c = mul_unit(ch[i], s * fre, -s * fim);
        if (pt == 2) p2[i] = cadd(p2[i], c);
        else p3[i] = cadd(p3[i], c);
      }
    }
  }
  // combine the partial sums of spins 2 and 3 over the thread pair
#pragma unroll
  for (int i = 0; i < NA; i++) {
    p2[i] = cadd(p2[i], shfl_pair(p2[i]));
    p3[i] = cadd(p3[i], shfl_pair(p3[i]));
  }
  const R ca = a.cacc;
  double nrm = 0.0;
  V *out = (V *)a.out + cb;
  const R sg = a.g5 ? (R)-1 : (R)1;
  if (EP == EP_AXPY) {
    // thread h writes spins h and 2+h
    const V *aux = (const V *)a.aux + cb;
#pragma unroll
    for (int i = 0; i < NA; i++) {
      V o0 = cscale(ca, rm[i]), o1 = cscale(ca, h ? p3[i] : p2[i]);
      if (aux != nullptr && a.caux != (R)0) {
        rmac(o0, a.caux, ld_c(aux + (long)(h * nf + i) * ld));
        rmac(o1, a.caux, ld_c(aux + (long)((2 + h) * nf + i) * ld));
      }
      o1 = cscale(sg, o1);
      if (active) {
        out[(long)(h * nf + i) * ld] = o0;
        out[(long)((2 + h) * nf + i) * ld] = o1;
      }
      nrm += (double)o0.x * o0.x + (double)o0.y * o0.y + (double)o1.x * o1.x + (double)o1.y * o1.y;
    }
  } else {
    // thread h applies clover block h: block 0 on spins (0,1), block 1 on spins (2,3)
    V other[NA];
#pragma unroll
    for (int i = 0; i < NA; i++) other[i] = shfl_pair(rm[i]);
    V xin[2 * NA], yout[2 * NA];
    const long lp = 2L * g.ld, site = (long)outp * g.ld + cb;
    const int n2 = 2 * nf, no = nf * (2 * nf - 1);
#pragma unroll
    for (int i = 0; i < NA; i++) {
      V u0 = h ? p2[i] : rm[i];     // spin 2h
      V u1 = h ? p3[i] : other[i];  // spin 2h+1
      if (EP == EP_CLOV_INV) {
        xin[i] = cscale(ca, u0);
        xin[nf + i] = cscale(ca, u1);
      } else {
        const V *aux = (const V *)a.aux + cb;
        xin[i] = ld_c(aux + (long)((2 * h) * nf + i) * ld);
        xin[nf + i] = ld_c(aux + (long)((2 * h + 1) * nf + i) * ld);
        hv[i] = u0;
        ch[i] = u1;
      }
    }
    herm_apply<NA, 1>(yout, xin, a.cdg + (long)h * n2 * lp, a.cod + (long)h * no * lp, lp, site, nf);
    const R sb = h ? sg : (R)1;
#pragma unroll
    for (int i = 0; i < NA; i++) {
      V o0 = yout[i], o1 = yout[nf + i];
      if (EP == EP_CLOV) {
        o0 = cadd(cscale(ca, hv[i]), o0);
        o1 = cadd(cscale(ca, ch[i]), o1);
      }
      o0 = cscale(sb, o0);
      o1 = cscale(sb, o1);
      if (active) {
        out[(long)((2 * h) * nf + i) * ld] = o0;
        out[(long)((2 * h + 1) * nf + i) * ld] = o1;
      }
      nrm += (double)o0.x * o0.x + (double)o0.y * o0.y + (double)o1.x * o1.x + (double)o1.y * o1.y;
    }
  }
  return active ? nrm : 0.0;
}

template <int NFT, bool REAL, typename R, int EP, int MINB, typename LE = typename LinkE<REAL, R>::T>
__global__ void __launch_bounds__(HOP_THREADS, MINB) k_hop2(HopArgs<R> a) {
  pdl_enter();
  if (a.stop && *a.stop) return;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = a.cb0 + (tid >> 1) < a.cb1;
  const int cb = active ? a.cb0 + (tid >> 1) : a.cb1 - 1;
  double nrm = hop2_site<NFT, REAL, R, EP, LE>(a, cb, tid & 1, active);
  if (a.red) block_partial<R>(nrm, a.red);
}

}  // namespace hrgpu
