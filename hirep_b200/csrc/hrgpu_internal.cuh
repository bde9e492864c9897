// hrgpu_internal.cuh -- shared definitions of the B200 fermion library.
//
// Device data layout (HBM), chosen for coalesced FP64/FP32 streaming:
//   site index     d = p * ld + cb, p = (t+x+y+z)&1, cb = lex >> 1,
//                  lex = ((t*Z + z)*Y + y)*X + x    (x fastest, X even)
//   spinor field   one parity: [4*NF complex components][ld] as double2/float2
//                  full lattice: [2 parities][4*NF][ld]
//   links          [4 dirs][NF*NF elements][2*ld] (double2/float2, or double/float
//                  for real representations)
//   clover blocks  two Hermitian 2NF x 2NF blocks per site, packed lower
//                  triangle: diag [2][2NF][2*ld] real, off [2][NF(2NF-1)][2*ld] complex
// HiRep's own (host) layout and site numbering are translated at the boundary by
// a permutation table built from HiRep's ipt[] map.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <string>

#include "../../include/hrgpu.h"

namespace hrgpu {

// ---------------------------------------------------------------------------
// error handling: every CUDA call is checked; failures set the library error
// string and make the entry point return a non-zero status.
// ---------------------------------------------------------------------------
void set_error(const char *fmt, ...);
int fail_cuda(cudaError_t e, const char *what, const char *file, int line);

#define HR_CUDA(call)                                                   \
  do {                                                                  \
    cudaError_t _e = (call);                                            \
    if (_e != cudaSuccess) return hrgpu::fail_cuda(_e, #call, __FILE__, __LINE__); \
  } while (0)

#define HR_LAUNCH_CHECK() HR_CUDA(cudaGetLastError())

#define HR_REQUIRE(cond, code, ...)      \
  do {                                   \
    if (!(cond)) {                       \
      hrgpu::set_error(__VA_ARGS__);     \
      return (code);                     \
    }                                    \
  } while (0)

constexpr int MAXNF = 64;
constexpr int RED_THREADS = 256;
constexpr int RED_MAX_BLOCKS = 1184;  // 8 x 148 SMs
constexpr int HOP_VARIANTS = 7;
constexpr int HOPB_VARIANTS = 6;   // batch hopping kernel variants (3, 4: tensor cores; 5: packed FP32 FMAs)
constexpr int HOPB_MAXNB = 64;     // fields per batch

struct Lattice {
  bool ready = false;
  int T = 0, X = 0, Y = 0, Z = 0;
  long V = 0, VH = 0;
  int ld = 0;  // plane stride of one parity (>= VH, multiple of 32)
  int ng = 0, nf = 0, repr = 0, real = 0, dimg = 0;
  // HiRep site index -> device site index (p*ld+cb); and inverse
  int *d_h2d = nullptr, *d_d2h = nullptr;
  int *h_h2d = nullptr;
  // gauge fields
  void *U = nullptr;      // represented links, double (double2 or double)
  void *Uf = nullptr;     // represented links, float
  float2 *Ugf = nullptr;  // fundamental links, float (for the FP32 hop of link modes 3 and 4)
  double2 *Ug = nullptr;  // fundamental links [4][ng*ng][2*ld]
  bool have_gauge = false, have_gauge_flt = false, have_fund = false;
  // clover
  bool clover = false;
  bool expclover = false;         // WITH_EXPCLOVER: diagonal (4+m) exp(A/(4+m))
  double csw = 0.0;
  double sigma = 0xF00F;          // mass term (4+m) the inverse was built for
  double2 *cl_term = nullptr;     // A blocks s0..s3 [4][nf*nf][2*ld]
  double *cl_dg = nullptr;        // (4+m)+A packed: diag [2][2nf][2*ld]
  double2 *cl_od = nullptr;       //                 off  [2][nf(2nf-1)][2*ld]
  double *cl_idg = nullptr;       // inverse, same packing
  double *cl_ldet = nullptr;      // [2ld] product of the LDL diagonals of both blocks (det D_oo)
  double2 *cl_iod = nullptr;
  float *cl_dg_f = nullptr, *cl_idg_f = nullptr;
  float2 *cl_od_f = nullptr, *cl_iod_f = nullptr;
  double sigma_diag = 0xF00F;     // mass term the packed diag was built for
  double sigma_flt = 0xF00F;
  // force and HMC
  double *force_sum = nullptr;    // [4][dimg][2*ld]
  double *mom = nullptr;          // momenta [4][dimg][2*ld]
  int bc_t = 1;                   // time boundary condition of the last represent_gauge_field
  // hopping kernels rebuild row 2 of each 3x3 link (SU(3) fundamental, SU(2)
  // adjoint) from rows 0 and 1: 0 no (full loads), 1 yes, 2 yes with the
  // antiperiodic-T sign on mu = 0 links at t = 0 (set by represent_gauge_field
  // after checking every link)
  int recon12 = 0;
  bool recon_allow = true;        // hrgpu_set_link_recon
  double2 *cl_force = nullptr;    // [6][nf*nf][2*ld]
  // algebra projection tables (sparse): for each generator A, entries (k=i*nf+j, coeff)
  int *d_proj_off = nullptr;      // [dimg+1]
  int *d_proj_k = nullptr;
  double2 *d_proj_c = nullptr;    // conj(R(iT_A))_k / C(R)
  // the same table by matrix element k: for each k the (A, coefficient) pairs
  int *d_projk_off = nullptr;     // [nf*nf+1]
  int *d_projk_A = nullptr;
  double2 *d_projk_c = nullptr;
  double repr_norm2 = 0.0, fund_norm2 = 0.5;
  double *h_rT = nullptr;         // host copy of R(iT_A) as complex pairs [dimg][nf*nf][2]
  double *h_gT = nullptr;         // host copy of T_A [dimg][ng*ng][2]
  // scratch
  double *partials = nullptr;     // reduction partials (npart doubles, results after them)
  long npart = 0;
  double *h_partials = nullptr;   // pinned host mirror of the final values
  double *d_scalars = nullptr;    // CG scalars
  const int *cur_stop = nullptr;  // set by the inverters while they drive the operator
  // tuned hopping-kernel variant [FP64, FP32, FP32 with BF16 links][epilogue]
  int hop_variant[3][3] = {{-1, -1, -1}, {-1, -1, -1}, {-1, -1, -1}};
  int hop_force = -1;             // forced variant (-1: autotune)
  unsigned *hop_err = nullptr;    // device error word of the TMA-staged variant
  bool hop_pdl = true;            // whole-lattice hops with programmatic dependent launch
  float hop_tune_ms[3][3][HOP_VARIANTS] = {};  // tuning times of the variants [slot][epilogue][variant]
  // storage of the links read by the FP32 operators: HRGPU_LINKS_F32 (Uf) or HRGPU_LINKS_BF16 (Ubf)
  int flt_links = 0;
  void *Ubf = nullptr;
  unsigned long ubf_gen = ~0UL;
  // multi-field kernel: tuned variant + 1 (0 = not tuned yet) [prec][epilogue][nb], its timings, forced variant
  signed char hopb_variant[2][3][HOPB_MAXNB + 1] = {};
  float hopb_tune_ms[2][3][HOPB_MAXNB + 1][HOPB_VARIANTS] = {};
  int hopb_force = -1;
  unsigned *hopb_err = nullptr;   // device error word of the tensor-core batch kernel
  int num_sms = 0;                // multiprocessors of the device (persistent grids)
  int force_variant = 0;          // kernel of the hopping force (0: the measured default)
  // change counters: links (double and float are rewritten together) and the
  // packed clover blocks of each precision; copies made from them record these
  unsigned long gauge_gen = 0, clover_gen[2] = {0, 0};
  cudaStream_t stream = 0;
  // temporaries (lazily allocated, sized for one parity unless noted)
  void *tmp_o = nullptr, *tmp_e = nullptr, *tmp_e2 = nullptr, *tmp_full = nullptr, *tmp_full2 = nullptr;
  void *tmp_o_f = nullptr, *tmp_e_f = nullptr, *tmp_full_f = nullptr;
  void *stage = nullptr;
  size_t stage_bytes = 0;
};

extern Lattice L;

inline size_t spinor_elems(int par) { return (size_t)(par == HRGPU_FULL ? 2 : 1) * 4 * L.nf * L.ld; }
inline size_t spinor_bytes(int par, int prec) {
  return spinor_elems(par) * (prec == HRGPU_DOUBLE ? sizeof(double2) : sizeof(float2));
}

int ensure_tmp(void **p, size_t bytes);
int library_device();  // the device of hrgpu_init (-1 before)
int ensure_links_bf16();  // the BF16 copy of the links, made from the FP64 ones when they changed
int detect_recon12();     // check links set already represented for row-2 reconstruction
void fund_links_changed(); // the fundamental links were written: stop building represented links from them
int compute_clover_term_dev();
void cg_release();
int ensure_stage(size_t bytes);
int spinor_scatter_even(void *dev, const void *stage, int base, int nsites, int prec, cudaStream_t s);
int spinor_gather_even(void *stage, const void *dev, int base, int nsites, int prec, cudaStream_t s);
void hostop_release();

// ---------------------------------------------------------------------------
// small complex helpers
// ---------------------------------------------------------------------------
template <typename R> struct C2;
template <> struct C2<double> { typedef double2 T; };
template <> struct C2<float> { typedef float2 T; };

template <typename V> __device__ __forceinline__ V cmk(double a, double b);
template <> __device__ __forceinline__ double2 cmk<double2>(double a, double b) { return make_double2(a, b); }
template <> __device__ __forceinline__ float2 cmk<float2>(double a, double b) { return make_float2((float)a, (float)b); }

template <typename V> __device__ __forceinline__ V cadd(V a, V b) { V r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { V r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
// a + i b, a - i b
template <typename V> __device__ __forceinline__ V caddi(V a, V b) { V r; r.x = a.x - b.y; r.y = a.y + b.x; return r; }
template <typename V> __device__ __forceinline__ V csubi(V a, V b) { V r; r.x = a.x + b.y; r.y = a.y - b.x; return r; }
// acc += u * s
template <typename V> __device__ __forceinline__ void cmac(V &acc, V u, V s) {
  acc.x = fma(u.x, s.x, acc.x); acc.x = fma(-u.y, s.y, acc.x);
  acc.y = fma(u.x, s.y, acc.y); acc.y = fma(u.y, s.x, acc.y);
}
// acc += conj(u) * s
template <typename V> __device__ __forceinline__ void cmacc(V &acc, V u, V s) {
  acc.x = fma(u.x, s.x, acc.x); acc.x = fma(u.y, s.y, acc.x);
  acc.y = fma(u.x, s.y, acc.y); acc.y = fma(-u.y, s.x, acc.y);
}
// acc += r * s (r real)
template <typename V, typename R> __device__ __forceinline__ void rmac(V &acc, R r, V s) {
  acc.x = fma(r, s.x, acc.x); acc.y = fma(r, s.y, acc.y);
}
template <typename V, typename R> __device__ __forceinline__ V cscale(R r, V a) { V o; o.x = r * a.x; o.y = r * a.y; return o; }
template <typename V> __device__ __forceinline__ V cmul(V a, V b) {
  V r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}

// Row 2 of a unitary 3x3 link with determinant s from rows 0 and 1 (elements
// u[0..5], row-major): u[6..8] = s conj(r0 x r1).  For U in SU(3) (s = 1), and
// for -U (s = -1, a link that carries the antiperiodic time sign), this is the
// stored row to rounding.
// the same for a real orthogonal 3x3 link (SU(2) in the adjoint
// representation, SO(3)): u[6..8] = s (r0 x r1)
template <typename R>
__device__ __forceinline__ void so3_row2(R *u, R s) {
  u[6] = s * (u[1] * u[5] - u[2] * u[4]);
  u[7] = s * (u[2] * u[3] - u[0] * u[5]);
  u[8] = s * (u[0] * u[4] - u[1] * u[3]);
}

template <typename V, typename R>
__device__ __forceinline__ void su3_row2(V *u, R s) {
  V q;
  q = csub(cmul(u[1], u[5]), cmul(u[2], u[4]));
  u[6].x = s * q.x; u[6].y = -s * q.y;
  q = csub(cmul(u[2], u[3]), cmul(u[0], u[5]));
  u[7].x = s * q.x; u[7].y = -s * q.y;
  q = csub(cmul(u[0], u[4]), cmul(u[1], u[3]));
  u[8].x = s * q.x; u[8].y = -s * q.y;
}

// Sum of v over the thread block in a fixed order, so the result is the same on
// every run: a shuffle tree inside each warp, then warp 0 adds the warp sums
// with a second shuffle tree.  Every thread gets the sum.  blockDim.x must be a
// multiple of 32 and every thread of the block must call it.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double warp_sums[32];
  __shared__ double total;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) warp_sums[w] = v;
  __syncthreads();
  if (w == 0) {
    double s = lane < nw ? warp_sums[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) total = s;
  }
  __syncthreads();
  // a following call writes warp_sums only after this barrier and total only
  // after its own first barrier, which every thread reaches after reading total
  return total;
}

// ---------------------------------------------------------------------------
// lattice coordinates on the device
// ---------------------------------------------------------------------------
struct Geo {
  int X, Y, Z, T;  // sizes
  int Xh;          // X/2
  int ld;
  int VH;
};

__device__ __forceinline__ void cb_to_coords(const Geo &g, int cb, int p, int &t, int &x, int &y, int &z) {
  int xh = cb % g.Xh;
  int row = cb / g.Xh;
  y = row % g.Y;
  row /= g.Y;
  z = row % g.Z;
  t = row / g.Z;
  x = 2 * xh + ((p + t + y + z) & 1);
}

__device__ __forceinline__ int coords_to_cb(const Geo &g, int t, int x, int y, int z) {
  return (((t * g.Z + z) * g.Y + y) * g.X + x) >> 1;
}

Geo make_geo();

// reductions: block partial sums written to L.partials, folded on the device
int finish_reduction(int nblocks, int nvals, double *host_out);

}  // namespace hrgpu
