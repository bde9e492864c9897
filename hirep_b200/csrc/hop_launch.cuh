// hop_launch.cuh -- host-side dispatch of the hopping kernel over NF and the
// epilogue; instantiated once per precision (dirac_d.cu, dirac_f.cu) so the two
// compile in parallel.
#pragma once
#include "dirac.cuh"

namespace hrgpu {

template <typename R, int EP>
int launch_ep_variant(HopArgs<R> &a, int variant) {
  a.g = make_geo();
  a.nf = L.nf;
  // variants: 0 one thread per site, 1 two threads per site (spin split),
  // 2 and 3 the same with the register budget capped for 4 resident blocks per SM
  const long threads = (variant & 1) ? 2L * L.VH : L.VH;
  dim3 grid((unsigned)((threads + HOP_THREADS - 1) / HOP_THREADS)), block(HOP_THREADS);
  cudaStream_t s = L.stream;
#define HOPV(N, RL)                                                                    \
  case N:                                                                              \
    switch (variant) {                                                                 \
      case 0: k_hop<N, RL, R, EP, 1><<<grid, block, 0, s>>>(a); break;                 \
      case 1: k_hop2<N, RL, R, EP, 1><<<grid, block, 0, s>>>(a); break;                \
      case 2: k_hop<N, RL, R, EP, 4><<<grid, block, 0, s>>>(a); break;                 \
      default: k_hop2<N, RL, R, EP, 4><<<grid, block, 0, s>>>(a); break;               \
    }                                                                                  \
    break;
#define HOPC(N) HOPV(N, false)
#define HOPR(N) HOPV(N, true)
  if (!L.real) {
    switch (L.nf) {
      HOPC(2) HOPC(3) HOPC(4) HOPC(5) HOPC(6) HOPC(10)
      default: set_error("no hopping kernel instantiated for complex NF=%d", L.nf); return HRGPU_E_NF;
    }
  } else {
    switch (L.nf) {
      HOPR(3) HOPR(8) HOPR(15)
      default: set_error("no hopping kernel instantiated for real NF=%d", L.nf); return HRGPU_E_NF;
    }
  }
#undef HOPC
#undef HOPR
#undef HOPV
  HR_LAUNCH_CHECK();
  return 0;
}

// Autotuner: the first launch of each (precision, epilogue) on a lattice times
// both variants on the real arguments (3 launches each, CUDA events on the
// library stream) and keeps the faster one.  The output is rewritten by the
// final launch, so tuning does not change results.  hrgpu_set_hop_variant forces
// a variant (tests use it to check both).
template <typename R, int EP>
int launch_ep(HopArgs<R> &a) {
  const int pi = sizeof(R) == 8 ? 0 : 1;
  int &v = L.hop_variant[pi][EP];
  if (L.hop_force >= 0) return launch_ep_variant<R, EP>(a, L.hop_force);
  if (v < 0) {
    float best = 1e30f;
    int bestv = 0;
    cudaEvent_t e0, e1;
    HR_CUDA(cudaEventCreate(&e0));
    HR_CUDA(cudaEventCreate(&e1));
    for (int cand = 0; cand < HOP_VARIANTS; cand++) {
      if (int rc = launch_ep_variant<R, EP>(a, cand)) return rc;  // warm-up
      HR_CUDA(cudaEventRecord(e0, L.stream));
      for (int r = 0; r < 3; r++)
        if (int rc = launch_ep_variant<R, EP>(a, cand)) return rc;
      HR_CUDA(cudaEventRecord(e1, L.stream));
      HR_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      HR_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      L.hop_tune_ms[pi][EP][cand] = ms / 3.0f;
      if (ms < best) {
        best = ms;
        bestv = cand;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    v = bestv;
  }
  return launch_ep_variant<R, EP>(a, v);
}




}  // namespace hrgpu
