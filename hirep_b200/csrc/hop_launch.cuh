// hop_launch.cuh -- host-side dispatch of the hopping kernel over NF and the
// epilogue; instantiated once per precision (dirac_d.cu, dirac_f.cu) so the two
// compile in parallel.
#pragma once
#include "dirac.cuh"

namespace hrgpu {

template <typename R, int EP>
int launch_ep(HopArgs<R> &a) {
  a.g = make_geo();
  a.nf = L.nf;
  dim3 grid((unsigned)((L.VH + HOP_THREADS - 1) / HOP_THREADS)), block(HOP_THREADS);
  cudaStream_t s = L.stream;
#define HOPC(N) case N: k_hop<N, false, R, EP><<<grid, block, 0, s>>>(a); break;
#define HOPR(N) case N: k_hop<N, true, R, EP><<<grid, block, 0, s>>>(a); break;
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
  HR_LAUNCH_CHECK();
  return 0;
}

template <typename R>
int launch_hop(int ep, HopArgs<R> &a) {
  if (ep == EP_AXPY) return launch_ep<R, EP_AXPY>(a);
  if (ep == EP_CLOV_INV) return launch_ep<R, EP_CLOV_INV>(a);
  return launch_ep<R, EP_CLOV>(a);
}


}  // namespace hrgpu
