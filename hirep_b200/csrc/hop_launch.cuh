// hop_launch.cuh -- host-side dispatch of the hopping kernel over NF and the
// epilogue; instantiated once per precision (dirac_d.cu, dirac_f.cu) so the two
// compile in parallel.
#pragma once
#include "dirac.cuh"
#include "hop_async.cuh"
#include "hop_tma.cuh"

namespace hrgpu {

// A whole-lattice FP64 hop is launched with programmatic stream serialisation
// (the kernels wait on their predecessor with griddepcontrol.wait before
// reading memory), so its blocks fill the SMs the previous hop's last wave
// leaves idle: Cphi_eopre 62.5 -> 60.4 us at 16^3x32 (alternating A/B in one
// process), the FP64 CG unchanged.  Without it: FP32 hops (inside the mixed
// solve's graphs it cost 3 %: 18.7 -> 19.3 ms) and launches over a few time
// slabs (the host-field pipeline, where the early, waiting blocks held SMs
// that the copy-stream kernels beside them needed: 0.47 -> 0.69 ms).
template <typename R>
static inline cudaError_t launch_pdl(void (*kernel)(HopArgs<R>), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                     HopArgs<R> &a) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = (L.hop_pdl && sizeof(R) == 8 && a.cb0 == 0 && a.cb1 == (int)L.VH) ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, a);
}

template <int N, bool RL, typename R, int EP>
int launch_async(HopArgs<R> &a, dim3 grid, dim3 block, cudaStream_t s) {
  if constexpr (AsyncOK<N, RL>::v) {
    constexpr int smem = AsyncLayout<N, RL, R>::SMEM;
    static bool attr = false;
    if (!attr) {
      HR_CUDA(cudaFuncSetAttribute(k_hop_async<N, RL, R, EP>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      attr = true;
    }
    HR_CUDA(launch_pdl<R>(k_hop_async<N, RL, R, EP>, grid, block, smem, s, a));
    return 0;
  } else {
    return -1;  // not built for this NF
  }
}

// variant 5: the time halo staged by bulk copies, for the small representations
// and where blocks of HOP_THREADS sites tile the time slabs of the launch
template <int N, bool RL, typename R, int EP>
int launch_tma(HopArgs<R> &a, dim3 grid, dim3 block, cudaStream_t s) {
  if constexpr (AsyncOK<N, RL>::v) {
    const int S = a.g.Xh * a.g.Y * a.g.Z;
    if (S % HOP_THREADS != 0 || a.cb0 % HOP_THREADS != 0 || (a.cb1 - a.cb0) % HOP_THREADS != 0) return -1;
    constexpr int smem = TmaLayout<N, R>::SMEM;
    static bool attr = false;
    if (!attr) {
      HR_CUDA(cudaFuncSetAttribute(k_hop_tma<N, RL, R, EP>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      attr = true;
    }
    HR_CUDA(launch_pdl<R>(k_hop_tma<N, RL, R, EP>, grid, block, smem, s, a));
    return 0;
  } else {
    return -1;  // not built for this NF
  }
}

// k_hop for variants 0 and 2: the instantiation that rebuilds row 2 of the
// 3x3 links (SU(3) fundamental, SU(2) adjoint) when the links passed the
// check, else the one reading full links
template <int N, bool RL, typename R, int EP, int MINB>
static inline void (*hop_kernel(int recon))(HopArgs<R>) {
  if constexpr (N == 3) {
    if (recon) return k_hop<N, RL, R, EP, MINB, typename LinkE<RL, R>::T, true>;
  }
  return k_hop<N, RL, R, EP, MINB>;
}

// variant 6: k_hop (variant 0's register budget) building the NF = 6
// two-index links from the fundamental ones (FP64 from L.Ug, FP32 from its
// float copy L.Ugf) while the fundamental links are those the represented
// field was made from (link modes 3 and 4); -1 otherwise
template <int N, bool RL, typename R, int EP>
int launch_fund(HopArgs<R> &a, dim3 grid, dim3 block, cudaStream_t s) {
  if constexpr (N == 6 && !RL) {
    if (a.recon < 3 || !a.Ug) return -1;
    if (L.repr == HRGPU_SYM)
      HR_CUDA(launch_pdl<R>(k_hop<N, RL, R, EP, 1, typename LinkE<RL, R>::T, false, 1>, grid, block, 0, s, a));
    else
      HR_CUDA(launch_pdl<R>(k_hop<N, RL, R, EP, 1, typename LinkE<RL, R>::T, false, 2>, grid, block, 0, s, a));
    return 0;
  } else {
    return -1;
  }
}

template <typename R, int EP>
int launch_ep_variant(HopArgs<R> &a, int variant) {
  a.g = make_geo();
  a.nf = L.nf;
  a.recon = L.recon_allow ? L.recon12 : 0;
  // variants: 0 one thread per site, 1 two threads per site (spin split),
  // 2 and 3 the same with the register budget capped for 4 resident blocks per SM,
  // 4 one thread per site with the per-direction loads pipelined through shared memory,
  // 5 one thread per site with the time halo staged by bulk (TMA) copies,
  // 6 one thread per site building the NF = 6 two-index links from the fundamental ones
  const long nsites = a.cb1 - a.cb0;
  const long threads = hop_threads_per_site(variant) * nsites;
  dim3 grid((unsigned)((threads + HOP_THREADS - 1) / HOP_THREADS)), block(HOP_THREADS);
  cudaStream_t s = L.stream;
#define HOPV(N, RL)                                                                    \
  case N:                                                                              \
    switch (variant) {                                                                 \
      case 0: HR_CUDA(launch_pdl<R>(hop_kernel<N, RL, R, EP, 1>(a.recon), grid, block, 0, s, a)); break; \
      case 1: HR_CUDA(launch_pdl<R>(k_hop2<N, RL, R, EP, 1>, grid, block, 0, s, a)); break; \
      case 2: HR_CUDA(launch_pdl<R>(hop_kernel<N, RL, R, EP, 4>(a.recon), grid, block, 0, s, a)); break; \
      case 3: HR_CUDA(launch_pdl<R>(k_hop2<N, RL, R, EP, 4>, grid, block, 0, s, a)); break; \
      case 4:                                                                          \
        if (int rc_ = launch_async<N, RL, R, EP>(a, grid, block, s)) return rc_;       \
        break;                                                                         \
      case 5:                                                                          \
        if (int rc_ = launch_tma<N, RL, R, EP>(a, grid, block, s)) return rc_;         \
        break;                                                                         \
      default:                                                                         \
        if (int rc_ = launch_fund<N, RL, R, EP>(a, grid, block, s)) return rc_;        \
        break;                                                                         \
    }                                                                                  \
    break;
#define HOPC(N) HOPV(N, false)
#define HOPR(N) HOPV(N, true)
  // FP32 operator with BF16 link storage: variants 0-3 (no cp.async form)
#define HOPVB(N, RL)                                                                            \
  case N:                                                                                       \
    switch (variant) {                                                                          \
      case 0: HR_CUDA(launch_pdl<float>(k_hop<N, RL, float, EP, 1, typename LinkBF16<RL>::T>, grid, block, 0, s, a)); break;  \
      case 1: HR_CUDA(launch_pdl<float>(k_hop2<N, RL, float, EP, 1, typename LinkBF16<RL>::T>, grid, block, 0, s, a)); break; \
      case 2: HR_CUDA(launch_pdl<float>(k_hop<N, RL, float, EP, 4, typename LinkBF16<RL>::T>, grid, block, 0, s, a)); break;  \
      case 3: HR_CUDA(launch_pdl<float>(k_hop2<N, RL, float, EP, 4, typename LinkBF16<RL>::T>, grid, block, 0, s, a)); break; \
      default: return -1;                                                                       \
    }                                                                                           \
    break;
  if constexpr (std::is_same<R, float>::value) {
    if (L.flt_links == HRGPU_LINKS_BF16) {
      if (!L.real) {
        switch (L.nf) {
          HOPVB(2, false) HOPVB(3, false) HOPVB(4, false) HOPVB(5, false) HOPVB(6, false) HOPVB(10, false)
          default: set_error("no hopping kernel instantiated for complex NF=%d", L.nf); return HRGPU_E_NF;
        }
      } else {
        switch (L.nf) {
          HOPVB(3, true) HOPVB(8, true) HOPVB(15, true)
          default: set_error("no hopping kernel instantiated for real NF=%d", L.nf); return HRGPU_E_NF;
        }
      }
      HR_LAUNCH_CHECK();
      return 0;
    }
  }
#undef HOPVB
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

// variant 5 (pinned with hrgpu_set_hop_variant): the launch gets the device
// error word, and outside a stream capture the word is read back at once, so a
// bounded wait that gave up (copies possibly still in flight into shared
// memory) is reported as an error status instead of passing silently
template <typename R, int EP>
int launch_tma_checked(HopArgs<R> &a) {
  if (!L.hop_err) {
    HR_CUDA(cudaMalloc(&L.hop_err, sizeof(unsigned)));
    HR_CUDA(cudaMemsetAsync(L.hop_err, 0, sizeof(unsigned), L.stream));
  }
  a.err = L.hop_err;
  int rc = launch_ep_variant<R, EP>(a, 5);
  a.err = nullptr;
  if (rc < 0) {
    set_error("hopping-kernel variant 5 is not built for NF=%d (or this lattice)", L.nf);
    return HRGPU_E_NF;
  }
  if (rc) return rc;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  HR_CUDA(cudaStreamIsCapturing(L.stream, &cs));
  if (cs != cudaStreamCaptureStatusNone) return 0;
  unsigned h = 0;
  HR_CUDA(cudaMemcpyAsync(&h, L.hop_err, sizeof(unsigned), cudaMemcpyDeviceToHost, L.stream));
  HR_CUDA(cudaStreamSynchronize(L.stream));
  if (h) {
    HR_CUDA(cudaMemsetAsync(L.hop_err, 0, sizeof(unsigned), L.stream));
    set_error("hopping-kernel variant 5: a bounded wait for the staged time halo gave up (error word %u)", h);
    return HRGPU_E_CUDA;
  }
  return 0;
}

// Autotuner: the first launch of each (precision, epilogue) on a lattice times
// every variant on the real arguments (3 launches each, CUDA events on the
// library stream) and keeps the faster one.  The output is rewritten by the
// final launch, so tuning does not change results.  hrgpu_set_hop_variant forces
// a variant (tests use it to check both).
template <typename R, int EP>
int launch_ep(HopArgs<R> &a) {
  // tuning slots: FP64, FP32, FP32 with BF16 links
  const int pi = sizeof(R) == 8 ? 0 : (L.flt_links == HRGPU_LINKS_BF16 ? 2 : 1);
  int &v = L.hop_variant[pi][EP];
  if (L.hop_force >= 0) {
    if (L.hop_force == 5) return launch_tma_checked<R, EP>(a);
    int rc = launch_ep_variant<R, EP>(a, L.hop_force);
    if (rc < 0) {
      set_error("hopping-kernel variant %d is not built for NF=%d", L.hop_force, L.nf);
      return HRGPU_E_NF;
    }
    return rc;
  }
  if (v < 0 && (a.cb0 != 0 || a.cb1 != L.VH)) {
    // a launch over part of the lattice is no measure for the full operator:
    // run the default variant and leave tuning to the first full launch
    return launch_ep_variant<R, EP>(a, 0);
  }
  if (v < 0) {
    // nothing can be timed while the stream is being captured into a CUDA
    // graph: run the default variant and leave tuning to an uncaptured launch
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    HR_CUDA(cudaStreamIsCapturing(L.stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return launch_ep_variant<R, EP>(a, 0);
  }
  if (v < 0) {
    float best = 1e30f;
    int bestv = 0;
    cudaEvent_t e0, e1;
    HR_CUDA(cudaEventCreate(&e0));
    if (cudaError_t err = cudaEventCreate(&e1)) {
      cudaEventDestroy(e0);
      return fail_cuda(err, "cudaEventCreate(&e1)", __FILE__, __LINE__);
    }
    // the events are destroyed on every way out of the loop
    auto tune = [&]() -> int {
      for (int cand = 0; cand < HOP_VARIANTS; cand++) {
        if (cand == 5) {  // the TMA-staged variant: slower in every measured case, pinned only
          L.hop_tune_ms[pi][EP][cand] = -1.0f;
          continue;
        }
        int rc0 = launch_ep_variant<R, EP>(a, cand);  // warm-up
        if (rc0 < 0) {  // variant not built for this NF
          L.hop_tune_ms[pi][EP][cand] = -1.0f;
          continue;
        }
        if (rc0) return rc0;
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
      return 0;
    };
    const int trc = tune();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (trc) return trc;
    // the candidates are timed on back-to-back launches with the operands
    // warm in L2, which favours the register-capped variants slightly over a
    // cold step (16^3x32 FP64: variant 2 1.5 % ahead warm, variant 0 1.5 %
    // ahead with L2 flushed): another variant replaces variant 0 only when it
    // is at least 3 % faster
    const float t0 = L.hop_tune_ms[pi][EP][0];
    if (bestv != 0 && t0 > 0.0f && best / 3.0f > 0.97f * t0) bestv = 0;
    v = bestv;
  }
  int rc = launch_ep_variant<R, EP>(a, v);
  // variant 6 chosen while the links could be built from the fundamental ones,
  // and the fundamental links written since: the stored links, variant 0
  if (rc < 0 && v == 6) rc = launch_ep_variant<R, EP>(a, 0);
  if (rc < 0) {
    set_error("hopping-kernel variant %d is not built for NF=%d", v, L.nf);
    return HRGPU_E_NF;
  }
  return rc;
}




}  // namespace hrgpu
