// hop_batch_launch.cuh -- host-side dispatch of the batch hopping kernel
// (k_hopt) over NF and variant, with its autotuner; instantiated per precision
// and epilogue in dirac_b_*.cu.
#pragma once
#include "dirac.cuh"
#include "hop_tc.cuh"
#include "hop_tcp.cuh"
#include "hop_tile.cuh"

namespace hrgpu {

// Outside a stream capture the error word of a tensor-core launch is read back
// at once, so a bounded wait that gave up is reported as an error status.
inline int tc_check_error_word(const char *what) {
  HR_LAUNCH_CHECK();
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  HR_CUDA(cudaStreamIsCapturing(L.stream, &cs));
  if (cs != cudaStreamCaptureStatusNone) return 0;
  unsigned h = 0;
  HR_CUDA(cudaMemcpyAsync(&h, L.hopb_err, sizeof(unsigned), cudaMemcpyDeviceToHost, L.stream));
  HR_CUDA(cudaStreamSynchronize(L.stream));
  if (h) {
    HR_CUDA(cudaMemsetAsync(L.hopb_err, 0, sizeof(unsigned), L.stream));
    set_error("%s: a bounded wait for its MMAs gave up (error word %u)", what, h);
    return HRGPU_E_CUDA;
  }
  return 0;
}

inline int tc_prepare() {
  if (!L.hopb_err) {
    HR_CUDA(cudaMalloc(&L.hopb_err, sizeof(unsigned)));
    HR_CUDA(cudaMemsetAsync(L.hopb_err, 0, sizeof(unsigned), L.stream));
  }
  if (!L.num_sms) {
    int dev = 0;
    HR_CUDA(cudaGetDevice(&dev));
    HR_CUDA(cudaDeviceGetAttribute(&L.num_sms, cudaDevAttrMultiProcessorCount, dev));
  }
  return 0;
}

// variant 3: the tensor-core kernel (FP32, complex NF = 6, nb <= 32; -1 where
// it is not built), a persistent grid of up to four CTAs per SM.
// variant 4: the same GEMM with the neighbours prefetched (nb <= 16), one CTA
// of two warpgroups per SM.
template <typename R, int EP>
int launch_batch_tc(TileArgs<R> &a, int variant) {
  if constexpr (sizeof(R) != 4) {
    return -1;
  } else {
    if (L.real || L.nf != 6 || a.nb > (variant == 4 ? TCP_NBMAX : 32)) return -1;
    if (int rc = tc_prepare()) return rc;
    if (variant == 3) {
      const size_t smem = tc_smem_bytes<6>();
      HR_CUDA(cudaFuncSetAttribute(k_hopt_tc<6, EP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      const long grid = std::min<long>(L.VH, 4L * L.num_sms);
      k_hopt_tc<6, EP><<<(unsigned)grid, TC_THREADS, smem, L.stream>>>(a, L.hopb_err);
      return tc_check_error_word("tensor-core batch kernel");
    }
    const size_t smem = TcpLayout<6>::SMEM;
    HR_CUDA(cudaFuncSetAttribute(k_hopt_tcp<6, EP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long grid = std::min<long>(L.VH, (long)L.num_sms);
    k_hopt_tcp<6, EP><<<(unsigned)grid, TCP_THREADS, smem, L.stream>>>(a, L.hopb_err);
    return tc_check_error_word("tensor-core batch kernel (prefetched)");
  }
}

// variants: the register budget for 1, 3 or 4 resident blocks of 128 threads per SM; 5:
// the budget of 1 block with the link products in packed FP32 FMAs (complex FP32)
template <typename R, int EP>
int launch_batch_variant(TileArgs<R> &a, int variant) {
  a.g = make_geo();
  if (variant == 3 || variant == 4) return launch_batch_tc<R, EP>(a, variant);
  // 32 threads per (group of 8 sites, tile)
  const long threads = ((L.VH + TILE_S - 1) / TILE_S) * 32L * ((a.nb + TILE_F - 1) / TILE_F);
  dim3 grid((unsigned)((threads + HOPT_THREADS - 1) / HOPT_THREADS)), block(HOPT_THREADS);
  cudaStream_t s = L.stream;
#define HOPTV(N, RL)                                                       \
  case N:                                                                  \
    switch (variant) {                                                     \
      case 0: k_hopt<N, RL, R, EP, 1><<<grid, block, 0, s>>>(a); break;     \
      case 1: k_hopt<N, RL, R, EP, 3><<<grid, block, 0, s>>>(a); break;     \
      case 5:                                                              \
        if constexpr (!RL && sizeof(R) == 4) {                             \
          k_hopt<N, RL, R, EP, 1, true><<<grid, block, 0, s>>>(a);         \
          break;                                                           \
        } else {                                                           \
          return -1;                                                       \
        }                                                                  \
      default: k_hopt<N, RL, R, EP, 4><<<grid, block, 0, s>>>(a); break;    \
    }                                                                      \
    break;
  if (!L.real) {
    switch (L.nf) {
      HOPTV(2, false) HOPTV(3, false) HOPTV(4, false) HOPTV(5, false) HOPTV(6, false) HOPTV(10, false)
      default: set_error("no batch hopping kernel for complex NF=%d", L.nf); return HRGPU_E_NF;
    }
  } else {
    switch (L.nf) {
      HOPTV(3, true) HOPTV(8, true) HOPTV(15, true)
      default: set_error("no batch hopping kernel for real NF=%d", L.nf); return HRGPU_E_NF;
    }
  }
#undef HOPTV
  HR_LAUNCH_CHECK();
  return 0;
}

// Autotuner: the first launch for a (precision, epilogue, nb) times every
// variant (3 launches each after a warm-up, CUDA events on the library stream)
// and keeps the fastest; the final launch rewrites the output, so tuning does
// not change results.  While the stream is being captured into a CUDA graph
// nothing can be timed: an untuned case then runs variant 0 untuned.
template <typename R, int EP>
int launch_batch(TileArgs<R> &a) {
  const int pi = sizeof(R) == 8 ? 0 : 1;
  if (L.hopb_force >= 0) {
    const int rc = launch_batch_variant<R, EP>(a, L.hopb_force);
    if (rc < 0) {
      set_error("batch hopping-kernel variant %d is not built for this case (precision, NF=%d, nb=%d)", L.hopb_force,
                L.nf, a.nb);
      return HRGPU_E_NF;
    }
    return rc;
  }
  signed char &v = L.hopb_variant[pi][EP][a.nb];
  if (v == 0) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    HR_CUDA(cudaStreamIsCapturing(L.stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return launch_batch_variant<R, EP>(a, 0);
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
      for (int cand = 0; cand < HOPB_VARIANTS; cand++) {
        if (cand == 3 || cand == 4) {  // the tensor-core kernels run when pinned (hrgpu_set_batch_variant(3 or 4))
          L.hopb_tune_ms[pi][EP][a.nb][cand] = -1.0f;
          continue;
        }
        const int rc0 = launch_batch_variant<R, EP>(a, cand);
        if (rc0 < 0) {  // not built for this precision or representation
          L.hopb_tune_ms[pi][EP][a.nb][cand] = -1.0f;
          continue;
        }
        if (rc0) return rc0;
        HR_CUDA(cudaEventRecord(e0, L.stream));
        for (int r = 0; r < 3; r++)
          if (int rc = launch_batch_variant<R, EP>(a, cand)) return rc;
        HR_CUDA(cudaEventRecord(e1, L.stream));
        HR_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        HR_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        L.hopb_tune_ms[pi][EP][a.nb][cand] = ms / 3.0f;
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
    v = (signed char)(bestv + 1);
  }
  return launch_batch_variant<R, EP>(a, v - 1);
}

}  // namespace hrgpu
