// noalloc.cu -- an even-odd Wilson operator entry point that allocates nothing.
//
// hrgpu_Dphi_eopre needs one odd-parity temporary (D_oe in) between its two
// hops, and on its first call it obtains it with cudaMalloc.  Some callers
// cannot let a library allocate device memory: a host framework that owns the
// whole GPU through its own memory pool (PyTorch's caching allocator, or a job
// that claims the device up front) either has no memory left for a raw
// cudaMalloc or must not have its accounting bypassed.  For them this file
// keeps the temporary in a fixed-size array in the library's own static device
// memory.
//
// The array is NOALLOC_SCRATCH_BYTES (32 MiB) per GPU, reserved on every device
// that loads the library until the process exits.  It holds one odd-parity
// FP64 spinor field, so the entry point accepts lattices with
// 4 * NF * (V/2 rounded up to 32) * 16 bytes <= 32 MiB (for example 16^3 x 32
// with NF = 3 needs 12.6 MB, with NF = 6 25.2 MB) and rejects larger ones with
// HRGPU_E_ARG.
//
// In host code the array's name is only a host-side stand-in, so its device
// address is looked up with cudaGetSymbolAddress once per device, with that
// device current, by the first call made on that device.  If no FP64 operator
// has run on the lattice yet, that first call also times the hopping-kernel
// variants (two CUDA events and a synchronisation, no device memory).  Make
// that first call before any stream capture.
//
// All calls share the one array and it keeps whatever the last call left
// there.  Nothing in it has to start at zero: the first hop writes every site
// the second hop reads.  Calls that overlap on the GPU (different streams, or
// different host threads driving the same device) race on the array; callers
// must order them.
#include "dirac.cuh"

namespace hrgpu {

constexpr size_t NOALLOC_SCRATCH_BYTES = 32u << 20;

static __device__ __align__(256) double2 g_noalloc_scratch[NOALLOC_SCRATCH_BYTES / sizeof(double2)];

constexpr int MAX_DEVICES = 64;
static void *g_scratch_addr[MAX_DEVICES] = {nullptr};

// The lookup is made with the library's own device current (the one its
// stream and lattice live on): a caller whose framework left another device
// current is refused, rather than handed an address on the wrong GPU (or a
// second 32 MiB reservation on it).
static int scratch_address(void **p) {
  int dev = -1;
  HR_CUDA(cudaGetDevice(&dev));
  HR_REQUIRE(dev == library_device(), HRGPU_E_STATE,
             "Dphi_eopre_noalloc: device %d is current, but the library runs on device %d (make it current first)",
             dev, library_device());
  HR_REQUIRE(dev >= 0 && dev < MAX_DEVICES, HRGPU_E_ARG, "Dphi_eopre_noalloc: device %d out of range", dev);
  if (!g_scratch_addr[dev]) {
    void *a = nullptr;
    HR_CUDA(cudaGetSymbolAddress(&a, g_noalloc_scratch));
    g_scratch_addr[dev] = a;
  }
  *p = g_scratch_addr[dev];
  return 0;
}

}  // namespace hrgpu

using namespace hrgpu;

extern "C" {

int hrgpu_Dphi_eopre_noalloc(double m0, void *out, const void *in) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "Dphi_eopre_noalloc: lattice not initialised");
  const size_t need = spinor_bytes(HRGPU_ODD, HRGPU_DOUBLE);
  HR_REQUIRE(need <= NOALLOC_SCRATCH_BYTES, HRGPU_E_ARG,
             "Dphi_eopre_noalloc: the odd temporary needs %zu bytes, more than the %zu-byte static scratch", need,
             NOALLOC_SCRATCH_BYTES);
  if (int rc = check_gauge(HRGPU_DOUBLE)) return rc;
  HR_REQUIRE(out && in && out != in, HRGPU_E_ARG, "Dphi_eopre_noalloc: input and output fields must be different");
  void *tmp = nullptr;
  if (int rc = scratch_address(&tmp)) return rc;
  if (int rc = hop<double>(HRGPU_ODD, tmp, in, EP_AXPY, -0.5, nullptr, 0.0, 0, nullptr, nullptr, nullptr)) return rc;
  const double rho = (4.0 + m0) * (4.0 + m0);
  return hop<double>(HRGPU_EVEN, out, tmp, EP_AXPY, 0.5, in, rho, 0, nullptr, nullptr, nullptr);
}

}  // extern "C"
