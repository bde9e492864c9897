// io.cu -- gauge configurations in HiRep's file format, read into and written
// from the device layout (LibHR/IO/archive.c:26-457, archive_su2quat.c).
//
// File: 5 big-endian int32 (NG, T, X, Y, Z), one big-endian double (the average
// plaquette, a checksum), then for t, x, y, z (z fastest) the four links mu =
// 0..3 of the site: NG x NG complex numbers row by row as (re, im) big-endian
// doubles, or for NG = 2 the quaternion (q0, q1, q2, q3) of
//   | q0 + i q3   -q2 + i q1 |
//   | q2 + i q1    q0 - i q3 |   (archive_su2quat.c:33-58).
// The reader of SU(2) files accepts both forms (matrix form: the file has the
// matrix size and the first link's rows are orthonormal, archive_su2quat.c:
// 500-512).  The file order is the coordinate order, so the links are gathered
// from / scattered to the device layout by coordinates on the device; the
// byte order is swapped on the host.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <vector>

#include "dirac.cuh"

namespace hrgpu {

// file site f = ((t*X + x)*Y + y)*Z + z  <->  device site p*ld + cb
__device__ __forceinline__ long file_to_dev(const Geo &g, long f) {
  const int z = (int)(f % g.Z);
  long r = f / g.Z;
  const int y = (int)(r % g.Y);
  r /= g.Y;
  const int x = (int)(r % g.X);
  const int t = (int)(r / g.X);
  return (long)((t + x + y + z) & 1) * g.ld + coords_to_cb(g, t, x, y, z);
}

// gather: out[f][mu][k] (k < NG*NG complex, or 4 quaternion doubles for quat)
__global__ void k_links_to_file(double *out, const double2 *Ug, Geo g, int n2, int quat) {
  const long V = 2L * g.VH;
  const long lp = 2L * g.ld;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < 4 * V; i += (long)gridDim.x * blockDim.x) {
    const long f = i / 4;
    const int mu = (int)(i % 4);
    const long d = file_to_dev(g, f);
    const double2 *u = Ug + (long)mu * n2 * lp + d;
    if (quat) {  // translate_su2_quat (the symmetrised form)
      const double2 c0 = u[0], c1 = u[lp], c2 = u[2 * lp], c3 = u[3 * lp];
      double *q = out + i * 4;
      q[0] = (c0.x + c3.x) / 2.;
      q[1] = (c1.y + c2.y) / 2.;
      q[2] = (c2.x - c1.x) / 2.;
      q[3] = (c0.y - c3.y) / 2.;
    } else {
      double *m = out + i * 2 * n2;
      for (int k = 0; k < n2; k++) {
        const double2 v = u[(long)k * lp];
        m[2 * k] = v.x;
        m[2 * k + 1] = v.y;
      }
    }
  }
}

__global__ void k_file_to_links(double2 *Ug, const double *in, Geo g, int n2, int quat) {
  const long V = 2L * g.VH;
  const long lp = 2L * g.ld;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < 4 * V; i += (long)gridDim.x * blockDim.x) {
    const long f = i / 4;
    const int mu = (int)(i % 4);
    const long d = file_to_dev(g, f);
    double2 *u = Ug + (long)mu * n2 * lp + d;
    if (quat) {  // translate_quat_su2
      const double *q = in + i * 4;
      u[0] = make_double2(q[0], q[3]);
      u[lp] = make_double2(-q[2], q[1]);
      u[2 * lp] = make_double2(q[2], q[1]);
      u[3 * lp] = make_double2(q[0], -q[3]);
    } else {
      const double *m = in + i * 2 * n2;
      for (int k = 0; k < n2; k++) u[(long)k * lp] = make_double2(m[2 * k], m[2 * k + 1]);
    }
  }
}

static void bswap_doubles(double *p, size_t n) {
  for (size_t i = 0; i < n; i++) {
    uint64_t v;
    memcpy(&v, p + i, 8);
    v = __builtin_bswap64(v);
    memcpy(p + i, &v, 8);
  }
}
static void bswap_ints(int32_t *p, size_t n) {
  for (size_t i = 0; i < n; i++) p[i] = (int32_t)__builtin_bswap32((uint32_t)p[i]);
}

static unsigned io_grid(long n) {
  long b = (n + 255) / 256;
  return (unsigned)(b < 148L * 8 ? b : 148L * 8);
}

}  // namespace hrgpu

using namespace hrgpu;

extern "C" {

int hrgpu_avr_plaquette(double *plaq);

int hrgpu_write_gauge_field(const char *filename) {
  HR_REQUIRE(L.ready && L.have_fund, HRGPU_E_STATE, "write_gauge_field: no fundamental gauge field");
  HR_REQUIRE(filename, HRGPU_E_ARG, "write_gauge_field: NULL file name");
  double plaq = 0;
  if (int rc = hrgpu_avr_plaquette(&plaq)) return rc;
  const int quat = L.ng == 2;
  const int n2 = L.ng * L.ng;
  const size_t per_link = quat ? 4 : 2 * n2;
  const size_t nd = (size_t)4 * L.V * per_link;
  double *dbuf = nullptr;
  HR_CUDA(cudaMalloc(&dbuf, nd * sizeof(double)));
  const Geo g = make_geo();
  k_links_to_file<<<io_grid(4L * L.V), 256, 0, L.stream>>>(dbuf, L.Ug, g, n2, quat);
  cudaError_t e = cudaGetLastError();
  std::vector<double> h(nd);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), dbuf, nd * sizeof(double), cudaMemcpyDeviceToHost, L.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(L.stream);
  cudaFree(dbuf);
  if (e != cudaSuccess) return fail_cuda(e, "write_gauge_field gather", __FILE__, __LINE__);
  FILE *fp = fopen(filename, "wb");
  HR_REQUIRE(fp, HRGPU_E_ARG, "write_gauge_field: cannot open %s for writing", filename);
  int32_t d[5] = {L.ng, L.T, L.X, L.Y, L.Z};
  bswap_ints(d, 5);
  double p = plaq;
  bswap_doubles(&p, 1);
  bswap_doubles(h.data(), nd);
  const bool ok = fwrite(d, sizeof(int32_t), 5, fp) == 5 && fwrite(&p, sizeof(double), 1, fp) == 1 &&
                  fwrite(h.data(), sizeof(double), nd, fp) == nd;
  const bool closed = fclose(fp) == 0;
  HR_REQUIRE(ok && closed, HRGPU_E_ARG, "write_gauge_field: write to %s failed", filename);
  return 0;
}

// plaq_file: the plaquette stored in the header; plaq_read: the plaquette of the
// links read (the reference warns when they differ by more than 1e-12).
int hrgpu_read_gauge_field(const char *filename, double *plaq_file, double *plaq_read) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "read_gauge_field: lattice not initialised");
  HR_REQUIRE(filename, HRGPU_E_ARG, "read_gauge_field: NULL file name");
  FILE *fp = fopen(filename, "rb");
  HR_REQUIRE(fp, HRGPU_E_ARG, "read_gauge_field: cannot open %s", filename);
  fseek(fp, 0, SEEK_END);
  const long fsize = ftell(fp);
  fseek(fp, 0, SEEK_SET);
  int32_t d[5];
  double p = 0;
  const bool hdr = fread(d, sizeof(int32_t), 5, fp) == 5 && fread(&p, sizeof(double), 1, fp) == 1;
  if (!hdr) {
    fclose(fp);
    HR_REQUIRE(false, HRGPU_E_ARG, "read_gauge_field: %s: short header", filename);
  }
  bswap_ints(d, 5);
  bswap_doubles(&p, 1);
  if (d[0] != L.ng || d[1] != L.T || d[2] != L.X || d[3] != L.Y || d[4] != L.Z) {
    fclose(fp);
    set_error("read_gauge_field: %s holds NG=%d %dx%dx%dx%d, the lattice is NG=%d %dx%dx%dx%d", filename, d[0], d[1],
              d[2], d[3], d[4], L.ng, L.T, L.X, L.Y, L.Z);
    return HRGPU_E_ARG;
  }
  const int n2 = L.ng * L.ng;
  const long header = 5 * sizeof(int32_t) + sizeof(double);
  const long matrix_size = header + (long)4 * L.V * 2 * n2 * sizeof(double);
  int quat = 0;
  if (L.ng == 2) {
    // archive_su2quat.c:500-512: the matrix form has the matrix size and
    // orthonormal rows in its first link
    double b[8];
    const bool got = fread(b, sizeof(double), 8, fp) == 8;
    bswap_doubles(b, 8);
    const bool matrix = got && fsize == matrix_size && fabs(b[0] * b[4] + b[1] * b[5] + b[2] * b[6] + b[3] * b[7]) < 1e-10 &&
                        fabs(b[0] * b[5] - b[4] * b[1] + b[2] * b[7] - b[6] * b[3]) < 1e-10;
    quat = matrix ? 0 : 1;
    fseek(fp, header, SEEK_SET);
  }
  const size_t per_link = quat ? 4 : 2 * n2;
  const size_t nd = (size_t)4 * L.V * per_link;
  if ((long)(header + nd * sizeof(double)) != fsize) {
    fclose(fp);
    set_error("read_gauge_field: %s has %ld bytes, %ld expected", filename, fsize, (long)(header + nd * sizeof(double)));
    return HRGPU_E_ARG;
  }
  std::vector<double> h(nd);
  const bool body = fread(h.data(), sizeof(double), nd, fp) == nd;
  fclose(fp);
  HR_REQUIRE(body, HRGPU_E_ARG, "read_gauge_field: %s: short body", filename);
  bswap_doubles(h.data(), nd);
  if (!L.Ug) {
    HR_CUDA(cudaMalloc(&L.Ug, sizeof(double2) * 4 * n2 * 2 * L.ld));
    HR_CUDA(cudaMemsetAsync(L.Ug, 0, sizeof(double2) * 4 * n2 * 2 * L.ld, L.stream));  // padding sites
  }
  double *dbuf = nullptr;
  HR_CUDA(cudaMalloc(&dbuf, nd * sizeof(double)));
  cudaError_t e = cudaMemcpyAsync(dbuf, h.data(), nd * sizeof(double), cudaMemcpyHostToDevice, L.stream);
  const Geo g = make_geo();
  if (e == cudaSuccess) {
    k_file_to_links<<<io_grid(4L * L.V), 256, 0, L.stream>>>(L.Ug, dbuf, g, n2, quat);
    e = cudaGetLastError();
    fund_links_changed();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(L.stream);
  cudaFree(dbuf);
  if (e != cudaSuccess) return fail_cuda(e, "read_gauge_field scatter", __FILE__, __LINE__);
  L.have_fund = true;
  double now = 0;
  if (int rc = hrgpu_avr_plaquette(&now)) return rc;
  if (plaq_file) *plaq_file = p;
  if (plaq_read) *plaq_read = now;
  return 0;
}

}  // extern "C"
