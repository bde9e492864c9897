// represent.cu -- gauge field in the fermion representation on the device
// (LibHR/Update/representation.c:16-200 _group_represent2 and :391-468
// represent_gauge_field), followed by the antiperiodic-T link sign
// (LibHR/Utils/boundary_conditions.c:321-341), the float copy and the clover term.
//
// The basis conventions are those of HiRep's explicit formulas, so the
// represented links agree element by element with the reference's u_gauge_f.
#include "dirac.cuh"

namespace hrgpu {

constexpr int MAXNG = 8;

// one link: u (NG x NG, complex) -> v (NF x NF) written to the link planes at (mu, d)
__global__ void k_represent(void *Uout, const double2 *Ug, int ng, int repr, Geo g, int bc_t_anti) {
  long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int mu = blockIdx.y;
  if (d >= 2L * g.ld) return;
  int p = d >= g.ld ? 1 : 0;
  if (d - p * g.ld >= g.VH) return;
  int t, x, y, z;
  dev_coords(g, (int)d, t, x, y, z);
  const long lp = 2L * g.ld;
  const int N = ng, N2 = ng * ng;
  double2 u[MAXNG * MAXNG], m[MAXNG * MAXNG];
  for (int k = 0; k < N2; k++) u[k] = Ug[((long)mu * N2 + k) * lp + d];
  const double sgn = (bc_t_anti && mu == 0 && t == 0) ? -1.0 : 1.0;
#define UG(a, b) u[(a) * N + (b)]
#define MF(a, b) m[(a) * N + (b)]
  auto cm = [](double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); };
  auto cmc = [](double2 a, double2 b) { return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); };  // a conj(b)
  if (repr == HRGPU_FUND) {
    double2 *v = (double2 *)Uout;
    for (int k = 0; k < N2; k++) v[((long)mu * N2 + k) * lp + d] = make_double2(sgn * u[k].x, sgn * u[k].y);
    return;
  }
  if (repr == HRGPU_ADJ) {
    const int F = N2 - 1;
    double *v = (double *)Uout;
    int A = 0;
    for (int a = 0; a < N; a++)
      for (int b = (a == 0) ? 1 : 0; b < N; b++) {
        for (int i = 0; i < N; i++)
          for (int j = i; j < N; j++) {
            if (a > b) {
              MF(i, j) = cadd(cmc(UG(i, a), UG(j, b)), cmc(UG(i, b), UG(j, a)));
            } else if (a < b) {
              double2 q1 = cmc(UG(i, a), UG(j, b)), q2 = cmc(UG(i, b), UG(j, a));
              // I*q1 - I*q2
              MF(i, j) = make_double2(-(q1.y - q2.y), q1.x - q2.x);
            } else {
              double2 q = cmc(UG(i, a), UG(j, a));
              double2 s = make_double2(-a * q.x, -a * q.y);
              for (int k = 0; k < a; k++) s = cadd(s, cmc(UG(i, k), UG(j, k)));
              double f = sqrt(2. / (a * (a + 1.)));
              MF(i, j) = make_double2(s.x * f, s.y * f);
            }
          }
        int C = 0;
        for (int c = 0; c < N; c++)
          for (int e = (c == 0) ? 1 : 0; e < N; e++) {
            double val;
            if (c > e) val = MF(e, c).x;
            else if (c < e) val = MF(c, e).y;
            else {
              val = -c * MF(c, c).x;
              for (int k = 0; k < c; k++) val += MF(k, k).x;
              val *= sqrt(.5 / (c * (c + 1.)));
            }
            v[((long)mu * F * F + C * F + A) * lp + d] = sgn * val;
            C++;
          }
        A++;
      }
    return;
  }
  double2 *v = (double2 *)Uout;
  if (repr == HRGPU_SYM) {
    const int F = N * (N + 1) / 2;
    const double st = sqrt(2.);
    int A = 0;
    for (int a = 0; a < N; a++) {
      for (int b = 0; b <= a; b++) {
        const bool diag = (b == a);
        for (int i = 0; i < N; i++)
          for (int j = i; j < N; j++)
            MF(i, j) = diag ? cm(UG(i, a), UG(j, a)) : cadd(cm(UG(i, a), UG(j, b)), cm(UG(i, b), UG(j, a)));
        int C = 0;
        for (int c = 0; c < N; c++) {
          for (int e = 0; e < c; e++) {
            double2 w = diag ? make_double2(MF(e, c).x * st, MF(e, c).y * st) : MF(e, c);
            v[((long)mu * F * F + C * F + A) * lp + d] = make_double2(sgn * w.x, sgn * w.y);
            C++;
          }
          double2 w = diag ? MF(c, c) : make_double2(MF(c, c).x / st, MF(c, c).y / st);
          v[((long)mu * F * F + C * F + A) * lp + d] = make_double2(sgn * w.x, sgn * w.y);
          C++;
        }
        A++;
      }
    }
    return;
  }
  // antisymmetric
  const int F = N * (N - 1) / 2;
  int A = 0;
  for (int a = 1; a < N; a++)
    for (int b = 0; b < a; b++) {
      for (int i = 0; i < N; i++)
        for (int j = i; j < N; j++) MF(i, j) = csub(cm(UG(i, a), UG(j, b)), cm(UG(i, b), UG(j, a)));
      int C = 0;
      for (int c = 1; c < N; c++)
        for (int e = 0; e < c; e++) {
          double2 w = MF(e, c);
          v[((long)mu * F * F + C * F + A) * lp + d] = make_double2(-sgn * w.x, -sgn * w.y);
          C++;
        }
      A++;
    }
#undef UG
#undef MF
}


// bad = 1 when row 2 of some link differs from s conj(r0 x r1) by more than tol
// (s = -1 on the links that carry the antiperiodic time sign); grid: sites of
// both parities x 4 directions
__global__ void k_check_row2(const double2 *U, Geo g, int bc, double tol, int *bad) {
  const long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (d >= 2L * g.ld) return;
  const int p = d >= g.ld ? 1 : 0, cb = (int)(d - (long)p * g.ld);
  if (cb >= g.VH) return;
  int t, x, y, z;
  cb_to_coords(g, cb, p, t, x, y, z);
  const long plane = 2L * g.ld;
  const double2 *Um = U + (long)mu * 9 * plane + d;
  double2 u[9];
  for (int e = 0; e < 9; e++) u[e] = Um[(long)e * plane];
  const double2 r6 = u[6], r7 = u[7], r8 = u[8];
  su3_row2(u, (bc && mu == 0 && t == 0) ? -1.0 : 1.0);
  double dev = fmax(fmax(fabs(u[6].x - r6.x), fabs(u[6].y - r6.y)), fmax(fabs(u[7].x - r7.x), fabs(u[7].y - r7.y)));
  dev = fmax(dev, fmax(fabs(u[8].x - r8.x), fabs(u[8].y - r8.y)));
  if (!(dev <= tol)) atomicOr(bad, 1);  // NaN counts as a mismatch
}

// the same for real links (SU(2) adjoint): row 2 against s (r0 x r1)
__global__ void k_check_row2_real(const double *U, Geo g, int bc, double tol, int *bad) {
  const long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (d >= 2L * g.ld) return;
  const int p = d >= g.ld ? 1 : 0, cb = (int)(d - (long)p * g.ld);
  if (cb >= g.VH) return;
  int t, x, y, z;
  cb_to_coords(g, cb, p, t, x, y, z);
  const long plane = 2L * g.ld;
  const double *Um = U + (long)mu * 9 * plane + d;
  double u[9];
  for (int e = 0; e < 9; e++) u[e] = Um[(long)e * plane];
  const double r6 = u[6], r7 = u[7], r8 = u[8];
  so3_row2(u, (bc && mu == 0 && t == 0) ? -1.0 : 1.0);
  const double dev = fmax(fabs(u[6] - r6), fmax(fabs(u[7] - r7), fabs(u[8] - r8)));
  if (!(dev <= tol)) atomicOr(bad, 1);  // NaN counts as a mismatch
}

// The hopping kernels may rebuild row 2 of the SU(3) fundamental or SU(2)
// adjoint links when every link passes the check at 1e-14 (unitary links of
// determinant 1, up to the boundary sign); otherwise they read the full links.
// For the NF = 6 two-index representations (SU(3) symmetric, SU(4)
// antisymmetric) the FP64 kernels may build the links from the fundamental ones
// (modes 3, and 4 with the antiperiodic sign) as long as the fundamental field
// is the one the represented field was made from: set by
// represent_gauge_field, cleared by whatever writes the fundamental links
// (fund_links_changed) or uploads represented links.
static int set_recon12(int bc, bool from_fund) {
  L.recon12 = 0;
  const bool two6 = !L.real && L.nf == 6 && ((L.repr == HRGPU_SYM && L.ng == 3) || (L.repr == HRGPU_ASYM && L.ng == 4));
  if (two6) {
    if (from_fund && L.Ug) L.recon12 = bc ? 4 : 3;
    return 0;
  }
  const bool su3 = !L.real && L.nf == 3 && L.ng == 3 && L.repr == HRGPU_FUND;
  const bool so3 = L.real && L.nf == 3 && L.ng == 2 && L.repr == HRGPU_ADJ;
  if (!su3 && !so3) return 0;
  static int *d_bad = nullptr;
  if (!d_bad) HR_CUDA(cudaMalloc(&d_bad, sizeof(int)));
  HR_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), L.stream));
  const long n = 2L * L.ld;
  const dim3 grid((unsigned)((n + 127) / 128), 4);
  if (su3)
    k_check_row2<<<grid, 128, 0, L.stream>>>((const double2 *)L.U, make_geo(), bc, 1e-14, d_bad);
  else
    k_check_row2_real<<<grid, 128, 0, L.stream>>>((const double *)L.U, make_geo(), bc, 1e-14, d_bad);
  HR_LAUNCH_CHECK();
  int bad = 1;
  HR_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, L.stream));
  HR_CUDA(cudaStreamSynchronize(L.stream));
  L.recon12 = bad ? 0 : (bc ? 2 : 1);
  return 0;
}

// links uploaded already represented (hrgpu_gauge_set_f): the boundary
// condition is not known, so try the antiperiodic sign, then none
int detect_recon12() {
  if (int rc = set_recon12(1, false)) return rc;
  if (L.recon12 == 0)
    if (int rc = set_recon12(0, false)) return rc;
  return 0;
}

void fund_links_changed() {
  if (L.recon12 >= 3) L.recon12 = 0;
}

}  // namespace hrgpu

using namespace hrgpu;

extern "C" {

int hrgpu_link_recon(int *mode) {
  HR_REQUIRE(mode, HRGPU_E_ARG, "link_recon: NULL argument");
  *mode = L.recon_allow ? L.recon12 : 0;
  return 0;
}

int hrgpu_set_link_recon(int on) {
  L.recon_allow = on != 0;
  return 0;
}

int hrgpu_represent_gauge_field(int bc_t_antiperiodic) {
  HR_REQUIRE(L.ready && L.have_fund, HRGPU_E_STATE, "represent_gauge_field: no fundamental gauge field (hrgpu_gauge_set)");
  HR_REQUIRE(L.ng <= MAXNG, HRGPU_E_ARG, "represent_gauge_field: NG=%d > %d", L.ng, MAXNG);
  int nel = L.nf * L.nf;
  size_t esz = L.real ? sizeof(double) : sizeof(double2);
  if (!L.U) HR_CUDA(cudaMalloc(&L.U, (size_t)4 * nel * 2 * L.ld * esz));
  Geo g = make_geo();
  long n = 2L * L.ld;
  k_represent<<<dim3((unsigned)((n + 127) / 128), 4), 128, 0, L.stream>>>(L.U, L.Ug, L.ng, L.repr, g, bc_t_antiperiodic);
  HR_LAUNCH_CHECK();
  L.have_gauge = true;
  L.bc_t = bc_t_antiperiodic;
  if (int rc = set_recon12(bc_t_antiperiodic, true)) return rc;
  if (int rc = hrgpu_assign_ud2u_f()) return rc;
  if (L.clover) {
    if (int rc = compute_clover_term_dev()) return rc;
  }
  L.sigma = L.sigma_diag = L.sigma_flt = 0xF00F;
  return 0;
}

}  // extern "C"
