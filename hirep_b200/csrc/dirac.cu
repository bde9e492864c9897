// dirac.cu -- Wilson / clover Dirac operators on the device (LibHR/Update/Dphi.c,
// Dphi_flt.c, D_update.c), built from the fused hopping kernel in hop.cuh.
#include "dirac.cuh"

namespace hrgpu {

template <typename R, int EP>
int launch_ep(HopArgs<R> &a);  // hop_launch.cuh, instantiated in dirac_{d,f}_ep*.cu

template <typename R>
int launch_hop(int ep, HopArgs<R> &a) {
  if (ep == EP_AXPY) return launch_ep<R, EP_AXPY>(a);
  if (ep == EP_CLOV_INV) return launch_ep<R, EP_CLOV_INV>(a);
  return launch_ep<R, EP_CLOV>(a);
}
template int launch_hop<double>(int, HopArgs<double> &);
template int launch_hop<float>(int, HopArgs<float> &);

static unsigned long g_mvm = 0;
static double g_static_mass = 0.0;

template <typename R>
static const void *links() {
  if (sizeof(R) == 8) return L.U;
  return L.flt_links == HRGPU_LINKS_BF16 ? L.Ubf : L.Uf;
}

// one hop onto parity outp with the given epilogue; fields are parity fields
template <typename R>
int hop(int outp, void *out, const void *in, int ep, double cacc, const void *aux, double caux, int g5, double *red,
        const R *cdg, const typename C2<R>::T *cod, int cb0, int cb1) {
  HopArgs<R> a;
  a.cb0 = cb0;
  a.cb1 = cb1 < 0 ? (int)L.VH : cb1;
  if (a.cb1 <= a.cb0) return 0;
  a.in = in;
  a.out = out;
  a.U = links<R>();
  a.aux = aux;
  a.cdg = cdg;
  a.cod = cod;
  a.red = red;
  a.cacc = (R)cacc;
  a.caux = (R)caux;
  a.outp = outp;
  a.g5 = g5;
  a.stop = L.cur_stop;
  a.err = nullptr;
  a.Ug = sizeof(R) == 8 ? (const void *)L.Ug : (const void *)L.Ugf;
  if (sizeof(R) == 4 && L.flt_links == HRGPU_LINKS_BF16) {
    if (int rc = ensure_links_bf16()) return rc;
    a.U = L.Ubf;
  }
  if (a.cb0 == 0 && a.cb1 == (int)L.VH) g_mvm++;  // partial launches are counted by their caller
  return launch_hop<R>(ep, a);
}
template int hop<double>(int, void *, const void *, int, double, const void *, double, int, double *, const double *,
                         const double2 *, int, int);
template int hop<float>(int, void *, const void *, int, double, const void *, double, int, double *, const float *,
                        const float2 *, int, int);

int check_gauge(int prec) {
  HR_REQUIRE(L.ready, HRGPU_E_STATE, "lattice not initialised");
  if (prec == HRGPU_DOUBLE) HR_REQUIRE(L.have_gauge, HRGPU_E_STATE, "no gauge field set");
  else HR_REQUIRE(L.have_gauge_flt, HRGPU_E_STATE, "no float gauge field set");
  return 0;
}

template <typename R>
static size_t par_elems() {
  return (size_t)4 * L.nf * L.ld;  // complex elements of one parity field
}

template <typename R>
static inline void *par_ptr(void *f, int p) {
  return (char *)f + (size_t)p * par_elems<R>() * sizeof(typename C2<R>::T);
}
template <typename R>
static inline const void *par_ptr(const void *f, int p) {
  return (const char *)f + (size_t)p * par_elems<R>() * sizeof(typename C2<R>::T);
}

// Dphi_ on parity or full fields
template <typename R>
int Dphi_hop(void *out, int out_par, const void *in) {
  if (int rc = check_gauge(sizeof(R) == 8 ? HRGPU_DOUBLE : HRGPU_FLOAT)) return rc;
  HR_REQUIRE(out && in && out != in, HRGPU_E_ARG, "Dphi_: input and output fields must be different");
  HR_REQUIRE(out_par >= 0 && out_par <= 2, HRGPU_E_ARG, "Dphi_: bad parity");
  if (out_par == HRGPU_FULL) {
    for (int p = 0; p < 2; p++)
      if (int rc = hop<R>(p, par_ptr<R>(out, p), par_ptr<R>(in, p ^ 1), EP_AXPY, -0.5, nullptr, 0.0, 0, nullptr,
                          nullptr, nullptr))
        return rc;
    g_mvm++;  // a full-lattice application counts twice (Dphi.c:205-207)
    return 0;
  }
  return hop<R>(out_par, out, in, EP_AXPY, -0.5, nullptr, 0.0, 0, nullptr, nullptr, nullptr);
}

// full lattice: out = -1/2 H in + (4+m) in, optionally gamma_5 (Dphi / g5Dphi)
template <typename R>
int Dphi_full(double m0, void *out, const void *in, int g5) {
  if (int rc = check_gauge(sizeof(R) == 8 ? HRGPU_DOUBLE : HRGPU_FLOAT)) return rc;
  HR_REQUIRE(out && in && out != in, HRGPU_E_ARG, "Dphi: input and output fields must be different");
  for (int p = 0; p < 2; p++)
    if (int rc = hop<R>(p, par_ptr<R>(out, p), par_ptr<R>(in, p ^ 1), EP_AXPY, -0.5, par_ptr<R>(in, p), 4.0 + m0, g5,
                        nullptr, nullptr, nullptr))
      return rc;
  return 0;
}

// one hop of an even-odd preconditioned operator with output parity p, on the
// output sites cb0 <= cb < cb1 of its parity:
//   stage 0: tmp = D_qp in on parity q = 1-p (clover: times D_qq^-1)
//   stage 1: out = rho in + 1/2 D_pq tmp with rho = (4+m)^2 (Wilson), or
//            D_pp in + 1/2 D_pq tmp (clover), optionally times gamma_5.
// Stage 1 on a range needs stage 0 done on the neighbouring range (one site
// further in every direction).
template <typename R>
int eo_stage(int clover, double mass, int stage, int outp, void *out, const void *in, int g5, double *red, int cb0,
             int cb1) {
  void **tmp = sizeof(R) == 8 ? &L.tmp_o : &L.tmp_o_f;
  if (int rc = ensure_tmp(tmp, spinor_bytes(HRGPU_EVEN, sizeof(R) == 8 ? HRGPU_DOUBLE : HRGPU_FLOAT))) return rc;
  if (clover) {
    const R *idg, *ddg;
    const typename C2<R>::T *iod, *dod;
    clover_blocks<R>(&ddg, &dod, &idg, &iod);
    if (stage == 0) return hop<R>(outp ^ 1, *tmp, in, EP_CLOV_INV, -0.5, nullptr, 0.0, 0, nullptr, idg, iod, cb0, cb1);
    return hop<R>(outp, out, *tmp, EP_CLOV, 0.5, in, 0.0, g5, red, ddg, dod, cb0, cb1);
  }
  if (stage == 0) return hop<R>(outp ^ 1, *tmp, in, EP_AXPY, -0.5, nullptr, 0.0, 0, nullptr, nullptr, nullptr, cb0, cb1);
  double rho = 4.0 + mass;
  if (sizeof(R) == 4) {
    float r = 4.f + (float)mass;
    rho = (double)(r * r);
  } else {
    rho = rho * rho;
  }
  return hop<R>(outp, out, *tmp, EP_AXPY, 0.5, in, rho, g5, red, nullptr, nullptr, cb0, cb1);
}
template int eo_stage<double>(int, double, int, int, void *, const void *, int, double *, int, int);
template int eo_stage<float>(int, double, int, int, void *, const void *, int, double *, int, int);

// even-odd: out = (4+m)^2 in - D_pq D_qp in on parity p, optionally gamma_5
template <typename R>
int Dphi_eo(double m0, void *out, const void *in, int outp, int g5, double *red) {
  if (int rc = check_gauge(sizeof(R) == 8 ? HRGPU_DOUBLE : HRGPU_FLOAT)) return rc;
  HR_REQUIRE(out && in && out != in, HRGPU_E_ARG, "Dphi_eopre: input and output fields must be different");
  if (int rc = eo_stage<R>(0, m0, 0, outp, out, in, g5, nullptr, 0, -1)) return rc;
  return eo_stage<R>(0, m0, 1, outp, out, in, g5, red, 0, -1);
}

template int Dphi_eo<double>(double, void *, const void *, int, int, double *);
template int Dphi_eo<float>(double, void *, const void *, int, int, double *);

// ------------------------------------------------------------------ clover
template <typename R>
int Cphi_eo(double mass, void *out, const void *in, int g5, double *red) {
  if (int rc = check_gauge(sizeof(R) == 8 ? HRGPU_DOUBLE : HRGPU_FLOAT)) return rc;
  HR_REQUIRE(L.clover, HRGPU_E_STATE, "Cphi_eopre: no clover term (hrgpu_clover_init)");
  HR_REQUIRE(out && in && out != in, HRGPU_E_ARG, "Cphi_eopre: input and output fields must be different");
  if (int rc = clover_prepare(mass, sizeof(R) == 8 ? HRGPU_DOUBLE : HRGPU_FLOAT)) return rc;
  if (int rc = eo_stage<R>(1, mass, 0, HRGPU_EVEN, out, in, g5, nullptr, 0, -1)) return rc;
  return eo_stage<R>(1, mass, 1, HRGPU_EVEN, out, in, g5, red, 0, -1);
}
template int Cphi_eo<double>(double, void *, const void *, int, double *);
template int Cphi_eo<float>(double, void *, const void *, int, double *);

static int Cphi_full(double mass, void *out, const void *in, int g5) {
  if (int rc = check_gauge(HRGPU_DOUBLE)) return rc;
  HR_REQUIRE(L.clover, HRGPU_E_STATE, "Cphi: no clover term (hrgpu_clover_init)");
  HR_REQUIRE(out && in && out != in, HRGPU_E_ARG, "Cphi: input and output fields must be different");
  if (int rc = clover_prepare(mass, HRGPU_DOUBLE)) return rc;
  const double *idg, *ddg;
  const double2 *iod, *dod;
  clover_blocks<double>(&ddg, &dod, &idg, &iod);
  for (int p = 0; p < 2; p++)
    if (int rc = hop<double>(p, par_ptr<double>(out, p), par_ptr<double>(in, p ^ 1), EP_CLOV, -0.5,
                             par_ptr<double>(in, p), 0.0, g5, nullptr, ddg, dod))
      return rc;
  return 0;
}

template <typename R>
static int sq(int (*op)(double, void *, const void *, int), double m, void *out, const void *in, int par) {
  void **tmp = par == HRGPU_FULL ? (sizeof(R) == 8 ? &L.tmp_full : &L.tmp_full_f) : (sizeof(R) == 8 ? &L.tmp_e : &L.tmp_e_f);
  if (int rc = ensure_tmp(tmp, spinor_bytes(par, sizeof(R) == 8 ? HRGPU_DOUBLE : HRGPU_FLOAT))) return rc;
  if (int rc = op(m, *tmp, in, 1)) return rc;
  return op(m, out, *tmp, 1);
}

static int op_Dfull_d(double m, void *o, const void *i, int g5) { return Dphi_full<double>(m, o, i, g5); }
static int op_Dfull_f(double m, void *o, const void *i, int g5) { return Dphi_full<float>(m, o, i, g5); }
static int op_eo_d(double m, void *o, const void *i, int g5) { return Dphi_eo<double>(m, o, i, HRGPU_EVEN, g5, nullptr); }
static int op_eo_f(double m, void *o, const void *i, int g5) { return Dphi_eo<float>(m, o, i, HRGPU_EVEN, g5, nullptr); }
static int op_ceo_d(double m, void *o, const void *i, int g5) { return Cphi_eo<double>(m, o, i, g5, nullptr); }
static int op_ceo_f(double m, void *o, const void *i, int g5) { return Cphi_eo<float>(m, o, i, g5, nullptr); }
static int op_cfull_d(double m, void *o, const void *i, int g5) { return Cphi_full(m, o, i, g5); }

// operator used by the inverters: M = op(mass) on fields of the returned parity
int apply_op(int op, int prec, double mass, void *out, const void *in) {
  if (prec == HRGPU_DOUBLE) {
    switch (op) {
      case HRGPU_OP_G5DPHI_SQ: return sq<double>(op_Dfull_d, mass, out, in, HRGPU_FULL);
      case HRGPU_OP_G5DPHI_EOPRE_SQ: return sq<double>(op_eo_d, mass, out, in, HRGPU_EVEN);
      case HRGPU_OP_G5CPHI_EOPRE_SQ: return sq<double>(op_ceo_d, mass, out, in, HRGPU_EVEN);
      case HRGPU_OP_G5CPHI_SQ: return sq<double>(op_cfull_d, mass, out, in, HRGPU_FULL);
      case HRGPU_OP_DPHI_EOPRE: return op_eo_d(mass, out, in, 0);
      case HRGPU_OP_G5DPHI_EOPRE: return op_eo_d(mass, out, in, 1);
      case HRGPU_OP_CPHI_EOPRE: return op_ceo_d(mass, out, in, 0);
      case HRGPU_OP_G5CPHI_EOPRE: return op_ceo_d(mass, out, in, 1);
      case HRGPU_OP_DPHI: return op_Dfull_d(mass, out, in, 0);
      case HRGPU_OP_CPHI: return op_cfull_d(mass, out, in, 0);
    }
  } else {
    switch (op) {
      case HRGPU_OP_G5DPHI_SQ: return sq<float>(op_Dfull_f, mass, out, in, HRGPU_FULL);
      case HRGPU_OP_G5DPHI_EOPRE_SQ: return sq<float>(op_eo_f, mass, out, in, HRGPU_EVEN);
      case HRGPU_OP_G5CPHI_EOPRE_SQ: return sq<float>(op_ceo_f, mass, out, in, HRGPU_EVEN);
      default: break;
    }
  }
  set_error("operator %d has no %s version", op, prec == HRGPU_DOUBLE ? "double" : "float");
  return HRGPU_E_ARG;
}

// The even-odd H^2 (op G5DPHI_EOPRE_SQ or G5CPHI_EOPRE_SQ), the same launches
// as apply_op, with the |H in|^2 partial sums of the first H application (one
// per block of its last hop) in red[0 .. *nblocks): with H Hermitian,
// <in, H^2 in> = |H in|^2, the CG's alpha without a dot-product pass.
// Returns -1 when op has no such form (the caller takes the dot product), else
// 0 or an error status.
template <typename R>
static int sq_eo_sqnorm(bool clover, double m, void *out, const void *in, double *red, int *nblocks) {
  void **tmp = sizeof(R) == 8 ? &L.tmp_e : &L.tmp_e_f;
  if (int rc = ensure_tmp(tmp, spinor_bytes(HRGPU_EVEN, sizeof(R) == 8 ? HRGPU_DOUBLE : HRGPU_FLOAT))) return rc;
  if (int rc = clover ? Cphi_eo<R>(m, *tmp, in, 1, red) : Dphi_eo<R>(m, *tmp, in, HRGPU_EVEN, 1, red)) return rc;
  // the block count of the variant that ran (tuned now if it was the first launch)
  const int pi = sizeof(R) == 8 ? 0 : (L.flt_links == HRGPU_LINKS_BF16 ? 2 : 1);
  const int ep = clover ? EP_CLOV : EP_AXPY;
  const int v = L.hop_force >= 0 ? L.hop_force : L.hop_variant[pi][ep];
  const long threads = hop_threads_per_site(v) * (long)L.VH;
  *nblocks = (int)((threads + HOP_THREADS - 1) / HOP_THREADS);
  return clover ? Cphi_eo<R>(m, out, *tmp, 1, nullptr) : Dphi_eo<R>(m, out, *tmp, HRGPU_EVEN, 1, nullptr);
}

int apply_op_sqnorm(int op, int prec, double mass, void *out, const void *in, double *red, int *nblocks) {
  if (op != HRGPU_OP_G5DPHI_EOPRE_SQ && op != HRGPU_OP_G5CPHI_EOPRE_SQ) return -1;
  const bool clover = op == HRGPU_OP_G5CPHI_EOPRE_SQ;
  return prec == HRGPU_DOUBLE ? sq_eo_sqnorm<double>(clover, mass, out, in, red, nblocks)
                              : sq_eo_sqnorm<float>(clover, mass, out, in, red, nblocks);
}

int op_parity(int op) {
  return (op == HRGPU_OP_G5DPHI_SQ || op == HRGPU_OP_G5CPHI_SQ || op == HRGPU_OP_DPHI || op == HRGPU_OP_CPHI)
             ? HRGPU_FULL
             : HRGPU_EVEN;
}

double static_mass() { return g_static_mass; }

void add_mvm(unsigned long n) { g_mvm += n; }
unsigned long mvm_count() { return g_mvm; }
void mvm_restore(unsigned long n) { g_mvm = n; }

}  // namespace hrgpu

using namespace hrgpu;

extern "C" {

int hrgpu_Dphi_(void *out, int out_par, const void *in) { return Dphi_hop<double>(out, out_par, in); }
int hrgpu_Dphi(double m0, void *out, const void *in) { return Dphi_full<double>(m0, out, in, 0); }
int hrgpu_g5Dphi(double m0, void *out, const void *in) { return Dphi_full<double>(m0, out, in, 1); }
int hrgpu_g5Dphi_sq(double m0, void *out, const void *in) { return sq<double>(op_Dfull_d, m0, out, in, HRGPU_FULL); }
int hrgpu_Dphi_eopre(double m0, void *out, const void *in) { return Dphi_eo<double>(m0, out, in, HRGPU_EVEN, 0, nullptr); }
int hrgpu_Dphi_oepre(double m0, void *out, const void *in) { return Dphi_eo<double>(m0, out, in, HRGPU_ODD, 0, nullptr); }
int hrgpu_g5Dphi_eopre(double m0, void *out, const void *in) { return Dphi_eo<double>(m0, out, in, HRGPU_EVEN, 1, nullptr); }
int hrgpu_g5Dphi_eopre_sq(double m0, void *out, const void *in) { return sq<double>(op_eo_d, m0, out, in, HRGPU_EVEN); }

int hrgpu_Dphi_flt_(void *out, int out_par, const void *in) { return Dphi_hop<float>(out, out_par, in); }
int hrgpu_Dphi_flt(double m0, void *out, const void *in) { return Dphi_full<float>(m0, out, in, 0); }
int hrgpu_g5Dphi_flt(double m0, void *out, const void *in) { return Dphi_full<float>(m0, out, in, 1); }
int hrgpu_g5Dphi_sq_flt(double m0, void *out, const void *in) { return sq<float>(op_Dfull_f, m0, out, in, HRGPU_FULL); }
int hrgpu_Dphi_eopre_flt(double m0, void *out, const void *in) { return Dphi_eo<float>(m0, out, in, HRGPU_EVEN, 0, nullptr); }
int hrgpu_g5Dphi_eopre_flt(double m0, void *out, const void *in) { return Dphi_eo<float>(m0, out, in, HRGPU_EVEN, 1, nullptr); }
int hrgpu_g5Dphi_eopre_sq_flt(double m0, void *out, const void *in) { return sq<float>(op_eo_f, m0, out, in, HRGPU_EVEN); }

int hrgpu_set_hop_variant(int variant) {
  HR_REQUIRE(variant >= -1 && variant < HOP_VARIANTS, HRGPU_E_ARG, "set_hop_variant: variant must be -1..%d",
             HOP_VARIANTS - 1);
  L.hop_force = variant;
  return 0;
}

int hrgpu_hop_tuning(int prec, int epilogue, int *chosen, float *ms) {
  HR_REQUIRE(prec >= 0 && prec <= 2 && epilogue >= 0 && epilogue <= 2 && chosen && ms, HRGPU_E_ARG,
             "hop_tuning: bad arguments");
  *chosen = L.hop_variant[prec][epilogue];
  for (int v = 0; v < HOP_VARIANTS; v++) ms[v] = L.hop_tune_ms[prec][epilogue][v];
  return 0;
}

int hrgpu_set_hop_pdl(int on) {
  L.hop_pdl = on != 0;
  return 0;
}

unsigned long hrgpu_getMVM(void) {
  unsigned long r = g_mvm >> 1;
  g_mvm = 0;
  return r;
}

int hrgpu_Cphi(double mass, void *out, const void *in) { return Cphi_full(mass, out, in, 0); }
int hrgpu_g5Cphi(double mass, void *out, const void *in) { return Cphi_full(mass, out, in, 1); }
int hrgpu_g5Cphi_sq(double mass, void *out, const void *in) { return sq<double>(op_cfull_d, mass, out, in, HRGPU_FULL); }
int hrgpu_Cphi_eopre(double mass, void *out, const void *in) { return Cphi_eo<double>(mass, out, in, 0, nullptr); }
int hrgpu_g5Cphi_eopre(double mass, void *out, const void *in) { return Cphi_eo<double>(mass, out, in, 1, nullptr); }
int hrgpu_g5Cphi_eopre_sq(double mass, void *out, const void *in) { return sq<double>(op_ceo_d, mass, out, in, HRGPU_EVEN); }
int hrgpu_g5Cphi_eopre_flt(double mass, void *out, const void *in) { return Cphi_eo<float>(mass, out, in, 1, nullptr); }
int hrgpu_g5Cphi_eopre_sq_flt(double mass, void *out, const void *in) { return sq<float>(op_ceo_f, mass, out, in, HRGPU_EVEN); }

int hrgpu_set_flt_link_storage(int kind) {
  HR_REQUIRE(kind == HRGPU_LINKS_F32 || kind == HRGPU_LINKS_BF16, HRGPU_E_ARG,
             "set_flt_link_storage: kind must be HRGPU_LINKS_F32 or HRGPU_LINKS_BF16");
  L.flt_links = kind;
  return 0;
}

int hrgpu_set_dirac_mass(double mass) {
  g_static_mass = mass;
  return 0;
}
double hrgpu_get_dirac_mass(void) { return g_static_mass; }

// H2, H, D of D_update.c:41-95 in the UPDATE_EO build
int hrgpu_H2(void *out, const void *in) {
  return L.clover ? hrgpu_g5Cphi_eopre_sq(g_static_mass, out, in) : hrgpu_g5Dphi_eopre_sq(g_static_mass, out, in);
}
int hrgpu_H(void *out, const void *in) {
  return L.clover ? hrgpu_g5Cphi_eopre(g_static_mass, out, in) : hrgpu_g5Dphi_eopre(g_static_mass, out, in);
}
int hrgpu_D(void *out, const void *in) {
  return L.clover ? hrgpu_Cphi_eopre(g_static_mass, out, in) : hrgpu_Dphi_eopre(g_static_mass, out, in);
}

}  // extern "C"
