"""ctypes wrapper around the CPU oracle (oracle/hr_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of bench.py, as the checker.  The GPU library never imports it.

Fields are numpy arrays in HiRep's host layout:
  spinor field   complex128 [nsites, 4, NF]   (nsites = V/2 for one parity, V full)
  represented    complex128 [V, 4, NF, NF] or float64 for the adjoint representation
  fundamental    complex128 [V, 4, NG, NG]
  force          float64    [V, 4, NG*NG-1]
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libhroracle.so")

FUND, ADJ, SYM, ASYM = 0, 1, 2, 3
EVEN, ODD, FULL = 0, 1, 2
OP_G5DPHI_SQ, OP_G5DPHI_EOPRE_SQ, OP_G5CPHI_EOPRE_SQ, OP_G5CPHI_SQ = 0, 1, 2, 3
OP_DPHI_EOPRE, OP_G5DPHI_EOPRE, OP_CPHI_EOPRE, OP_G5CPHI_EOPRE, OP_DPHI, OP_CPHI = 4, 5, 6, 7, 8, 9
REPR_NAMES = {"FUND": FUND, "ADJ": ADJ, "SYM": SYM, "ASYM": ASYM}


def build():
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.orc_avr_plaquette.restype = ctypes.c_double
        for name in ("orc_sqnorm", "orc_prod_re", "orc_prod_im", "orc_g5_prod_re", "orc_g5_prod_im"):
            getattr(_lib, name).restype = ctypes.c_double
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def nf_of(ng, repr_):
    return {FUND: ng, ADJ: ng * ng - 1, SYM: ng * (ng + 1) // 2, ASYM: ng * (ng - 1) // 2}[repr_]


class Oracle:
    """One lattice + representation, mirroring HiRep's global state (serial build)."""

    def __init__(self, T, X, Y, Z, ng, repr_, threads=None):
        self.L = lib()
        if threads is not None:
            self.L.orc_set_threads(int(threads))
        rc = self.L.orc_init(T, X, Y, Z, ng, repr_)
        if rc != 0:
            raise ValueError("oracle: bad lattice/representation")
        self.dims = (T, X, Y, Z)
        self.ng, self.repr = ng, repr_
        self.nf = self.L.orc_nf()
        self.real = bool(self.L.orc_real_links())
        self.V = T * X * Y * Z
        self.VH = self.V // 2
        self.dimg = self.L.orc_group_dim()
        self._keep = {}

    # geometry ------------------------------------------------------------
    def geometry(self):
        ipt = np.empty(self.V, np.int32)
        iup = np.empty(4 * self.V, np.int32)
        idn = np.empty(4 * self.V, np.int32)
        self.L.orc_geometry(_p(ipt), _p(iup), _p(idn))
        return ipt, iup, idn

    # algebra -------------------------------------------------------------
    def generators(self):
        gT = np.empty((self.dimg, self.ng, self.ng), np.complex128)
        rT = np.empty((self.dimg, self.nf, self.nf), np.complex128)
        norms = np.empty(2, np.float64)
        self.L.orc_generators(_p(gT), _p(rT), _p(norms))
        return gT, rT, norms

    def link_dtype(self):
        return np.float64 if self.real else np.complex128

    def group_represent(self, u):
        u = np.ascontiguousarray(u, np.complex128)
        v = np.empty((self.nf, self.nf), self.link_dtype())
        self.L.orc_group_represent(_p(v), _p(u))
        return v

    def algebra_project(self, m):
        m = np.ascontiguousarray(m, self.link_dtype())
        h = np.empty(self.dimg, np.float64)
        self.L.orc_algebra_project(_p(h), _p(m))
        return h

    def fund_algebra_represent(self, h):
        h = np.ascontiguousarray(h, np.float64)
        m = np.empty((self.ng, self.ng), np.complex128)
        self.L.orc_fund_algebra_represent(_p(m), _p(h))
        return m

    def represent_gauge_field(self, u, bc_t_antiperiodic=True):
        u = np.ascontiguousarray(u, np.complex128)
        uf = np.empty((self.V, 4, self.nf, self.nf), self.link_dtype())
        self.L.orc_represent_gauge_field(_p(uf), _p(u), int(bool(bc_t_antiperiodic)))
        return uf

    def set_gauge(self, uf):
        uf = np.ascontiguousarray(uf, self.link_dtype())
        self._keep["uf"] = uf
        self.L.orc_set_gauge(_p(uf))
        uflt = uf.astype(np.float32 if self.real else np.complex64)
        self._keep["uf_flt"] = uflt
        self.L.orc_set_gauge_flt(_p(uflt))

    def set_mass(self, m):
        self.L.orc_set_mass(ctypes.c_double(m))

    # fields --------------------------------------------------------------
    def nsites(self, par):
        return self.V if par == FULL else self.VH

    def zeros(self, par, dtype=np.complex128):
        return np.zeros((self.nsites(par), 4, self.nf), dtype)

    def _c(self, a, dtype=np.complex128):
        return np.ascontiguousarray(a, dtype)

    # Wilson operator -----------------------------------------------------
    def Dphi_(self, inp, in_par, out_par):
        inp = self._c(inp)
        out = self.zeros(out_par)
        self.L.orc_Dphi_(_p(out), out_par, _p(inp), in_par)
        return out

    def _mop(self, name, m, inp, par):
        inp = self._c(inp)
        out = self.zeros(par)
        getattr(self.L, name)(ctypes.c_double(m), _p(out), _p(inp))
        return out

    def Dphi(self, m, inp): return self._mop("orc_Dphi", m, inp, FULL)
    def g5Dphi(self, m, inp): return self._mop("orc_g5Dphi", m, inp, FULL)
    def g5Dphi_sq(self, m, inp): return self._mop("orc_g5Dphi_sq", m, inp, FULL)
    def Dphi_eopre(self, m, inp): return self._mop("orc_Dphi_eopre", m, inp, EVEN)
    def Dphi_oepre(self, m, inp): return self._mop("orc_Dphi_oepre", m, inp, ODD)
    def g5Dphi_eopre(self, m, inp): return self._mop("orc_g5Dphi_eopre", m, inp, EVEN)
    def g5Dphi_eopre_sq(self, m, inp): return self._mop("orc_g5Dphi_eopre_sq", m, inp, EVEN)

    def Dphi_flt_(self, inp, in_par, out_par):
        inp = self._c(inp, np.complex64)
        out = self.zeros(out_par, np.complex64)
        self.L.orc_Dphi_flt_(_p(out), out_par, _p(inp), in_par)
        return out

    def _mop_flt(self, name, m, inp, par):
        inp = self._c(inp, np.complex64)
        out = self.zeros(par, np.complex64)
        getattr(self.L, name)(ctypes.c_double(m), _p(out), _p(inp))
        return out

    def Dphi_flt(self, m, inp): return self._mop_flt("orc_Dphi_flt", m, inp, FULL)
    def g5Dphi_eopre_flt(self, m, inp): return self._mop_flt("orc_g5Dphi_eopre_flt", m, inp, EVEN)
    def g5Dphi_eopre_sq_flt(self, m, inp): return self._mop_flt("orc_g5Dphi_eopre_sq_flt", m, inp, EVEN)
    def Dphi_eopre_flt(self, m, inp): return self._mop_flt("orc_Dphi_eopre_flt", m, inp, EVEN)

    # clover --------------------------------------------------------------
    def clover_init(self, csw):
        self.L.orc_clover_init(ctypes.c_double(csw))

    def expclover_init(self, csw):
        """WITH_EXPCLOVER: diagonal (4+m) exp(A/(4+m)) (Dphi.c:1292-1482)."""
        self.L.orc_expclover_init(ctypes.c_double(csw))

    def compute_clover_term(self):
        self.L.orc_compute_clover_term()

    def clover_term(self):
        cl = np.empty((self.V, 4, self.nf, self.nf), np.complex128)
        self.L.orc_get_clover_term(_p(cl))
        return cl

    def compute_ldl_decomp(self, sigma):
        self.L.orc_compute_ldl_decomp(ctypes.c_double(sigma))

    def clover_ldl(self):
        n = self.nf * (2 * self.nf + 1)
        a = np.empty((self.V, 2, n), np.complex128)
        self.L.orc_get_clover_ldl(_p(a))
        return a

    def Cphi(self, m, inp): return self._mop("orc_Cphi", m, inp, FULL)
    def g5Cphi(self, m, inp): return self._mop("orc_g5Cphi", m, inp, FULL)
    def g5Cphi_sq(self, m, inp): return self._mop("orc_g5Cphi_sq", m, inp, FULL)
    def Cphi_eopre(self, m, inp): return self._mop("orc_Cphi_eopre", m, inp, EVEN)
    def g5Cphi_eopre(self, m, inp): return self._mop("orc_g5Cphi_eopre", m, inp, EVEN)
    def g5Cphi_eopre_sq(self, m, inp): return self._mop("orc_g5Cphi_eopre_sq", m, inp, EVEN)

    def Cphi_diag(self, m, inp, par):
        inp = self._c(inp)
        out = self.zeros(par)
        self.L.orc_Cphi_diag(ctypes.c_double(m), _p(out), _p(inp), par)
        return out

    def Cphi_diag_inv(self, m, inp, par):
        inp = self._c(inp)
        out = self.zeros(par)
        self.L.orc_Cphi_diag_inv(ctypes.c_double(m), _p(out), _p(inp), par)
        return out

    # linear algebra ------------------------------------------------------
    def sqnorm(self, s):
        s = self._c(s)
        return self.L.orc_sqnorm(s.shape[0], _p(s))

    def prod_re(self, a, b):
        a, b = self._c(a), self._c(b)
        return self.L.orc_prod_re(a.shape[0], _p(a), _p(b))

    def prod_im(self, a, b):
        a, b = self._c(a), self._c(b)
        return self.L.orc_prod_im(a.shape[0], _p(a), _p(b))

    def g5_prod_re(self, a, b):
        a, b = self._c(a), self._c(b)
        return self.L.orc_g5_prod_re(a.shape[0], _p(a), _p(b))

    def g5_prod_im(self, a, b):
        a, b = self._c(a), self._c(b)
        return self.L.orc_g5_prod_im(a.shape[0], _p(a), _p(b))

    def gamma(self, mu, s):
        s = self._c(s)
        out = np.empty_like(s)
        if mu == 5:
            self.L.orc_g5(s.shape[0], _p(out), _p(s))
        else:
            self.L.orc_gamma(mu, s.shape[0], _p(out), _p(s))
        return out

    # inverters -----------------------------------------------------------
    def cg_mshift(self, op, shifts, err2, inp, max_iter=0, guess=None, flt=False):
        inp = self._c(inp)
        n = len(shifts)
        sh = np.ascontiguousarray(shifts, np.float64)
        out = np.zeros((n,) + inp.shape, np.complex128)
        if guess is not None:
            out[0] = guess
        fn = self.L.orc_cg_mshift_flt if flt else self.L.orc_cg_mshift
        it = fn(op, n, _p(sh), ctypes.c_double(err2), max_iter, _p(inp), _p(out))
        if it < 0:
            raise ValueError("oracle: operator has no float version")
        return out, it

    def g5QMR_mshift(self, op, shifts, err2, inp, max_iter=0, guess=None):
        """g5QMR_mshift (LibHR/Inverters/g5QMR_mshift.c:481-542); op is the gamma_5-hermitian M."""
        inp = self._c(inp)
        n = len(shifts)
        sh = np.ascontiguousarray(shifts, np.float64)
        out = np.zeros((n,) + inp.shape, np.complex128)
        if guess is not None:
            out[0] = guess
        it = self.L.orc_g5QMR_mshift(op, n, _p(sh), ctypes.c_double(err2), max_iter, _p(inp), _p(out))
        if it < 0:
            raise ValueError("oracle g5QMR: gamma_5 norm of the start vector is zero")
        return out, it

    def MINRES(self, op, err2, inp, trial=None, max_iter=0, g5=False, sh=0.0):
        """MINRES (LibHR/Inverters/MINRES.c:160-172) on the hermitian operator
        op - sh, or g5 (op - sh) when g5 is set."""
        inp = self._c(inp)
        out = np.zeros_like(inp)
        tr = None if trial is None else self._c(trial)
        it = self.L.orc_MINRES(op, int(bool(g5)), ctypes.c_double(sh), ctypes.c_double(err2), max_iter, _p(inp),
                               _p(out), None if tr is None else _p(tr))
        return out, it

    def mre_guess(self, op, solutions, pf):
        """mre_guess (LibHR/Update/mre.c:230-268) from past solutions (newest first)."""
        pf = self._c(pf)
        s = np.ascontiguousarray(np.asarray(solutions, np.complex128))
        out = np.zeros_like(pf)
        self.L.orc_mre_guess(op, len(solutions), _p(s), _p(out), _p(pf))
        return out

    # HMC pieces ------------------------------------------------------------
    def force0(self, dt, beta, u, mom):
        """force0 (LibHR/Update/force0.c:22-99): mom += -dt beta/NG proj(U staples^+); returns mom."""
        u = np.ascontiguousarray(u, np.complex128)
        mom = np.ascontiguousarray(mom, np.float64).copy()
        self.L.orc_force0(ctypes.c_double(dt), ctypes.c_double(beta), _p(u), _p(mom))
        return mom

    def update_gauge_field(self, dt, u, mom):
        """U <- exp(dt X(mom)) U on every link (field_update.c:18-66, ExpX); returns U."""
        u = np.ascontiguousarray(u, np.complex128).copy()
        mom = np.ascontiguousarray(mom, np.float64)
        self.L.orc_update_gauge_field(ctypes.c_double(dt), _p(u), _p(mom))
        return u

    def project_gauge_field(self, u):
        u = np.ascontiguousarray(u, np.complex128).copy()
        self.L.orc_project_gauge_field(_p(u))
        return u

    def local_hmc_action(self, beta, u, mom):
        """per-site 0.5 C(F) |mom|^2 - beta/NG (6 plaquettes) (local_action.c, mon_pg.c)"""
        u = np.ascontiguousarray(u, np.complex128)
        mom = np.ascontiguousarray(mom, np.float64)
        loc = np.zeros(self.V, np.float64)
        self.L.orc_local_hmc_action(ctypes.c_double(beta), _p(u), _p(mom), _p(loc))
        return loc

    # force ---------------------------------------------------------------
    def fermion_force_begin(self):
        self.L.orc_fermion_force_begin()

    def force_fermion_core(self, Xs, Ys, auto_fill_odd, dt, residue):
        """Xs, Ys: full-lattice spinors; with auto_fill_odd the odd halves are overwritten."""
        Xs = self._c(Xs).copy()
        Ys = self._c(Ys).copy()
        self.L.orc_force_fermion_core(_p(Xs), _p(Ys), int(auto_fill_odd), ctypes.c_double(dt), ctypes.c_double(residue))
        return Xs, Ys

    def clover_la_logdet(self, nf, mass, la):
        """la (per site, HiRep order) -= nf log det D_oo on the odd sites."""
        la = np.ascontiguousarray(la, np.float64)
        self.L.orc_clover_la_logdet(ctypes.c_double(nf), ctypes.c_double(mass), _p(la))
        return la

    def force_clover_logdet(self, mass, residue):
        self.L.orc_force_clover_logdet(ctypes.c_double(mass), ctypes.c_double(residue))

    def fermion_force_end(self, dt, force):
        force = self._c(force, np.float64).copy()
        self.L.orc_fermion_force_end(ctypes.c_double(dt), _p(force))
        return force

    def force_sum(self):
        f = np.empty((self.V, 4, self.dimg), np.float64)
        self.L.orc_get_force_sum(_p(f))
        return f

    def clover_force(self):
        cf = np.empty((self.V, 6, self.nf, self.nf), np.complex128)
        self.L.orc_get_clover_force(_p(cf))
        return cf

    # utilities -----------------------------------------------------------
    def avr_plaquette(self, u):
        u = self._c(u)
        return self.L.orc_avr_plaquette(_p(u))
