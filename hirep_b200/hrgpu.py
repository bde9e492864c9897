"""Python host mirror of the B200 fermion library (libhrgpu.so, C ABI in include/hrgpu.h).

The method names follow HiRep's C API (LibHR/Update/Dphi.c, D_update.c,
LibHR/Inverters/linear_algebra.c, cg_mshift*.c, LibHR/Update/force_fermion_core.c),
so host code and tests read like HiRep's own.  Device memory comes from
PyTorch (plumbing only); every computation runs in libhrgpu.so.  There is no
CPU fallback: if the library is missing the import fails.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhrgpu.so")

EVEN, ODD, FULL = 0, 1, 2
DOUBLE, FLOAT = 0, 1
FUND, ADJ, SYM, ASYM = 0, 1, 2, 3
OP_G5DPHI_SQ, OP_G5DPHI_EOPRE_SQ, OP_G5CPHI_EOPRE_SQ, OP_G5CPHI_SQ = 0, 1, 2, 3
OP_DPHI_EOPRE, OP_G5DPHI_EOPRE, OP_CPHI_EOPRE, OP_G5CPHI_EOPRE, OP_DPHI, OP_CPHI = 4, 5, 6, 7, 8, 9
E_NOCONV = 5
E_BREAKDOWN = 6
LINKS_F32, LINKS_BF16 = 0, 1

_lib = None


class HRGPUError(RuntimeError):
    pass


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise HRGPUError("libhrgpu.so is not built (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        L.hrgpu_last_error.restype = ctypes.c_char_p
        L.hrgpu_spinor_bytes.restype = ctypes.c_size_t
        L.hrgpu_getMVM.restype = ctypes.c_ulong
        L.hrgpu_get_dirac_mass.restype = ctypes.c_double
        L.hrgpu_batch_bytes.restype = ctypes.c_size_t
        L.hrgpu_mre_init.restype = ctypes.c_void_p
        L.hrgpu_random_seed.argtypes = [ctypes.c_ulonglong]
        _lib = L
    return _lib


def _check(rc, what):
    if rc != 0:
        msg = lib().hrgpu_last_error().decode()
        raise HRGPUError(f"{what}: status {rc}: {msg}")


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


D = ctypes.c_double


def geometry(T, X, Y, Z):
    """HiRep's serial site maps (ipt, iup, idn) built by the library (no GPU needed)."""
    V = T * X * Y * Z
    ipt = np.empty(V, np.int32)
    iup = np.empty(4 * V, np.int32)
    idn = np.empty(4 * V, np.int32)
    _check(lib().hrgpu_geometry(T, X, Y, Z, _ptr(ipt), _ptr(iup), _ptr(idn)), "geometry")
    return ipt, iup, idn


class Field:
    """A device spinor field in the library layout (parity, precision)."""

    def __init__(self, lat, par, prec=DOUBLE):
        import torch

        self.lat, self.par, self.prec = lat, par, prec
        self.nbytes = lib().hrgpu_spinor_bytes(par, prec)
        self.buf = torch.zeros(self.nbytes, dtype=torch.uint8, device="cuda")
        self.ptr = ctypes.c_void_p(self.buf.data_ptr())

    def upload(self, host):
        dt = np.complex128 if self.prec == DOUBLE else np.complex64
        host = np.ascontiguousarray(host, dt)
        assert host.shape == (self.lat.nsites(self.par), 4, self.lat.nf), host.shape
        _check(lib().hrgpu_spinor_upload(self.ptr, _ptr(host), self.par, self.prec), "spinor_upload")
        return self

    def download(self):
        dt = np.complex128 if self.prec == DOUBLE else np.complex64
        out = np.empty((self.lat.nsites(self.par), 4, self.lat.nf), dt)
        _check(lib().hrgpu_spinor_download(_ptr(out), self.ptr, self.par, self.prec), "spinor_download")
        return out


class Batch:
    """nb even-parity fields interleaved in one device buffer (field index fastest)."""

    def __init__(self, lat, nb, prec=DOUBLE):
        import torch

        self.lat, self.nb, self.prec = lat, nb, prec
        self.nbytes = lib().hrgpu_batch_bytes(prec, nb)
        if self.nbytes == 0:
            raise HRGPUError("batch_bytes: lattice not initialised or nb <= 0")
        self.buf = torch.zeros(self.nbytes, dtype=torch.uint8, device="cuda")
        self.ptr = ctypes.c_void_p(self.buf.data_ptr())

    def pack(self, fields):
        assert len(fields) == self.nb
        arr = (ctypes.c_void_p * self.nb)(*[f.ptr.value for f in fields])
        _check(lib().hrgpu_batch_pack(self.ptr, arr, self.nb, self.prec), "batch_pack")
        return self

    def unpack(self, fields):
        assert len(fields) == self.nb
        arr = (ctypes.c_void_p * self.nb)(*[f.ptr.value for f in fields])
        _check(lib().hrgpu_batch_unpack(arr, self.ptr, self.nb, self.prec), "batch_unpack")


class MREHandle:
    """Past solutions for the chronological initial guess (mre_store / mre_guess)."""

    def __init__(self, lat, h):
        self.lat, self.h = lat, h

    def store(self, p, field):
        _check(self.lat.L.hrgpu_mre_store(self.h, p, field.ptr), "mre_store")

    def guess(self, p, out, op, mass, pf):
        _check(self.lat.L.hrgpu_mre_guess(self.h, p, out.ptr, op, D(mass), pf.ptr), "mre_guess")

    def free(self):
        if self.h:
            _check(self.lat.L.hrgpu_mre_free(self.h), "mre_free")
            self.h = None


class Lattice:
    """One lattice on one GPU: geometry, gauge field, clover term, force accumulator."""

    def __init__(self, T, X, Y, Z, ng, repr_, ipt=None, device=0):
        import torch

        self.L = lib()
        if ipt is None:
            ipt = geometry(T, X, Y, Z)[0]
        _check(self.L.hrgpu_init(device), "init")
        torch.cuda.set_device(device)
        _check(self.L.hrgpu_set_stream(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), "set_stream")
        ipt = np.ascontiguousarray(ipt, np.int32)
        _check(self.L.hrgpu_lattice_init(T, X, Y, Z, ng, repr_, _ptr(ipt)), "lattice_init")
        self.dims = (T, X, Y, Z)
        self.V = T * X * Y * Z
        self.VH = self.V // 2
        self.ng, self.repr = ng, repr_
        self.nf = self.L.hrgpu_nf()
        self.real = repr_ == ADJ
        self.dimg = ng * ng - 1
        self.csw = None  # clover coefficient once clover_init was called
        self.expclover = False  # the exponential form (expclover_init)

    def nsites(self, par):
        return self.V if par == FULL else self.VH

    def field(self, par, prec=DOUBLE, host=None):
        f = Field(self, par, prec)
        if host is not None:
            f.upload(host)
        return f

    def sync(self):
        _check(self.L.hrgpu_synchronize(), "synchronize")

    # gauge ---------------------------------------------------------------
    def set_gauge_f(self, uf):
        dt = np.float64 if self.real else np.complex128
        uf = np.ascontiguousarray(uf, dt)
        _check(self.L.hrgpu_gauge_set_f(_ptr(uf)), "gauge_set_f")

    def set_gauge(self, u):
        u = np.ascontiguousarray(u, np.complex128)
        _check(self.L.hrgpu_gauge_set(_ptr(u)), "gauge_set")

    def represent_gauge_field(self, bc_t_antiperiodic=True):
        _check(self.L.hrgpu_represent_gauge_field(int(bool(bc_t_antiperiodic))), "represent_gauge_field")

    def link_recon(self):
        """0: the hopping kernels read full links; 1, 2: they rebuild row 2 of the
        SU(3) links (2: with the antiperiodic time sign)."""
        m = ctypes.c_int(-1)
        _check(self.L.hrgpu_link_recon(ctypes.byref(m)), "link_recon")
        return m.value

    def gauge_f(self):
        dt = np.float64 if self.real else np.complex128
        uf = np.empty((self.V, 4, self.nf, self.nf), dt)
        _check(self.L.hrgpu_gauge_get_f(_ptr(uf)), "gauge_get_f")
        return uf

    # Dirac operator --------------------------------------------------------
    def Dphi_(self, out, inp):
        _check(self.L.hrgpu_Dphi_(out.ptr, out.par, inp.ptr), "Dphi_")

    def Dphi_flt_(self, out, inp):
        _check(self.L.hrgpu_Dphi_flt_(out.ptr, out.par, inp.ptr), "Dphi_flt_")

    def _m(self, name, m, out, inp):
        _check(getattr(self.L, "hrgpu_" + name)(D(m), out.ptr, inp.ptr), name)

    def Dphi(self, m, out, inp): self._m("Dphi", m, out, inp)
    def g5Dphi(self, m, out, inp): self._m("g5Dphi", m, out, inp)
    def g5Dphi_sq(self, m, out, inp): self._m("g5Dphi_sq", m, out, inp)
    def Dphi_eopre(self, m, out, inp): self._m("Dphi_eopre", m, out, inp)
    def Dphi_oepre(self, m, out, inp): self._m("Dphi_oepre", m, out, inp)
    def g5Dphi_eopre(self, m, out, inp): self._m("g5Dphi_eopre", m, out, inp)
    def g5Dphi_eopre_sq(self, m, out, inp): self._m("g5Dphi_eopre_sq", m, out, inp)
    def Dphi_flt(self, m, out, inp): self._m("Dphi_flt", m, out, inp)
    def g5Dphi_flt(self, m, out, inp): self._m("g5Dphi_flt", m, out, inp)
    def g5Dphi_sq_flt(self, m, out, inp): self._m("g5Dphi_sq_flt", m, out, inp)
    def Dphi_eopre_flt(self, m, out, inp): self._m("Dphi_eopre_flt", m, out, inp)
    def g5Dphi_eopre_flt(self, m, out, inp): self._m("g5Dphi_eopre_flt", m, out, inp)
    def g5Dphi_eopre_sq_flt(self, m, out, inp): self._m("g5Dphi_eopre_sq_flt", m, out, inp)

    def getMVM(self):
        return self.L.hrgpu_getMVM()

    def set_dirac_mass(self, m):
        _check(self.L.hrgpu_set_dirac_mass(D(m)), "set_dirac_mass")

    def H2(self, out, inp): _check(self.L.hrgpu_H2(out.ptr, inp.ptr), "H2")
    def H(self, out, inp): _check(self.L.hrgpu_H(out.ptr, inp.ptr), "H")
    def D(self, out, inp): _check(self.L.hrgpu_D(out.ptr, inp.ptr), "D")

    # clover --------------------------------------------------------------
    def clover_init(self, csw):
        _check(self.L.hrgpu_clover_init(D(csw)), "clover_init")
        self.csw = csw
        self.expclover = False

    def expclover_init(self, csw):
        _check(self.L.hrgpu_expclover_init(D(csw)), "expclover_init")
        self.csw = csw
        self.expclover = True

    def compute_clover_term(self):
        _check(self.L.hrgpu_compute_clover_term(), "compute_clover_term")

    def clover_term(self):
        cl = np.empty((self.V, 4, self.nf, self.nf), np.complex128)
        _check(self.L.hrgpu_clover_term_get(_ptr(cl)), "clover_term_get")
        return cl

    def clover_force(self):
        cf = np.empty((self.V, 6, self.nf, self.nf), np.complex128)
        _check(self.L.hrgpu_clover_force_get(_ptr(cf)), "clover_force_get")
        return cf

    def Cphi(self, m, out, inp): self._m("Cphi", m, out, inp)
    def g5Cphi(self, m, out, inp): self._m("g5Cphi", m, out, inp)
    def g5Cphi_sq(self, m, out, inp): self._m("g5Cphi_sq", m, out, inp)
    def Cphi_eopre(self, m, out, inp): self._m("Cphi_eopre", m, out, inp)
    def g5Cphi_eopre(self, m, out, inp): self._m("g5Cphi_eopre", m, out, inp)
    def g5Cphi_eopre_sq(self, m, out, inp): self._m("g5Cphi_eopre_sq", m, out, inp)
    def g5Cphi_eopre_flt(self, m, out, inp): self._m("g5Cphi_eopre_flt", m, out, inp)
    def g5Cphi_eopre_sq_flt(self, m, out, inp): self._m("g5Cphi_eopre_sq_flt", m, out, inp)

    def Cphi_diag(self, m, out, inp):
        _check(self.L.hrgpu_Cphi_diag(D(m), out.ptr, inp.ptr, out.par), "Cphi_diag")

    def Cphi_diag_inv(self, m, out, inp):
        _check(self.L.hrgpu_Cphi_diag_inv(D(m), out.ptr, inp.ptr, out.par), "Cphi_diag_inv")

    # linear algebra --------------------------------------------------------
    def la(self, name, *args):
        """spinor_field_<name>_f / _f_flt: args as in HiRep; fields are Field objects."""
        fields = [a for a in args if isinstance(a, Field)]
        par, prec = fields[0].par, fields[0].prec
        cargs = []
        for a in args:
            if isinstance(a, Field):
                cargs.append(a.ptr)
            elif isinstance(a, complex):
                cargs += [D(a.real), D(a.imag)]
            else:
                cargs.append(D(a))
        _check(getattr(self.L, "hrgpu_spinor_field_" + name)(par, prec, *cargs), "spinor_field_" + name)

    def la_red(self, name, *fields, n=1):
        res = (ctypes.c_double * 2)()
        _check(getattr(self.L, "hrgpu_spinor_field_" + name)(fields[0].par, fields[0].prec,
                                                              *[f.ptr for f in fields], res), name)
        return res[0] if n == 1 else complex(res[0], res[1])

    def sqnorm(self, f): return self.la_red("sqnorm", f)
    def prod_re(self, a, b): return self.la_red("prod_re", a, b)
    def prod_im(self, a, b): return self.la_red("prod_im", a, b)
    def prod(self, a, b): return self.la_red("prod", a, b, n=2)
    def g5_prod_re(self, a, b): return self.la_red("g5_prod_re", a, b)
    def g5_prod_im(self, a, b): return self.la_red("g5_prod_im", a, b)

    def assign_sd2s(self, out, inp):
        _check(self.L.hrgpu_assign_sd2s(out.ptr, inp.ptr, inp.par), "assign_sd2s")

    def assign_s2sd(self, out, inp):
        _check(self.L.hrgpu_assign_s2sd(out.ptr, inp.ptr, inp.par), "assign_s2sd")

    # inverters -------------------------------------------------------------
    def cg_mshift(self, op, mass, shifts, err2, inp, outs, max_iter=0, flt=False):
        n = len(shifts)
        sh = np.ascontiguousarray(shifts, np.float64)
        arr = (ctypes.c_void_p * n)(*[o.ptr.value for o in outs])
        it = ctypes.c_int(0)
        fn = self.L.hrgpu_cg_mshift_flt if flt else self.L.hrgpu_cg_mshift
        rc = fn(op, D(mass), n, _ptr(sh), D(err2), max_iter, inp.ptr, arr, ctypes.byref(it))
        if rc == E_NOCONV:
            return it.value, False
        _check(rc, "cg_mshift_flt" if flt else "cg_mshift")
        return it.value, True

    def g5QMR_mshift(self, op, mass, shifts, err2, inp, outs, max_iter=0):
        n = len(shifts)
        sh = np.ascontiguousarray(shifts, np.float64)
        arr = (ctypes.c_void_p * n)(*[o.ptr.value for o in outs])
        it = ctypes.c_int(0)
        rc = self.L.hrgpu_g5QMR_mshift(op, D(mass), n, _ptr(sh), D(err2), max_iter, inp.ptr, arr, ctypes.byref(it))
        if rc == E_NOCONV:
            return it.value, False
        _check(rc, "g5QMR_mshift")
        return it.value, True

    def MINRES(self, op, mass, err2, inp, out, trial=None, max_iter=0):
        it = ctypes.c_int(0)
        rc = self.L.hrgpu_MINRES(op, D(mass), D(err2), max_iter, inp.ptr, out.ptr,
                                 None if trial is None else trial.ptr, ctypes.byref(it))
        if rc == E_NOCONV:
            return it.value, False
        _check(rc, "MINRES")
        return it.value, True

    def mre(self, max_, par):
        """An MRE handle (LibHR/Update/mre.c) for fields of parity par."""
        h = self.L.hrgpu_mre_init(max_, par)
        if not h:
            raise HRGPUError("mre_init: " + self.L.hrgpu_last_error().decode())
        return MREHandle(self, ctypes.c_void_p(h))

    # HMC pieces -----------------------------------------------------------------
    def momenta_set(self, mom):
        mom = np.ascontiguousarray(mom, np.float64)
        assert mom.shape == (self.V, 4, self.dimg)
        _check(self.L.hrgpu_momenta_set(_ptr(mom)), "momenta_set")

    def momenta_get(self):
        mom = np.empty((self.V, 4, self.dimg), np.float64)
        _check(self.L.hrgpu_momenta_get(_ptr(mom)), "momenta_get")
        return mom

    # random draws on the device (Philox4x32-10, Box-Muller) ---------------
    def random_seed(self, seed):
        _check(self.L.hrgpu_random_seed(int(seed) & (2**64 - 1)), "random_seed")

    def gaussian_momenta(self):
        """gaussian_momenta (random_momenta.c:18-38) into the device momenta."""
        _check(self.L.hrgpu_gaussian_momenta(), "gaussian_momenta")

    def gaussian_spinor_field(self, f):
        """gaussian_spinor_field (random_spinor_field.c:14-36) into a device field."""
        _check(self.L.hrgpu_gaussian_spinor_field(f.par, f.prec, f.ptr), "gaussian_spinor_field")
        return f

    def gauge_get(self):
        u = np.empty((self.V, 4, self.ng, self.ng), np.complex128)
        _check(self.L.hrgpu_gauge_get(_ptr(u)), "gauge_get")
        return u

    def force0(self, dt, beta):
        _check(self.L.hrgpu_force0(D(dt), D(beta)), "force0")

    def update_gauge_field(self, dt):
        _check(self.L.hrgpu_update_gauge_field(D(dt)), "update_gauge_field")

    def project_gauge_field(self):
        _check(self.L.hrgpu_project_gauge_field(), "project_gauge_field")

    def local_hmc_action(self, delta, beta):
        _check(self.L.hrgpu_local_hmc_action(int(bool(delta)), D(beta)), "local_hmc_action")

    def pf_local_action(self, pf):
        _check(self.L.hrgpu_pf_local_action(pf.ptr, pf.par), "pf_local_action")

    def clover_la_logdet(self, nf, mass):
        _check(self.L.hrgpu_clover_la_logdet(D(nf), D(mass)), "clover_la_logdet")

    def local_action_sum(self):
        s = ctypes.c_double()
        _check(self.L.hrgpu_local_action_sum(ctypes.byref(s)), "local_action_sum")
        return s.value

    def local_action(self):
        loc = np.empty(self.V, np.float64)
        _check(self.L.hrgpu_local_action_get(_ptr(loc)), "local_action_get")
        return loc

    def avr_plaquette(self):
        p = ctypes.c_double()
        _check(self.L.hrgpu_avr_plaquette(ctypes.byref(p)), "avr_plaquette")
        return p.value

    def write_gauge_field(self, filename):
        _check(self.L.hrgpu_write_gauge_field(str(filename).encode()), "write_gauge_field")

    def read_gauge_field(self, filename):
        """Returns (plaquette stored in the file, plaquette of the links read)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        _check(self.L.hrgpu_read_gauge_field(str(filename).encode(), ctypes.byref(a), ctypes.byref(b)),
               "read_gauge_field")
        return a.value, b.value

    def fermion_force_end_momenta(self, dt):
        _check(self.L.hrgpu_fermion_force_end_momenta(D(dt)), "fermion_force_end_momenta")

    # many right-hand sides -------------------------------------------------------
    def batch(self, nb, prec=DOUBLE, fields=None):
        b = Batch(self, nb, prec)
        if fields is not None:
            b.pack(fields)
        return b

    def apply_op_host(self, op, mass, host_in, prec=DOUBLE, out=None):
        """An even-odd operator (OP_DPHI_EOPRE .. OP_G5CPHI_EOPRE) on an even host
        field [VH][4][NF] in HiRep order; the copies overlap the computation.
        host_in / out may be pinned torch tensors viewed as numpy (the fast path)
        or plain numpy arrays."""
        dt = np.complex128 if prec == DOUBLE else np.complex64
        host_in = np.ascontiguousarray(host_in, dt)
        assert host_in.shape == (self.VH, 4, self.nf), host_in.shape
        if out is None:
            out = np.empty_like(host_in)
        _check(self.L.hrgpu_apply_op_host(op, D(mass), _ptr(out), _ptr(host_in), prec), "apply_op_host")
        return out

    def set_host_chunks(self, chunks):
        _check(self.L.hrgpu_set_host_chunks(chunks), "set_host_chunks")

    def apply_op_batch(self, op, mass, out, inp):
        _check(self.L.hrgpu_apply_op_batch(op, out.prec, D(mass), out.ptr, inp.ptr, out.nb), "apply_op_batch")

    def cg_mshift_batch(self, op, mass, sources, shifts, err2, outs, max_iter=0, flt=False):
        """sources: list of even Fields; shifts: list (per source) of shift lists;
        outs: flat list of Fields, source by source.  Returns (iters per source, ok)."""
        nsrc = len(sources)
        nsh = np.ascontiguousarray([len(s) for s in shifts], np.int32)
        sh = np.ascontiguousarray([x for s in shifts for x in s], np.float64)
        assert len(outs) == len(sh)
        ins = (ctypes.c_void_p * nsrc)(*[f.ptr.value for f in sources])
        arr = (ctypes.c_void_p * len(outs))(*[o.ptr.value for o in outs])
        it = np.zeros(nsrc, np.int32)
        rc = self.L.hrgpu_cg_mshift_batch(op, D(mass), nsrc, _ptr(nsh), _ptr(sh), D(err2), max_iter, ins, arr,
                                          int(bool(flt)), _ptr(it))
        if rc == E_NOCONV:
            return it, False
        _check(rc, "cg_mshift_batch")
        return it, True

    # force -------------------------------------------------------------------
    def generators(self):
        """T_A of su(NG) (Tr T_A T_B = delta/2), the basis of forces and momenta."""
        t = np.empty((self.dimg, self.ng, self.ng), np.complex128)
        _check(self.L.hrgpu_algebra_generators(_ptr(t)), "algebra_generators")
        return t

    def fermion_force_begin(self):
        _check(self.L.hrgpu_fermion_force_begin(), "fermion_force_begin")

    def force_fermion_core(self, Xs, Ys, auto_fill_odd, dt, residue):
        _check(self.L.hrgpu_force_fermion_core(Xs.ptr, Ys.ptr, int(auto_fill_odd), D(dt), D(residue)),
               "force_fermion_core")

    def force_clover_logdet(self, mass, residue):
        _check(self.L.hrgpu_force_clover_logdet(D(mass), D(residue)), "force_clover_logdet")

    def fermion_force_end(self, dt, force):
        force = np.ascontiguousarray(force, np.float64).copy()
        _check(self.L.hrgpu_fermion_force_end(D(dt), _ptr(force)), "fermion_force_end")
        return force

    def force_sum(self):
        f = np.empty((self.V, 4, self.dimg), np.float64)
        _check(self.L.hrgpu_force_sum_get(_ptr(f)), "force_sum_get")
        return f

    def finalize(self):
        _check(self.L.hrgpu_finalize(), "finalize")
