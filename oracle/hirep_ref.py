"""Python driver for HiRep's own library, built from the reference sources by
oracle/ref/Makefile into oracle/_ref/<config>/hr_ref (see oracle/ref/hr_ref.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the reference CPU arm of bench.py, as the checker and as the CPU baseline.  The
GPU library never imports it.

One ``HiRep`` object is one hr_ref process: one lattice, one compile-time
configuration (gauge group, representation, clover form), like a HiRep
program.  Fields are numpy arrays in HiRep's host layout, the same as the
oracle's (oracle/oracle.py):
  spinor field   complex128 [nsites, 4, NF]   (nsites = V/2 for one parity, V full)
  represented    complex128 [V, 4, NF, NF] or float64 for the adjoint representation
  fundamental    complex128 [V, 4, NG, NG]
  force          float64    [V, 4, NG*NG-1]
"""
import os
import shutil
import subprocess
import tempfile

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
EVEN, ODD, FULL = 0, 1, 2
_PAR = {EVEN: "e", ODD: "o", FULL: "f"}

# configuration name -> (NG, representation, clover form)
CONFIGS = {
    "su3_fund": (3, "FUND", None),
    "su3_fund_clover": (3, "FUND", "clover"),
    "su3_fund_expclover": (3, "FUND", "expclover"),
    "su4_asym": (4, "ASYM", None),
    "su3_sym_clover": (3, "SYM", "clover"),
    "su2_adj": (2, "ADJ", None),
    "su2_fund": (2, "FUND", None),
    "su3_adj": (3, "ADJ", None),
    "su4_fund": (4, "FUND", None),
    "su3_asym_clover": (3, "ASYM", "clover"),
}


def exe_path(cfg):
    return os.path.join(REF_DIR, cfg, "hr_ref")


def available(cfg):
    return os.access(exe_path(cfg), os.X_OK)


def build(cfg=None, jobs=8):
    """Build HiRep's library and the server (needs the reference sources)."""
    args = ["make", "-s", "-j", str(jobs), "-C", os.path.join(_HERE, "ref")]
    if cfg:
        args.append(cfg)
    subprocess.run(args, check=True)


def nf_of(ng, rep):
    return {"FUND": ng, "ADJ": ng * ng - 1, "SYM": ng * (ng + 1) // 2, "ASYM": ng * (ng - 1) // 2}[rep]


class HiRepError(RuntimeError):
    pass


class HiRep:
    """One HiRep process on a T x X x Y x Z lattice (serial build, OpenMP)."""

    def __init__(self, cfg, T, X, Y, Z, seed=12345, threads=None):
        if not available(cfg):
            raise HiRepError(f"HiRep build {cfg} missing: run make -C oracle/ref {cfg}")
        self.cfg = cfg
        self.ng, self.rep, self.clover = CONFIGS[cfg]
        self.nf = nf_of(self.ng, self.rep)
        self.real = self.rep == "ADJ"
        self.dims = (T, X, Y, Z)
        self.V = T * X * Y * Z
        self.VH = self.V // 2
        self.dimg = self.ng * self.ng - 1
        self.dir = tempfile.mkdtemp(prefix="hr_ref_")
        with open(os.path.join(self.dir, "input_file"), "w") as f:
            f.write(f"GLB_T = {T}\nGLB_X = {X}\nGLB_Y = {Y}\nGLB_Z = {Z}\n"
                    "NP_T = 1\nNP_X = 1\nNP_Y = 1\nNP_Z = 1\nN_REP = 1\n"
                    f"log:default = -1\nrlx_level = 1\nrlx_seed = {int(seed)}\nrlx_start = new\n")
        env = dict(os.environ)
        if threads is not None:
            env["OMP_NUM_THREADS"] = str(int(threads))
        env.setdefault("OMP_PROC_BIND", "close")
        self.p = subprocess.Popen([exe_path(cfg), "-i", "input_file"], cwd=self.dir, env=env,
                                  stdin=subprocess.PIPE, stdout=subprocess.PIPE, text=True)
        ready = self._reply()
        kv = dict(t.split("=") for t in ready.split()[1:] if "=" in t)
        self.threads = int(kv["threads"])
        if int(kv["NG"]) != self.ng or int(kv["NF"]) != self.nf or int(kv["V"]) != self.V:
            raise HiRepError(f"unexpected HiRep build: {ready}")
        self._slots = {}

    # process plumbing ------------------------------------------------------
    def _reply(self):
        line = self.p.stdout.readline()
        if not line:
            err = ""
            for name in ("err_0", "out_0"):
                path = os.path.join(self.dir, name)
                if os.path.exists(path):
                    err += open(path).read()[-2000:]
            raise HiRepError(f"hr_ref ended: {err.strip()}")
        line = line.strip()
        if not line.startswith("ok"):
            raise HiRepError(line)
        return line[2:].strip()

    def cmd(self, text):
        self.p.stdin.write(text + "\n")
        self.p.stdin.flush()
        return self._reply()

    def close(self):
        if self.p.poll() is None:
            try:
                self.p.stdin.write("quit\n")
                self.p.stdin.flush()
                self.p.wait(timeout=30)
            except Exception:
                self.p.kill()
        shutil.rmtree(self.dir, ignore_errors=True)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _path(self, name):
        return os.path.join(self.dir, name)

    def nsites(self, par):
        return self.V if par == FULL else self.VH

    def _slot(self, s, par, n=1):
        if self._slots.get(s) != (par, n):
            self.cmd(f"alloc {s} {_PAR[par]} {n}")
            self._slots[s] = (par, n)

    def _put(self, s, k, arr, par):
        a = np.ascontiguousarray(arr, np.complex128)
        assert a.shape == (self.nsites(par), 4, self.nf), a.shape
        a.tofile(self._path("in.bin"))
        self.cmd(f"load {s} {k} {self._path('in.bin')}")

    def _get(self, s, k, par):
        self.cmd(f"save {s} {k} {self._path('out.bin')}")
        return np.fromfile(self._path("out.bin"), np.complex128).reshape(self.nsites(par), 4, self.nf)

    # geometry and gauge field ----------------------------------------------
    def geometry(self):
        a, b, c = self._path("ipt.bin"), self._path("iup.bin"), self._path("idn.bin")
        self.cmd(f"geometry {a} {b} {c}")
        return np.fromfile(a, np.int32), np.fromfile(b, np.int32), np.fromfile(c, np.int32)

    def set_gauge(self, u):
        """Fundamental links [V,4,NG,NG] in HiRep site order, read as read_gauge_field
        does (boundary conditions applied), then represent_gauge_field()."""
        u = np.ascontiguousarray(u, np.complex128)
        assert u.shape == (self.V, 4, self.ng, self.ng)
        u.tofile(self._path("gauge.bin"))
        self.cmd(f"gauge {self._path('gauge.bin')}")

    def random_u(self):
        """HiRep's hot start: random_u(u_gauge) from ranlux (rlx_seed), represented."""
        self.cmd("random_u")
        return self.gauge()

    def gauge(self):
        self.cmd(f"gauge_save {self._path('g.bin')}")
        return np.fromfile(self._path("g.bin"), np.complex128).reshape(self.V, 4, self.ng, self.ng)

    def gauge_f(self):
        self.cmd(f"gauge_f_save {self._path('gf.bin')}")
        dt = np.float64 if self.real else np.complex128
        return np.fromfile(self._path("gf.bin"), dt).reshape(self.V, 4, self.nf, self.nf)

    def plaquette(self):
        return float(self.cmd("plaq"))

    def gaussian_spinor_field(self, par):
        """gaussian_spinor_field (random_spinor_field.c:14-24) from HiRep's ranlux."""
        self._slot(9, par)
        self.cmd("gaussian 9 0")
        return self._get(9, 0, par)

    # clover -----------------------------------------------------------------
    def set_csw(self, csw):
        self.cmd(f"csw {float(csw)!r}")

    def clover_term(self):
        self.cmd(f"clterm_save {self._path('cl.bin')}")
        return np.fromfile(self._path("cl.bin"), np.complex128).reshape(self.V, 4, self.nf, self.nf)

    def clover_ldl(self, mass):
        self.cmd(f"ldl_save {float(mass)!r} {self._path('ldl.bin')}")
        n = self.nf * (2 * self.nf + 1)
        return np.fromfile(self._path("ldl.bin"), np.complex128).reshape(self.V, 2, n)

    def clover_force(self):
        self.cmd(f"clforce_save {self._path('clf.bin')}")
        return np.fromfile(self._path("clf.bin"), np.complex128).reshape(self.V, 6, self.nf, self.nf)

    # operators --------------------------------------------------------------
    def apply(self, name, m, inp, in_par, out_par):
        self._slot(0, in_par)
        self._slot(1, out_par)
        self._put(0, 0, inp, in_par)
        self.cmd(f"op {name} {float(m)!r} 1 0")
        return self._get(1, 0, out_par)

    def Dphi_(self, inp, in_par, out_par): return self.apply("Dphi_", 0.0, inp, in_par, out_par)
    def Dphi(self, m, inp): return self.apply("Dphi", m, inp, FULL, FULL)
    def g5Dphi(self, m, inp): return self.apply("g5Dphi", m, inp, FULL, FULL)
    def g5Dphi_sq(self, m, inp): return self.apply("g5Dphi_sq", m, inp, FULL, FULL)
    def Dphi_eopre(self, m, inp): return self.apply("Dphi_eopre", m, inp, EVEN, EVEN)
    def Dphi_oepre(self, m, inp): return self.apply("Dphi_oepre", m, inp, ODD, ODD)
    def g5Dphi_eopre(self, m, inp): return self.apply("g5Dphi_eopre", m, inp, EVEN, EVEN)
    def g5Dphi_eopre_sq(self, m, inp): return self.apply("g5Dphi_eopre_sq", m, inp, EVEN, EVEN)
    def Cphi(self, m, inp): return self.apply("Cphi", m, inp, FULL, FULL)
    def g5Cphi(self, m, inp): return self.apply("g5Cphi", m, inp, FULL, FULL)
    def g5Cphi_sq(self, m, inp): return self.apply("g5Cphi_sq", m, inp, FULL, FULL)
    def Cphi_eopre(self, m, inp): return self.apply("Cphi_eopre", m, inp, EVEN, EVEN)
    def g5Cphi_eopre(self, m, inp): return self.apply("g5Cphi_eopre", m, inp, EVEN, EVEN)
    def g5Cphi_eopre_sq(self, m, inp): return self.apply("g5Cphi_eopre_sq", m, inp, EVEN, EVEN)
    def Cphi_diag(self, m, inp, par): return self.apply("Cphi_diag", m, inp, par, par)
    def Cphi_diag_inv(self, m, inp, par): return self.apply("Cphi_diag_inv", m, inp, par, par)

    def time_op(self, name, m, par, warmup=3, reps=20, inp=None):
        """Median and minimum wall time (us) of one application, HiRep's own loop."""
        self._slot(0, par)
        self._slot(1, par)
        if inp is None:
            self.cmd("gaussian 0 0")
        else:
            self._put(0, 0, inp, par)
        med, mn, thr = self.cmd(f"time {name} {float(m)!r} 1 0 {int(warmup)} {int(reps)}").split()
        return float(med), float(mn), int(thr)

    # inverters --------------------------------------------------------------
    def cg_mshift(self, name, m, shifts, err2, inp, par, max_iter=0, flt=False, guess=None):
        """cg_mshift (cg_mshift.c:150-195) on (M - shifts[i]), M = NAME(m); with flt,
        cg_mshift_flt (cg_mshift_flt.c) with NAME's float form.  Returns (out, MVM)."""
        n = len(shifts)
        self._slot(2, par)
        self._slot(3, par, n)
        self._put(2, 0, inp, par)
        for k in range(n):
            if k == 0 and guess is not None:
                self._put(3, 0, guess, par)
            else:
                self._put(3, k, np.zeros((self.nsites(par), 4, self.nf)), par)
        sh = " ".join(repr(float(s)) for s in shifts)
        mvm = int(self.cmd(f"{'cgflt' if flt else 'cg'} {name} {float(m)!r} {float(err2)!r} {int(max_iter)} 2 3 {n} {sh}"))
        return np.stack([self._get(3, k, par) for k in range(n)]), mvm

    def time_cg(self, name, m, err2, par, warmup=1, reps=3, inp=None):
        self._slot(2, par)
        self._slot(3, par)
        if inp is None:
            self.cmd("gaussian 2 0")
        else:
            self._put(2, 0, inp, par)
        med, mn, thr, mvm = self.cmd(f"timecg {name} {float(m)!r} {float(err2)!r} 2 3 {int(warmup)} {int(reps)}").split()
        return float(med), float(mn), int(thr), int(mvm)

    # force ------------------------------------------------------------------
    def force(self, m, dt, residue, Xs, Ys, auto_fill_odd=True):
        """fermion_force_begin; force_fermion_core(Xs, Ys, auto_fill_odd, dt, residue)
        (force_fermion_core.c:788-928, the clover derivative included in clover
        builds); fermion_force_end(dt, F) into a zero field F (:935-993).  Xs and Ys
        are full-lattice spinors.  Returns F [V, 4, NG*NG-1]."""
        self._slot(4, FULL)
        self._slot(5, FULL)
        self._put(4, 0, Xs, FULL)
        self._put(5, 0, Ys, FULL)
        path = self._path("force.bin")
        self.cmd(f"force {float(m)!r} {float(dt)!r} {float(residue)!r} {int(bool(auto_fill_odd))} 4 5 {path}")
        return np.fromfile(path, np.float64).reshape(self.V, 4, self.dimg)

    def sqnorm(self, inp, par):
        self._slot(0, par)
        self._put(0, 0, inp, par)
        return float(self.cmd("sqnorm 0 0"))

    # g5QMR, MINRES -----------------------------------------------------------
    def g5QMR_mshift(self, name, m, shifts, err2, inp, par, max_iter=0, guess=None):
        """g5QMR_mshift (g5QMR_mshift.c:481-542) on (M - shifts[i]), M = NAME(m), the
        gamma_5-hermitian Dirac operator.  Returns (out, MVM)."""
        n = len(shifts)
        self._slot(2, par)
        self._slot(3, par, n)
        self._put(2, 0, inp, par)
        for k in range(n):
            if k == 0 and guess is not None:
                self._put(3, 0, guess, par)
            else:
                self._put(3, k, np.zeros((self.nsites(par), 4, self.nf)), par)
        sh = " ".join(repr(float(s)) for s in shifts)
        mvm = int(self.cmd(f"g5qmr {name} {float(m)!r} {float(err2)!r} {int(max_iter)} 2 3 {n} {sh}"))
        return np.stack([self._get(3, k, par) for k in range(n)]), mvm

    def MINRES(self, name, m, err2, inp, par, max_iter=0):
        """MINRES (MINRES.c:160-172) on the hermitian NAME(m), no trial vector."""
        self._slot(2, par)
        self._slot(3, par)
        self._put(2, 0, inp, par)
        self._put(3, 0, np.zeros((self.nsites(par), 4, self.nf)), par)
        mvm = int(self.cmd(f"minres {name} {float(m)!r} {float(err2)!r} {int(max_iter)} 2 3"))
        return self._get(3, 0, par), mvm

    # HMC pieces and IO --------------------------------------------------------
    def momenta_set(self, mom):
        mom = np.ascontiguousarray(mom, np.float64)
        assert mom.shape == (self.V, 4, self.dimg)
        mom.tofile(self._path("mom.bin"))
        self.cmd(f"mom_load {self._path('mom.bin')}")

    def momenta_get(self):
        self.cmd(f"mom_save {self._path('mom.bin')}")
        return np.fromfile(self._path("mom.bin"), np.float64).reshape(self.V, 4, self.dimg)

    def force0(self, dt, beta):
        """force0 (force0.c:22-99, plaquette action): momenta += -dt beta/NG proj(U staples^+)."""
        self.cmd(f"force0 {float(dt)!r} {float(beta)!r}")

    def update_gauge_field(self, dt):
        """update_gauge_field (field_update.c:18-66): U <- ExpX(dt, momenta) U, every 17th
        call reunitarised, then represent_gauge_field."""
        self.cmd(f"update_gauge {float(dt)!r}")

    def write_gauge_field(self, path):
        self.cmd(f"gauge_write {path}")

    def read_gauge_field(self, path):
        self.cmd(f"gauge_read {path}")
