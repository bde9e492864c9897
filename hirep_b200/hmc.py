"""One HMC trajectory on the GPU, driven from the host as HiRep drives it.

update_ghmc (LibHR/Update/update_mt.c:148-260) with two monomials: the
plaquette gauge action (mon_pg.c; force0.c) and an Nf = 2 Wilson pseudofermion
on the even sites (mon_hmc.c; force_hmc.c, UPDATE_EO branch).  The integrator
is HiRep's multilevel scheme (integrators.c): a list of levels, each with an
integrator (leapfrog, O2MN or O4MN), a number of steps and the monomials whose
forces it applies; a level's field update moves the links if the gauge
monomial (which owns update_gauge_field, mon_pg.c:71) sits on it and then runs
the next level for the same time.  The default is one O2MN level with both
monomials.  With a clover term the fermion operator is Cphi_eopre
(D_update.c:26-95) and the clover force is part of force_fermion_core.  The
standard clover monomial also carries the log-det terms of WITH_CLOVER_EO:
clover_la_logdet(2, m) in its local action (mon_hmc.c:60-67) and
force_clover_logdet(m, 2) in its force (force_hmc.c:185-190, logdet = 1 as
mon_hmc.c:109 sets it); the exponential clover term (WITH_EXPCLOVER) has none
(its blocks are traceless, det D_oo is constant).  Links, momenta and
pseudofermions stay on the device; the host only holds the scalars of the
recursion and the random numbers.

The force solves are either HiRep's (two g5QMR solves on D) or, as the
mixed-precision form of this library, one CG on H^2 = (g5 D)^2 (FP64 or FP32
inner defect correction): Ys = (H^2)^-1 pf and Xs = H Ys, the pair that
force_fermion_core expects (for g5QMR: Xs = H^-1 pf, Ys = H^-1 Xs).
"""
import time

import numpy as np

from . import hrgpu as G

LAMBDA_O2MN = 0.1931833275037836
# fourth-order Omelyan-Mryglod-Folk (Comput. Phys. Commun. 151 (2003) 272), in
# the form of Takaishi and de Forcrand (hep-lat/0505020) that integrators.c uses
O4MN_RHO, O4MN_THETA, O4MN_LAMBDA = 0.1786178958448091, -0.06626458266981843, 0.7123418310626056
INTEGRATORS = ("leapfrog", "o2mn", "o4mn")
MONOMIALS = ("gauge", "fermion")


def integrate(kind, nsteps, tlen, force, field):
    """One level of the multilevel integrator (integrators.c:30-132):
    force(dt) kicks the momenta with the level's monomials, field(dt) moves
    the links and runs the next level."""
    if nsteps == 0:
        return
    dt = tlen / nsteps
    if kind == "leapfrog":  # leapfrog_multistep
        for n in range(nsteps):
            force(dt / 2 if n == 0 else dt)
            field(dt)
        force(dt / 2)
    elif kind == "o2mn":  # O2MN_multistep
        lam = LAMBDA_O2MN
        for n in range(nsteps):
            force(lam * dt if n == 0 else 2 * lam * dt)
            field(dt / 2)
            force((1 - 2 * lam) * dt)
            field(dt / 2)
        force(lam * dt)
    elif kind == "o4mn":  # O4MN_multistep
        rho, theta, lam = O4MN_RHO, O4MN_THETA, O4MN_LAMBDA
        for n in range(nsteps):
            force(rho * dt if n == 0 else 2 * rho * dt)
            field(lam * dt)
            force(theta * dt)
            field((0.5 - lam) * dt)
            force((1 - 2 * (theta + rho)) * dt)
            field((0.5 - lam) * dt)
            force(theta * dt)
            field(lam * dt)
        force(rho * dt)
    else:
        raise ValueError(f"integrator {kind!r}: one of {INTEGRATORS}")


class HMC:
    def __init__(self, lat, beta, mass, tau, nsteps, force_err2=1e-20, mt_err2=1e-28, force_solver="cg_mixed",
                 bc_t_antiperiodic=True, levels=None, mre_past=0, draws="host", mt_solver="cg"):
        """levels: [(integrator, nsteps, monomials), ...] from the outermost level
        in; None is [("o2mn", nsteps, ("gauge", "fermion"))].  mre_past > 0: the
        force solves start from the chronological (MRE) guess over that many past
        solutions (mre.c, as force_hmc.c:122-145 uses it); 0: the g5QMR solves
        start from zero and the CG solves from the previous solution.  draws:
        "host" draws the momenta and the pseudofermion source with the numpy
        Generator passed to trajectory(); "device" draws them on the GPU
        (gaussian_momenta, gaussian_spinor_field) with a seed taken from it.
        mt_solver: the accept/reject solve pf <- H^-1 pf (correct_la_pf), FP64 at
        mt_err2: "g5qmr" is HiRep's g5QMR on D with source g5 pf; "cg" solves
        H^2 y = pf and sets pf = H y, the same equation H x = pf with the same
        residual (H x - pf = H^2 y - pf), in about half the hopping-term
        applications on the captured CG iterations."""
        if mt_solver not in ("cg", "g5qmr"):
            raise ValueError("mt_solver: cg or g5qmr")
        self.mt_solver = mt_solver
        if draws not in ("host", "device"):
            raise ValueError("draws: host or device")
        self.draws = draws
        if force_solver not in ("cg_mixed", "cg", "g5qmr"):
            raise ValueError("force_solver: cg_mixed, cg or g5qmr")
        if levels is None:
            levels = [("o2mn", nsteps, MONOMIALS)]
        seen = []
        for kind, n, mons in levels:
            if kind not in INTEGRATORS or n < 0 or any(m not in MONOMIALS for m in mons):
                raise ValueError(f"bad integrator level {(kind, n, mons)}")
            seen += list(mons)
        if sorted(seen) != sorted(MONOMIALS):
            raise ValueError("each monomial (gauge, fermion) must sit on exactly one level")
        self.levels = [(kind, n, tuple(mons)) for kind, n, mons in levels]
        self.mre = lat.mre(mre_past, G.EVEN) if mre_past > 0 else None
        self.lat, self.beta, self.mass, self.tau, self.nsteps = lat, beta, mass, tau, nsteps
        self.force_err2, self.mt_err2, self.force_solver = force_err2, mt_err2, force_solver
        self.bc = bc_t_antiperiodic
        clover = lat.csw is not None
        self.logdet = clover and not lat.expclover
        self.op_d = G.OP_CPHI_EOPRE if clover else G.OP_DPHI_EOPRE
        self.op_h2 = G.OP_G5CPHI_EOPRE_SQ if clover else G.OP_G5DPHI_EOPRE_SQ
        self.apply_h = lat.g5Cphi_eopre if clover else lat.g5Dphi_eopre
        E = G.EVEN
        self.pf, self.x, self.y, self.tmp = (lat.field(E) for _ in range(4))
        self.Xs, self.Ys = lat.field(G.FULL), lat.field(G.FULL)
        self.iters = 0
        self.nforce = 0

    # -- monomial pieces ----------------------------------------------------------
    def _even_into_full(self, full, even):
        full.buf[: even.nbytes].copy_(even.buf)
        full.buf[even.nbytes:].zero_()

    def _solve(self, op, out, src, err2, flt):
        it, ok = self.lat.cg_mshift(op, self.mass, [0.0], err2, src, [out], flt=flt)
        self.iters += it
        if not ok:
            raise G.HRGPUError("HMC: force solve did not converge")

    def fermion_force(self, dt):
        """force_hmc (force_hmc.c:58-195) for the Nf = 2 Wilson monomial, UPDATE_EO."""
        lat = self.lat
        if self.force_solver == "g5qmr":
            # X = H^-1 pf = D^-1 g5 pf, Y = H^-1 X = D^-1 g5 X
            lat.la("g5", self.tmp, self.pf)
            if self.mre:
                self.mre.guess(0, self.x, self.op_d, self.mass, self.tmp)
            else:
                lat.la("zero", self.x)
            it, ok = lat.g5QMR_mshift(self.op_d, self.mass, [0.0], self.force_err2, self.tmp, [self.x])
            if self.mre:
                self.mre.store(0, self.x)
            lat.la("g5", self.tmp, self.x)
            if self.mre:
                self.mre.guess(1, self.y, self.op_d, self.mass, self.tmp)
            else:
                lat.la("zero", self.y)
            it2, ok2 = lat.g5QMR_mshift(self.op_d, self.mass, [0.0], self.force_err2, self.tmp, [self.y])
            if self.mre:
                self.mre.store(1, self.y)
            self.iters += it + it2
            if not (ok and ok2):
                raise G.HRGPUError("HMC: g5QMR force solve did not converge")
            X, Y = self.x, self.y
        else:
            # Y = (H^2)^-1 pf (start from the MRE guess or the previous solution), X = H Y
            if self.mre:
                self.mre.guess(0, self.y, self.op_h2, self.mass, self.pf)
            self._solve(self.op_h2, self.y, self.pf, self.force_err2, self.force_solver == "cg_mixed")
            if self.mre:
                self.mre.store(0, self.y)
            self.apply_h(self.mass, self.x, self.y)
            X, Y = self.x, self.y
        self._even_into_full(self.Xs, X)
        self._even_into_full(self.Ys, Y)
        lat.fermion_force_begin()
        lat.force_fermion_core(self.Xs, self.Ys, 1, dt, 1.0)
        if self.logdet:
            lat.force_clover_logdet(self.mass, 2.0)  # 2 flavours
        lat.fermion_force_end_momenta(dt)
        self.nforce += 1

    def force(self, level, dt):
        """monomial_force (integrators.c:12-19): the forces of the level's monomials."""
        for m in self.levels[level][2]:
            if m == "gauge":
                self.lat.force0(dt, self.beta)
            else:
                self.fermion_force(dt)

    def field(self, level, dt):
        """monomial_field (integrators.c:21-33): update_gauge_field if the gauge
        monomial is on this level, then the next level for the same time."""
        if "gauge" in self.levels[level][2]:
            self.lat.update_gauge_field(dt)
        if level + 1 < len(self.levels):
            self.run_level(level + 1, dt)

    def run_level(self, level, tlen):
        kind, n, _ = self.levels[level]
        integrate(kind, n, tlen, lambda dt: self.force(level, dt), lambda dt: self.field(level, dt))

    def md(self):
        """The molecular dynamics evolution of one trajectory (tau)."""
        self.run_level(0, self.tau)

    # -- one trajectory -------------------------------------------------------------
    def trajectory(self, rng, metropolis=True):
        """update_ghmc: returns dH, acceptance and timings.  rng: numpy Generator."""
        lat = self.lat
        lat.set_dirac_mass(self.mass)
        u_old = lat.gauge_get()
        t0 = time.perf_counter()
        # momenta (random_momenta.c: gauss / sqrt(C(F))) and pseudofermion heatbath
        # (gaussian_spinor_field: gauss / sqrt(2)); the starting action holds |eta|^2
        if self.draws == "device":
            lat.random_seed(int(rng.integers(2**63)))
            lat.gaussian_momenta()
            eta = lat.gaussian_spinor_field(lat.field(G.EVEN))
        else:
            lat.momenta_set(rng.standard_normal((lat.V, 4, lat.dimg)) / np.sqrt(0.5))
            eta_h = (rng.standard_normal((lat.VH, 4, lat.nf)) + 1j * rng.standard_normal((lat.VH, 4, lat.nf))) / np.sqrt(2)
            eta = lat.field(G.EVEN, host=eta_h)
        lat.local_hmc_action(False, self.beta)
        lat.pf_local_action(eta)
        if self.logdet:
            lat.clover_la_logdet(2.0, self.mass)
        self.apply_h(self.mass, self.pf, eta)  # correct_pf: pf = H eta
        lat.la("zero", self.y)
        self.iters = 0
        self.nforce = 0
        self.md()
        lat.project_gauge_field()
        lat.represent_gauge_field(self.bc)
        # correct_la_pf: pf <- H^-1 pf (FP64, MT precision)
        if self.mt_solver == "g5qmr":
            # D^-1 g5 pf by g5QMR, as HiRep
            lat.la("g5", self.tmp, self.pf)
            lat.la("zero", self.pf)
            it, ok = lat.g5QMR_mshift(self.op_d, self.mass, [0.0], self.mt_err2, self.tmp, [self.pf])
        else:
            # H^2 y = pf by CG from zero, then pf = H y
            lat.la("zero", self.tmp)
            it, ok = lat.cg_mshift(self.op_h2, self.mass, [0.0], self.mt_err2, self.pf, [self.tmp])
            self.apply_h(self.mass, self.pf, self.tmp)
        if not ok:
            raise G.HRGPUError("HMC: accept/reject solve did not converge")
        lat.local_hmc_action(True, self.beta)
        lat.pf_local_action(self.pf)
        if self.logdet:
            lat.clover_la_logdet(2.0, self.mass)
        dH = lat.local_action_sum()
        lat.sync()
        t1 = time.perf_counter()
        accepted = True
        if metropolis and dH > 0 and rng.uniform() >= np.exp(-dH):
            accepted = False
            lat.set_gauge(u_old)
            lat.represent_gauge_field(self.bc)
        return {"dH": dH, "accepted": accepted, "seconds": t1 - t0, "force_solve_iters": self.iters,
                "force_evaluations": self.nforce, "mt_iters": it}
