"""An HMC trajectory driven entirely by the oracle: update_ghmc
(LibHR/Update/update_mt.c:148-260) with the plaquette monomial and an Nf=2
Wilson, clover (with its log-det terms) or exponential clover pseudofermion on
the even sites, with HiRep's multilevel leapfrog / O2MN / O4MN integrators
(integrators.c:12-132).  Test infrastructure: the GPU driver's trajectories are
checked against it, and its own dH ~ dt^2 (dt^4 for O4MN) pins the oracle's
forces and the integrator coefficients."""
import numpy as np

import oracle as O

# integrators.c:64-132
_O2MN_L = 0.1931833275037836
_O4MN = (0.1786178958448091, -0.06626458266981843, 0.7123418310626056)


def _level(kind, nsteps, tlen, kick, move):
    """One integrator level: kick(dt) applies the level's forces, move(dt) the
    field update and the next level."""
    if nsteps == 0:
        return
    dt = tlen / nsteps
    if kind == "leapfrog":
        seq = [("k", 0.5), ("m", 1.0)]
        tail = [("k", 0.5)]
        merge = 1.0
    elif kind == "o2mn":
        lam = _O2MN_L
        seq = [("k", lam), ("m", 0.5), ("k", 1 - 2 * lam), ("m", 0.5)]
        tail = [("k", lam)]
        merge = 2 * lam
    else:
        rho, theta, lam = _O4MN
        seq = [("k", rho), ("m", lam), ("k", theta), ("m", 0.5 - lam), ("k", 1 - 2 * (theta + rho)),
               ("m", 0.5 - lam), ("k", theta), ("m", lam)]
        tail = [("k", rho)]
        merge = 2 * rho
    for n in range(nsteps):
        for j, (what, c) in enumerate(seq):
            if what == "k":
                kick((merge if (j == 0 and n > 0) else c) * dt)  # the end kick of step n-1 merged in
            else:
                move(c * dt)
    for what, c in tail:
        kick(c * dt)


def oracle_trajectory(o, u0, beta, mass, tau, nsteps, rng, force_err2, mt_err2, expclover_csw=None, clover_csw=None,
                      levels=None):
    """update_ghmc with the plaquette and Nf=2 Wilson (or clover) monomials,
    every piece from the oracle (the same random numbers as
    hirep_b200.hmc.HMC.trajectory).  levels: [(integrator, nsteps, monomials)],
    default one O2MN level with both monomials."""
    if levels is None:
        levels = [("o2mn", nsteps, ("gauge", "fermion"))]
    V, VH, nf, dimg = o.V, o.VH, o.nf, o.dimg
    g5 = np.array([1, 1, -1, -1])[None, :, None]
    keep = {}
    clover = expclover_csw is not None or clover_csw is not None
    logdet = clover_csw is not None  # the standard clover monomial's log-det terms
    if expclover_csw is not None:
        o.expclover_init(expclover_csw)
    elif clover_csw is not None:
        o.clover_init(clover_csw)
    op_h2 = O.OP_G5CPHI_EOPRE_SQ if clover else O.OP_G5DPHI_EOPRE_SQ
    op_d = O.OP_CPHI_EOPRE if clover else O.OP_DPHI_EOPRE
    apply_h = o.g5Cphi_eopre if clover else o.g5Dphi_eopre

    def represent(u):
        keep["uf"] = o.represent_gauge_field(u, True)
        o.set_gauge(keep["uf"])
        if clover:
            o.compute_clover_term()

    u = u0.copy()
    represent(u)
    o.set_mass(mass)
    mom = rng.standard_normal((V, 4, dimg)) / np.sqrt(0.5)
    eta = (rng.standard_normal((VH, 4, nf)) + 1j * rng.standard_normal((VH, 4, nf))) / np.sqrt(2)
    def logdet_action():
        return o.clover_la_logdet(2.0, mass, np.zeros(V)).sum() if logdet else 0.0

    H0 = o.local_hmc_action(beta, u, mom).sum() + np.sum(np.abs(eta) ** 2) + logdet_action()
    pf = apply_h(mass, eta)
    st = {"y": np.zeros_like(eta), "count": 0, "u": u, "mom": mom}

    def gauge_force(dt):
        st["mom"] = o.force0(dt, beta, st["u"], st["mom"])

    def fermion_force(dt):
        y, _ = o.cg_mshift(op_h2, [0.0], force_err2, pf, guess=st["y"])
        st["y"] = y[0]
        x = apply_h(mass, st["y"])
        Xs = np.zeros((V, 4, nf), complex)
        Ys = np.zeros_like(Xs)
        Xs[:VH], Ys[:VH] = x, st["y"]
        o.fermion_force_begin()
        o.force_fermion_core(Xs, Ys, 1, dt, 1.0)
        if logdet:
            o.force_clover_logdet(mass, 2.0)
        st["mom"] = o.fermion_force_end(dt, st["mom"])

    def field(dt):
        st["u"] = o.update_gauge_field(dt, st["u"], st["mom"])
        if st["count"] & 16:  # field_update.c:45-57
            st["count"] = 0
            st["u"] = o.project_gauge_field(st["u"])
        else:
            st["count"] += 1
        represent(st["u"])

    def run(i, tlen):
        kind, n, mons = levels[i]

        def kick(dt):
            for m in mons:
                (gauge_force if m == "gauge" else fermion_force)(dt)

        def move(dt):
            if "gauge" in mons:
                field(dt)
            if i + 1 < len(levels):
                run(i + 1, dt)

        _level(kind, n, tlen, kick, move)

    run(0, tau)
    st["u"] = o.project_gauge_field(st["u"])
    represent(st["u"])
    xo, _ = o.g5QMR_mshift(op_d, [0.0], mt_err2, g5 * pf)
    H1 = o.local_hmc_action(beta, st["u"], st["mom"]).sum() + np.sum(np.abs(xo[0]) ** 2) + logdet_action()
    return H1 - H0, st["u"]
