"""Gauge-side HMC pieces on the GPU against the oracle: force0 with staples,
update_gauge_field (ExpX and the reunitarisation of every 17th call), the
local HMC action, the plaquette, and the fermion force added to the device
momenta (LibHR/Update/force0.c, staples.c, field_update.c, local_action.c,
LibHR/Utils/suN_utils.c, LibHR/Observables/avr_plaquette.c)."""
import numpy as np
import pytest

import oracle as O
from hirep_b200 import fields as F
from hirep_b200 import hrgpu as G
from hmc_oracle import oracle_trajectory as _oracle_trajectory

pytestmark = pytest.mark.gpu


def setup(ng, rep=O.FUND, seed=4, eps=0.4, dims=(4, 4, 4, 4)):
    o = O.Oracle(*dims, ng, rep)
    u = F.smooth_gauge(seed, o.V, ng, eps)
    o.set_gauge(o.represent_gauge_field(u, True))
    lat = G.Lattice(*dims, ng, rep, ipt=o.geometry()[0])
    lat.set_gauge(u)
    lat.represent_gauge_field(True)
    mom = np.random.default_rng(seed + 1).standard_normal((o.V, 4, ng * ng - 1))
    lat.momenta_set(mom)
    return o, lat, u, mom


@pytest.mark.parametrize("ng", [2, 3, 4])
def test_force0_matches_oracle(ng):
    o, lat, u, mom = setup(ng)
    assert np.array_equal(lat.momenta_get(), mom)
    lat.force0(0.1, 2.25)
    ref = o.force0(0.1, 2.25, u, mom)
    assert np.abs(lat.momenta_get() - ref).max() < 1e-13


@pytest.mark.parametrize("ng", [2, 3])
def test_update_gauge_field_and_reunitarisation(ng):
    o, lat, u, mom = setup(ng, seed=6)
    uo = u.copy()
    dt = 0.02
    for k in range(17):  # the 17th call reunitarises (field_update.c:45-57)
        lat.update_gauge_field(dt)
        uo = o.update_gauge_field(dt, uo, mom)
        if k < 16:
            assert np.abs(lat.gauge_get() - uo).max() < 1e-13 * (k + 1)
    uo = o.project_gauge_field(uo)
    ug = lat.gauge_get()
    assert np.abs(ug - uo).max() < 1e-12
    m = ug.reshape(-1, ng, ng)
    assert np.abs(np.einsum("kij,klj->kil", m, m.conj()) - np.eye(ng)).max() < 1e-14
    # the represented links followed: the Dirac operator sees the updated field
    o.set_gauge(o.represent_gauge_field(uo, True))
    e = F.gaussian_spinor(3, o.VH, o.nf)
    fe, out = lat.field(O.EVEN, host=e), lat.field(O.EVEN)
    lat.Dphi_eopre(0.1, out, fe)
    ref = o.Dphi_eopre(0.1, e)
    assert np.abs(out.download() - ref).max() / np.abs(ref).max() < 1e-13


def test_local_action_plaquette_and_pf():
    o, lat, u, mom = setup(3, seed=8)
    beta = 5.5
    lat.local_hmc_action(False, beta)
    ref = o.local_hmc_action(beta, u, mom)
    assert np.abs(lat.local_action() - ref).max() < 1e-11
    assert lat.local_action_sum() == pytest.approx(ref.sum(), rel=1e-13)
    assert lat.avr_plaquette() == pytest.approx(o.avr_plaquette(u), rel=1e-13)
    # DELTA after a change of the momenta: new minus old per site
    mom2 = mom * 0.5
    lat.momenta_set(mom2)
    lat.local_hmc_action(True, beta)
    ref2 = o.local_hmc_action(beta, u, mom2) - ref
    assert np.abs(lat.local_action() - ref2).max() < 1e-11
    # pseudofermion term on the even sites
    pf = F.gaussian_spinor(9, o.VH, o.nf)
    lat.pf_local_action(lat.field(O.EVEN, host=pf))
    loc = lat.local_action()
    add = np.zeros(o.V)
    add[: o.VH] = np.sum(np.abs(pf) ** 2, axis=(1, 2))
    assert np.abs(loc - (ref2 + add)).max() < 1e-11


def test_fermion_force_into_device_momenta():
    o, lat, u, mom = setup(2, rep=O.ADJ, seed=10)
    X = F.gaussian_spinor(11, o.V, o.nf)
    Y = F.gaussian_spinor(12, o.V, o.nf)
    fX, fY = lat.field(O.FULL, host=X), lat.field(O.FULL, host=Y)
    lat.fermion_force_begin()
    lat.force_fermion_core(fX, fY, 0, 0.1, 1.0)
    host = lat.fermion_force_end(0.1, mom)
    lat.fermion_force_end_momenta(0.1)
    assert np.abs(lat.momenta_get() - host).max() < 1e-14


def test_hmc_trajectory_matches_oracle_trajectory():
    """One O2MN trajectory (10 steps, 20 link updates: one reunitarisation) of the
    SU(2) adjoint Nf=2 Wilson + plaquette system: dH and the final links."""
    from hirep_b200.hmc import HMC

    dims, ng, beta, mass = (4, 4, 4, 4), 2, 2.25, -1.0
    o = O.Oracle(*dims, ng, O.ADJ)
    u0 = F.smooth_gauge(99, o.V, ng, 0.2)
    lat = G.Lattice(*dims, ng, G.ADJ, ipt=o.geometry()[0])
    lat.set_gauge(u0)
    lat.represent_gauge_field(True)
    hmc = HMC(lat, beta, mass, tau=0.5, nsteps=10, force_err2=1e-26, mt_err2=1e-28, force_solver="cg")
    res = hmc.trajectory(np.random.default_rng(5), metropolis=False)
    dH_o, u_o = _oracle_trajectory(o, u0, beta, mass, 0.5, 10, np.random.default_rng(5), 1e-26, 1e-28)
    assert abs(res["dH"] - dH_o) < 1e-8 * max(1.0, abs(dH_o)), (res["dH"], dH_o)
    assert np.abs(lat.gauge_get() - u_o).max() < 1e-10
    assert res["force_evaluations"] == 2 * 10 + 1  # O2MN: two per step and a last one


def test_hmc_expclover_trajectory_matches_oracle_trajectory():
    """The same with Nf=2 exponential clover fermions (WITH_EXPCLOVER, csw=1.2),
    SU(3) fundamental: the clover term rebuilt after every link update, the
    force with the exponential's derivative, no log-det term."""
    from hirep_b200.hmc import HMC

    dims, ng, beta, mass, csw = (4, 4, 4, 4), 3, 5.6, -0.3, 1.2
    o = O.Oracle(*dims, ng, O.FUND)
    u0 = F.smooth_gauge(98, o.V, ng, 0.2)
    lat = G.Lattice(*dims, ng, G.FUND, ipt=o.geometry()[0])
    lat.set_gauge(u0)
    lat.represent_gauge_field(True)
    lat.expclover_init(csw)
    hmc = HMC(lat, beta, mass, tau=0.5, nsteps=8, force_err2=1e-26, mt_err2=1e-28, force_solver="cg")
    res = hmc.trajectory(np.random.default_rng(15), metropolis=False)
    dH_o, u_o = _oracle_trajectory(o, u0, beta, mass, 0.5, 8, np.random.default_rng(15), 1e-26, 1e-28,
                                   expclover_csw=csw)
    assert abs(res["dH"] - dH_o) < 1e-8 * max(1.0, abs(dH_o)), (res["dH"], dH_o)
    assert np.abs(lat.gauge_get() - u_o).max() < 1e-10


def test_clover_la_logdet_matches_oracle():
    """The standard clover monomial's log-det local action (clover_tools.c:312-331)."""
    o, lat, u, mom = setup(3, O.SYM, seed=6, eps=0.3)
    m, csw = -0.3, 1.1
    o.clover_init(csw)
    o.compute_clover_term()
    lat.clover_init(csw)
    lat.local_hmc_action(False, 5.6)
    lat.clover_la_logdet(2.0, m)
    la_o = o.clover_la_logdet(2.0, m, o.local_hmc_action(5.6, u, mom))
    la_g = lat.local_action()
    assert np.abs(la_g - la_o).max() < 1e-12 * np.abs(la_o).max()
    lat.expclover_init(csw)
    with pytest.raises(G.HRGPUError, match="no log-det term"):
        lat.clover_la_logdet(2.0, m)


def test_hmc_clover_logdet_trajectory_matches_oracle_trajectory():
    """Nf=2 standard clover fermions with the log-det terms in the action and
    the force (WITH_CLOVER_EO: mon_hmc.c:60-67, force_hmc.c:185-190), SU(3)
    fundamental, csw=1.2: dH and the final links against the oracle-driven one."""
    from hirep_b200.hmc import HMC

    dims, ng, beta, mass, csw = (4, 4, 4, 4), 3, 5.6, -0.3, 1.2
    o = O.Oracle(*dims, ng, O.FUND)
    u0 = F.smooth_gauge(97, o.V, ng, 0.2)
    lat = G.Lattice(*dims, ng, G.FUND, ipt=o.geometry()[0])
    lat.set_gauge(u0)
    lat.represent_gauge_field(True)
    lat.clover_init(csw)
    hmc = HMC(lat, beta, mass, tau=0.5, nsteps=8, force_err2=1e-26, mt_err2=1e-28, force_solver="cg")
    res = hmc.trajectory(np.random.default_rng(16), metropolis=False)
    dH_o, u_o = _oracle_trajectory(o, u0, beta, mass, 0.5, 8, np.random.default_rng(16), 1e-26, 1e-28,
                                   clover_csw=csw)
    assert abs(res["dH"] - dH_o) < 1e-8 * max(1.0, abs(dH_o)), (res["dH"], dH_o)
    assert np.abs(lat.gauge_get() - u_o).max() < 1e-10


def test_hmc_nested_o4mn_trajectory_matches_oracle_trajectory():
    """Two integrator levels as HiRep nests them (integrators.c:21-33): O4MN with
    the fermion monomial outside, O4MN with the gauge monomial (and the link
    updates) inside; clover with log-det terms.  dH and the final links against
    the oracle-driven trajectory."""
    from hirep_b200.hmc import HMC

    dims, ng, beta, mass, csw = (4, 4, 4, 4), 2, 6.0, -0.8, 1.0
    levels = [("o4mn", 3, ("fermion",)), ("o4mn", 4, ("gauge",))]
    o = O.Oracle(*dims, ng, O.ADJ)
    u0 = F.smooth_gauge(41, o.V, ng, 0.3)
    lat = G.Lattice(*dims, ng, G.ADJ, ipt=o.geometry()[0])
    lat.set_gauge(u0)
    lat.represent_gauge_field(True)
    lat.clover_init(csw)
    hmc = HMC(lat, beta, mass, tau=0.2, nsteps=0, force_err2=1e-26, mt_err2=1e-28, force_solver="cg", levels=levels)
    res = hmc.trajectory(np.random.default_rng(17), metropolis=False)
    dH_o, u_o = _oracle_trajectory(o, u0, beta, mass, 0.2, 0, np.random.default_rng(17), 1e-26, 1e-28,
                                   clover_csw=csw, levels=levels)
    assert abs(res["dH"] - dH_o) < 1e-8 * max(1.0, abs(dH_o)), (res["dH"], dH_o)
    assert np.abs(lat.gauge_get() - u_o).max() < 1e-10
    assert res["force_evaluations"] == 4 * 3 + 1  # O4MN: four fermion kicks a step and a last one


def test_md_reversibility():
    """TestProgram/Update/check_update_1 restated: from a random (hot) start on
    8x4^3 (SU(2) adjoint, clover csw=1.0 with log-det terms, m0=-0.8, beta=6.0),
    tau=0.2 with O4MN/O4MN nested 10/10, then the momenta flipped and the same
    evolution again: the plaquette returns to 1e-10 (the reference's bound)."""
    from hirep_b200.hmc import HMC

    dims, ng = (8, 4, 4, 4), 2
    lat = G.Lattice(*dims, ng, G.ADJ)
    lat.set_gauge(F.hot_gauge(35563, lat.V, ng))
    lat.represent_gauge_field(True)
    lat.clover_init(1.0)
    hmc = HMC(lat, 6.0, -0.8, tau=0.2, nsteps=0, force_err2=1e-26, force_solver="cg",
              levels=[("o4mn", 10, ("fermion",)), ("o4mn", 10, ("gauge",))])
    rng = np.random.default_rng(3)
    lat.set_dirac_mass(-0.8)
    u0, plaq0 = lat.gauge_get(), lat.avr_plaquette()
    lat.momenta_set(rng.standard_normal((lat.V, 4, lat.dimg)) / np.sqrt(0.5))
    eta = lat.field(G.EVEN, host=(rng.standard_normal((lat.VH, 4, lat.nf))
                                  + 1j * rng.standard_normal((lat.VH, 4, lat.nf))) / np.sqrt(2))
    hmc.apply_h(-0.8, hmc.pf, eta)
    lat.la("zero", hmc.y)
    hmc.md()
    plaq1 = lat.avr_plaquette()
    lat.momenta_set(-lat.momenta_get())  # flip_mom (update_mt.c:310)
    hmc.md()
    assert abs(plaq1 - plaq0) > 1e-3  # the evolution moved the links
    assert abs(lat.avr_plaquette() - plaq0) < 1e-10
    assert np.abs(lat.gauge_get() - u0).max() < 1e-8


@pytest.mark.parametrize("solver", ["cg", "g5qmr"])
def test_hmc_mre_guess_changes_no_trajectory(solver):
    """Force solves started from the MRE chronological guess (mre.c; force_hmc.c:
    122-145) end at the same trajectory to solver tolerance and take fewer MVMs."""
    from hirep_b200.hmc import HMC

    dims, ng, beta, mass = (4, 4, 4, 4), 2, 2.25, -1.0
    u0 = F.smooth_gauge(99, 256, ng, 0.2)
    out = {}
    for mre in (0, 3):
        lat = G.Lattice(*dims, ng, G.ADJ)
        lat.set_gauge(u0)
        lat.represent_gauge_field(True)
        hmc = HMC(lat, beta, mass, tau=0.5, nsteps=10, force_err2=1e-24, force_solver=solver, mre_past=mre)
        r = hmc.trajectory(np.random.default_rng(6), metropolis=False)
        out[mre] = (r["dH"], r["force_solve_iters"], lat.gauge_get())
    assert abs(out[3][0] - out[0][0]) < 1e-7 * max(1.0, abs(out[0][0]))
    assert np.abs(out[3][2] - out[0][2]).max() < 1e-9
    assert out[3][1] < out[0][1]


@pytest.mark.parametrize("solver", ["cg_mixed", "g5qmr"])
def test_hmc_force_solver_forms_agree(solver):
    from hirep_b200.hmc import HMC

    dims, ng, beta, mass = (4, 4, 4, 4), 2, 2.25, -1.0
    u0 = F.smooth_gauge(99, 256, ng, 0.2)
    out = {}
    for s in ("cg", solver):
        lat = G.Lattice(*dims, ng, G.ADJ)
        lat.set_gauge(u0)
        lat.represent_gauge_field(True)
        hmc = HMC(lat, beta, mass, tau=0.5, nsteps=10, force_err2=1e-24, force_solver=s)
        out[s] = hmc.trajectory(np.random.default_rng(6), metropolis=False)["dH"]
    assert abs(out[solver] - out["cg"]) < 1e-7 * max(1.0, abs(out["cg"]))


def test_hmc_energy_violation_scales_as_dt_squared():
    """Full system (plaquette + Nf=2 Wilson): O2MN's dH falls as dt^2, so the
    forces, the momenta's kinetic term and the actions are consistent."""
    from hirep_b200.hmc import HMC

    dims, ng, beta, mass = (4, 4, 4, 4), 2, 2.25, -1.0
    u0 = F.smooth_gauge(7, 256, ng, 0.3)
    dh = {}
    for n in (16, 32):
        lat = G.Lattice(*dims, ng, G.ADJ)
        lat.set_gauge(u0)
        lat.represent_gauge_field(True)
        hmc = HMC(lat, beta, mass, tau=0.5, nsteps=n, force_err2=1e-26, force_solver="cg")
        dh[n] = hmc.trajectory(np.random.default_rng(8), metropolis=False)["dH"]
    assert 3.5 < dh[16] / dh[32] < 4.5, dh  # the oracle trajectory gives 3.97 here


def test_hmc_accept_reject_solver_forms_agree():
    """correct_la_pf as HiRep's g5QMR on D and as CG on H^2 followed by H: the
    same equation H x = pf to the same residual, so the same dH (clover, so
    that both the log-det and the operator enter)."""
    from hirep_b200.hmc import HMC

    dims, ng, beta, mass = (4, 4, 4, 4), 3, 5.6, -0.3
    u0 = F.smooth_gauge(97, 256, ng, 0.2)
    out = {}
    for s in ("g5qmr", "cg"):
        lat = G.Lattice(*dims, ng, G.FUND)
        lat.set_gauge(u0)
        lat.represent_gauge_field(True)
        lat.clover_init(1.2)
        hmc = HMC(lat, beta, mass, tau=0.5, nsteps=10, force_err2=1e-24, mt_err2=1e-28, force_solver="cg",
                  mt_solver=s)
        out[s] = hmc.trajectory(np.random.default_rng(6), metropolis=False)["dH"]
    assert abs(out["cg"] - out["g5qmr"]) < 1e-9 * max(1.0, abs(out["g5qmr"])), out
