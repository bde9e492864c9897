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
