"""Exponential clover (WITH_EXPCLOVER: Dphi.c:1292-1482, LibHR/Utils/clover_exp.c,
force_fermion_core.c:484-772) on the GPU against the oracle: every Cphi operator,
the FP32 and batched forms, a solve, and the force."""
import numpy as np
import pytest

import oracle as O
from hirep_b200 import fields as F
from hirep_b200 import hrgpu as G

pytestmark = pytest.mark.gpu
TOL64 = 1e-13


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def setup(ng, rep, seed=5):
    o = O.Oracle(4, 4, 4, 4, ng, rep)
    u = F.smooth_gauge(seed, o.V, ng, 0.3)
    o.set_gauge(o.represent_gauge_field(u, True))
    o.expclover_init(1.0)
    o.compute_clover_term()
    lat = G.Lattice(4, 4, 4, 4, ng, rep, ipt=o.geometry()[0])
    lat.set_gauge(u)
    lat.represent_gauge_field(True)
    lat.expclover_init(1.0)
    return o, lat


@pytest.mark.parametrize("ng,rep", [(3, O.FUND), (2, O.ADJ), (3, O.SYM), (4, O.ASYM)])
def test_expclover_operators(ng, rep):
    o, lat = setup(ng, rep)
    m = -0.2
    e = F.gaussian_spinor(1, o.VH, o.nf)
    od = F.gaussian_spinor(2, o.VH, o.nf)
    full = F.gaussian_spinor(3, o.V, o.nf)
    fe, fo, ff = lat.field(O.EVEN, host=e), lat.field(O.ODD, host=od), lat.field(O.FULL, host=full)
    out_e, out_o, out_f = lat.field(O.EVEN), lat.field(O.ODD), lat.field(O.FULL)
    for name in ("Cphi_eopre", "g5Cphi_eopre", "g5Cphi_eopre_sq"):
        getattr(lat, name)(m, out_e, fe)
        assert rel(out_e.download(), getattr(o, name)(m, e)) < TOL64, name
    for name in ("Cphi", "g5Cphi_sq"):
        getattr(lat, name)(m, out_f, ff)
        assert rel(out_f.download(), getattr(o, name)(m, full)) < TOL64, name
    lat.Cphi_diag(m, out_o, fo)
    assert rel(out_o.download(), o.Cphi_diag(m, od, O.ODD)) < TOL64
    lat.Cphi_diag_inv(m, out_o, fo)
    assert rel(out_o.download(), o.Cphi_diag_inv(m, od, O.ODD)) < TOL64
    # FP32 operator and the batch kernel read the same packed blocks
    e32 = e.astype(np.complex64)
    f32, o32 = lat.field(O.EVEN, G.FLOAT, host=e32), lat.field(O.EVEN, G.FLOAT)
    lat.g5Cphi_eopre_flt(m, o32, f32)
    assert rel(o32.download(), o.g5Cphi_eopre(m, e32.astype(complex))) < 1e-5
    bi, bo = lat.batch(3, fields=[fe, fe, fe]), lat.batch(3)
    lat.apply_op_batch(G.OP_G5CPHI_EOPRE, m, bo, bi)
    outs = [lat.field(O.EVEN) for _ in range(3)]
    bo.unpack(outs)
    assert rel(outs[2].download(), o.g5Cphi_eopre(m, e)) < TOL64


def test_expclover_solve_and_switch_back():
    o, lat = setup(3, O.FUND, seed=7)
    m = -0.2
    o.set_mass(m)
    b = F.gaussian_spinor(4, o.VH, o.nf)
    xo, _ = o.cg_mshift(G.OP_G5CPHI_EOPRE_SQ, [0.0, 0.1], 1e-26, b)
    fb = lat.field(O.EVEN, host=b)
    outs = [lat.field(O.EVEN) for _ in range(2)]
    it, ok = lat.cg_mshift(G.OP_G5CPHI_EOPRE_SQ, m, [0.0, 0.1], 1e-26, fb, outs, flt=True)
    assert ok
    for i in range(2):
        assert rel(outs[i].download(), xo[i]) < 1e-10
    # back to the standard clover term: the LDL inverse again
    lat.clover_init(1.0)
    o.clover_init(1.0)
    o.compute_clover_term()
    out = lat.field(O.EVEN)
    lat.Cphi_eopre(m, out, fb)
    assert rel(out.download(), o.Cphi_eopre(m, b)) < TOL64


# complex NF 3, 6, 6, 10; real NF 3, 8 and 15 (the last one with 100 KB of
# shared memory per site block)
@pytest.mark.parametrize("ng,rep", [(3, O.FUND), (3, O.SYM), (4, O.ASYM), (4, O.SYM), (2, O.ADJ), (3, O.ADJ),
                                    (4, O.ADJ)])
def test_expclover_force_matches_oracle(ng, rep):
    """force_fermion_core with the exponential clover term (force_fermion_core.c:484-772):
    the odd-site fill with exp(-A/(4+m))/(4+m), the force matrices by the Frechet
    derivative of the exponential, and the six-leaf clover derivative."""
    o, lat = setup(ng, rep, seed=9)
    m = -0.1
    o.set_mass(m)
    lat.set_dirac_mass(m)
    X = F.gaussian_spinor(11, o.V, o.nf)
    Y = F.gaussian_spinor(12, o.V, o.nf)
    o.fermion_force_begin()
    Xo, Yo = o.force_fermion_core(X, Y, 1, 0.7, 1.3)
    lat.fermion_force_begin()
    fX, fY = lat.field(O.FULL, host=X), lat.field(O.FULL, host=Y)
    lat.force_fermion_core(fX, fY, 1, 0.7, 1.3)
    assert rel(fX.download(), Xo) < TOL64
    assert rel(fY.download(), Yo) < TOL64
    # no log-det force: det D_oo is constant for the exponential form
    o.force_clover_logdet(m, 0.4)
    lat.force_clover_logdet(m, 0.4)
    mom = np.zeros((o.V, 4, o.dimg))
    fo = o.fermion_force_end(0.7, mom.copy())
    fg = lat.fermion_force_end(0.7, mom.copy())
    assert rel(fg, fo) < 1e-12


@pytest.mark.parametrize("ng", [2, 3])
def test_expclover_force_matrices_two_forms(ng):
    """TestProgram/Update/check_update_2 restated: the exponential clover force
    matrices cl_force from Z2 volume sources, computed two ways - the oracle's
    Taylor form (force_clover_fermion_taylor) and the device's Frechet
    derivative by scaling and squaring - agree to an RMS of 1e-14 per element
    (the reference's bound), SU(2) and SU(3) fundamental as there."""
    o, lat = setup(ng, O.FUND, seed=23)
    m = -0.5
    o.set_mass(m)
    lat.set_dirac_mass(m)
    rng = np.random.default_rng(ng)

    def z2():
        return ((rng.integers(0, 2, (o.V, 4, o.nf)) * 2 - 1) + 1j * (rng.integers(0, 2, (o.V, 4, o.nf)) * 2 - 1)) / np.sqrt(2)

    X, Y = z2(), z2()
    o.fermion_force_begin()
    o.force_fermion_core(X, Y, 0, 1.0, 1.0)
    lat.fermion_force_begin()
    lat.force_fermion_core(lat.field(O.FULL, host=X), lat.field(O.FULL, host=Y), 0, 1.0, 1.0)
    d = lat.clover_force() - o.clover_force().reshape(o.V, 6, o.nf, o.nf)
    assert np.sqrt(np.sum(np.abs(d) ** 2) / (o.V * 6 * o.nf * o.nf)) < 1e-14
