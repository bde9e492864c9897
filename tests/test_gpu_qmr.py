"""g5QMR_mshift, MINRES and the MRE initial guess on the GPU against the oracle
(LibHR/Inverters/g5QMR_mshift.c, MINRES.c, LibHR/Update/mre.c; the reference's
own checks are check_inverters_2.c and check_inverters_3.c)."""
import ctypes

import numpy as np
import pytest

import oracle as O
from hirep_b200 import fields as F
from hirep_b200 import hrgpu as G

pytestmark = pytest.mark.gpu

SHIFTS6 = [0.1, -0.21, 0.05, -0.01, -0.15, -0.05]


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def setup(ng=3, rep=O.FUND, hot=True, clover=False, dims=(4, 4, 4, 4), seed=1234):
    o = O.Oracle(*dims, ng, rep)
    u = F.hot_gauge(seed, o.V, ng) if hot else F.smooth_gauge(seed, o.V, ng, 0.3)
    o.set_gauge(o.represent_gauge_field(u, True))
    lat = G.Lattice(*dims, ng, rep, ipt=o.geometry()[0])
    lat.set_gauge(u)
    lat.represent_gauge_field(True)
    if clover:
        o.clover_init(1.0)
        o.compute_clover_term()
        lat.clover_init(1.0)
    return o, lat


@pytest.mark.parametrize("op,clover", [(G.OP_DPHI_EOPRE, False), (G.OP_DPHI, False), (G.OP_CPHI_EOPRE, True)])
def test_g5qmr_six_shifts_match_oracle(op, clover):
    o, lat = setup(clover=clover, hot=not clover)
    m = 0.1
    o.set_mass(m)
    par = O.FULL if op == G.OP_DPHI else O.EVEN
    b = F.gaussian_spinor(5, o.nsites(par), o.nf)
    err2 = 1e-26
    shifts = SHIFTS6 if not clover else [0.0, -0.1, 0.05]
    xo, it_o = o.g5QMR_mshift(op, shifts, err2, b)
    fb = lat.field(par, host=b)
    outs = [lat.field(par) for _ in shifts]
    it, ok = lat.g5QMR_mshift(op, m, shifts, err2, fb, outs)
    assert ok
    Dop = {G.OP_DPHI_EOPRE: o.Dphi_eopre, G.OP_DPHI: o.Dphi, G.OP_CPHI_EOPRE: o.Cphi_eopre}[op]
    for i, s in enumerate(shifts):
        x = outs[i].download()
        r = Dop(m, x) - s * x - b
        assert o.sqnorm(r) / o.sqnorm(b) < err2, (i, s)
        assert rel(x, xo[i]) < 1e-8
    assert it > 0 and abs(it - it_o) <= max(3, it_o // 20), (it, it_o)


def test_g5qmr_single_shift_from_initial_guess():
    o, lat = setup(hot=False, seed=7)
    m = 0.1
    o.set_mass(m)
    b = F.gaussian_spinor(6, o.VH, o.nf)
    guess = 0.5 * F.gaussian_spinor(7, o.VH, o.nf)
    xo, it_o = o.g5QMR_mshift(G.OP_DPHI_EOPRE, [0.0], 1e-26, b, guess=guess)
    fb, x = lat.field(O.EVEN, host=b), lat.field(O.EVEN, host=guess)
    it, ok = lat.g5QMR_mshift(G.OP_DPHI_EOPRE, m, [0.0], 1e-26, fb, [x])
    assert ok
    assert rel(x.download(), xo[0]) < 1e-8
    assert abs(it - it_o) <= 3


def test_minres_matches_oracle():
    o, lat = setup(hot=True)
    m = 0.1
    o.set_mass(m)
    b = F.gaussian_spinor(8, o.VH, o.nf)
    err2 = 1e-26
    xo, _ = o.MINRES(O.OP_G5DPHI_EOPRE, err2, b)
    fb, x = lat.field(O.EVEN, host=b), lat.field(O.EVEN)
    it, ok = lat.MINRES(G.OP_G5DPHI_EOPRE, m, err2, fb, x)
    assert ok
    r = o.g5Dphi_eopre(m, x.download()) - b
    assert o.sqnorm(r) / o.sqnorm(b) < err2
    assert rel(x.download(), xo) < 1e-8
    # from a trial vector
    trial = lat.field(O.EVEN, host=xo + 1e-3 * F.gaussian_spinor(9, o.VH, o.nf))
    x2 = lat.field(O.EVEN)
    it2, ok2 = lat.MINRES(G.OP_G5DPHI_EOPRE, m, err2, fb, x2, trial=trial)
    assert ok2 and it2 < it


def test_mre_guess_matches_oracle():
    o, lat = setup(hot=False, seed=3)
    m = 0.1
    o.set_mass(m)
    sols = [F.gaussian_spinor(20 + k, o.VH, o.nf) for k in range(7)]
    pf = F.gaussian_spinor(30, o.VH, o.nf)
    h = lat.mre(5, O.EVEN)
    try:
        out = lat.field(O.EVEN)
        h.guess(0, out, G.OP_DPHI_EOPRE, m, lat.field(O.EVEN, host=pf))
        assert np.abs(out.download()).max() == 0  # nothing stored yet
        for s in sols:  # keeps the 5 newest, newest first
            h.store(0, lat.field(O.EVEN, host=s))
        h.guess(0, out, G.OP_DPHI_EOPRE, m, lat.field(O.EVEN, host=pf))
        ref = o.mre_guess(O.OP_DPHI_EOPRE, sols[::-1][:5], pf)
        assert rel(out.download(), ref) < 1e-11
        # sequence 1 is separate
        h.guess(1, out, G.OP_DPHI_EOPRE, m, lat.field(O.EVEN, host=pf))
        assert np.abs(out.download()).max() == 0
    finally:
        h.free()


def test_qmr_argument_errors():
    o, lat = setup(hot=False)
    L, D = lat.L, ctypes.c_double
    f, g = lat.field(O.EVEN), lat.field(O.EVEN)
    arr = (ctypes.c_void_p * 1)(g.ptr.value)
    sh = np.zeros(1)
    it = ctypes.c_int()
    # the positive CG operators are not Dirac operators D
    assert L.hrgpu_g5QMR_mshift(G.OP_G5DPHI_EOPRE_SQ, D(0.1), 1, G._ptr(sh), D(1e-20), 0, f.ptr, arr,
                                ctypes.byref(it)) == 2
    # a zero source has a zero gamma_5 norm: refused, not a fault
    assert L.hrgpu_g5QMR_mshift(G.OP_DPHI_EOPRE, D(0.1), 1, G._ptr(sh), D(1e-20), 0, f.ptr, arr,
                                ctypes.byref(it)) == 2
    assert "gamma_5 norm" in L.hrgpu_last_error().decode()
    assert L.hrgpu_MINRES(G.OP_DPHI_EOPRE, D(0.1), D(1e-20), 0, f.ptr, g.ptr, None, ctypes.byref(it)) == 2
    assert lat.L.hrgpu_mre_init(0, 0) is None
