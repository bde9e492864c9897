"""Failure paths of the inverters, made on the host: fields prepared so that
the solver must fail, never a GPU fault.  HiRep's cg_mshift has no error path
(it logs non-convergence and loops on a breakdown, LibHR/Inverters/cg_mshift.c);
here a NaN source, a singular system and a shift that makes the system
singular return HRGPU_E_BREAKDOWN (fatal: the solution is garbage), distinct
from HRGPU_E_NOCONV (max_iter reached, not fatal), and a zero source returns
the zero solution.

The singular systems are exact: with unit links, periodic boundary conditions
and a source of ones on the even sites, every hop of a constant spinor sums to
exactly 8 x the spinor (-1/2 x 8 = -4 per Dphi_), so Dphi_eopre(m) psi =
((4+m)^2 - 16) psi with no rounding: at m = 0 H^2 has psi in its kernel
(<k, M k> = 0 at the first step), at m = -2 psi is an eigenvector of H^2 with
eigenvalue 144 and the shift 144 makes (H^2 - 144) singular on it (there the
solver may also stop at max_iter: the test asks only that it does not report
success).
"""
import numpy as np
import pytest

from hirep_b200 import hrgpu as G

pytestmark = pytest.mark.gpu

DIMS = (4, 4, 4, 4)


def unit_lattice():
    lat = G.Lattice(*DIMS, 3, G.FUND)
    u = np.zeros((lat.V, 4, 3, 3), np.complex128)
    u[:, :, range(3), range(3)] = 1.0
    lat.set_gauge(u)
    lat.represent_gauge_field(False)  # periodic in time: the constant spinor is an exact eigenvector
    return lat


def ones(lat):
    return np.ones((lat.VH, 4, lat.nf), np.complex128)


def status_of(exc):
    return int(str(exc).split("status ")[1].split(":")[0])


def test_constant_mode_is_exact():
    lat = unit_lattice()
    fin, out = lat.field(G.EVEN, host=ones(lat)), lat.field(G.EVEN)
    lat.g5Dphi_eopre_sq(-2.0, out, fin)
    assert np.array_equal(out.download(), 144.0 * ones(lat))
    lat.Dphi_eopre(0.0, out, fin)
    assert np.array_equal(out.download(), 0.0 * ones(lat))


@pytest.mark.parametrize("flt", [False, True])
def test_nan_source_is_a_breakdown(flt):
    lat = unit_lattice()
    src = ones(lat)
    src[5, 2, 1] = np.nan
    fin, x = lat.field(G.EVEN, host=src), lat.field(G.EVEN)
    with pytest.raises(G.HRGPUError, match="not finite") as e:
        lat.cg_mshift(G.OP_G5DPHI_EOPRE_SQ, 0.3, [0.0], 1e-20, fin, [x], max_iter=200, flt=flt)
    assert status_of(e.value) == G.E_BREAKDOWN


def test_nan_source_in_a_batch_is_a_breakdown():
    lat = unit_lattice()
    good = lat.field(G.EVEN, host=ones(lat))
    src = ones(lat)
    src[0, 0, 0] = np.inf
    bad = lat.field(G.EVEN, host=src)
    outs = [lat.field(G.EVEN) for _ in range(2)]
    for flt in (False, True):
        with pytest.raises(G.HRGPUError, match="not finite") as e:
            lat.cg_mshift_batch(G.OP_G5DPHI_EOPRE_SQ, 0.3, [good, bad], [[0.0], [0.0]], 1e-20, outs, flt=flt)
        assert status_of(e.value) == G.E_BREAKDOWN


def test_singular_system_is_a_breakdown():
    """m0 = 0: the constant even spinor is in the kernel of H^2, so the first
    curvature <k, H^2 k> is exactly zero."""
    lat = unit_lattice()
    fin, x = lat.field(G.EVEN, host=ones(lat)), lat.field(G.EVEN)
    with pytest.raises(G.HRGPUError, match="breakdown") as e:
        lat.cg_mshift(G.OP_G5DPHI_EOPRE_SQ, 0.0, [0.0], 1e-20, fin, [x], max_iter=200)
    assert status_of(e.value) == G.E_BREAKDOWN


def test_shift_on_an_eigenvalue_is_a_breakdown():
    """m0 = -2: H^2 psi = 144 psi exactly; the multi-shift solve of (H^2 - s) for
    s = 0 and s = 144 must not report success for the singular second system."""
    lat = unit_lattice()
    fin = lat.field(G.EVEN, host=ones(lat))
    xs = [lat.field(G.EVEN), lat.field(G.EVEN)]
    # 1 + 144 omega vanishes up to the rounding of omega = -1/144: either the
    # recursion breaks down or the shifted system never converges; never success
    try:
        _, ok = lat.cg_mshift(G.OP_G5DPHI_EOPRE_SQ, -2.0, [0.0, 144.0], 1e-20, fin, xs, max_iter=200)
        assert not ok
    except G.HRGPUError as e:
        assert status_of(e) == G.E_BREAKDOWN
    # a regular shift beside it converges in one step (psi is an eigenvector)
    it, ok = lat.cg_mshift(G.OP_G5DPHI_EOPRE_SQ, -2.0, [0.0, 1.0], 1e-20, fin, xs, max_iter=200)
    assert ok
    assert np.abs(xs[0].download() - ones(lat) / 144.0).max() < 1e-15
    assert np.abs(xs[1].download() - ones(lat) / 143.0).max() < 1e-15


def test_max_iter_is_not_a_breakdown():
    from hirep_b200 import fields as F

    lat = G.Lattice(*DIMS, 3, G.FUND)
    lat.set_gauge(F.hot_gauge(3, lat.V, 3))
    lat.represent_gauge_field(True)
    fin, x = lat.field(G.EVEN, host=F.gaussian_spinor(4, lat.VH, lat.nf)), lat.field(G.EVEN)
    it, ok = lat.cg_mshift(G.OP_G5DPHI_EOPRE_SQ, -0.5, [0.0], 1e-28, fin, [x], max_iter=3)
    assert not ok and it >= 3


def test_zero_source_gives_zero():
    lat = unit_lattice()
    fin = lat.field(G.EVEN)
    xs = [lat.field(G.EVEN, host=ones(lat)), lat.field(G.EVEN, host=ones(lat))]
    for flt in (False, True):
        it, ok = lat.cg_mshift(G.OP_G5DPHI_EOPRE_SQ, 0.3, [0.0, 0.5], 1e-20, fin, xs, flt=flt)
        assert ok and it == 0
        assert not np.any(xs[0].download()) and not np.any(xs[1].download())
