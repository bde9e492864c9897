"""The five workloads at their full sizes.  Config 1 (8^4) is small enough for
the oracle itself; at the larger ones the checks are size-independent
properties (hermiticity, linearity, FP32 against FP64, batch against single
field, true residuals, bit-identical alternative paths) and, for the force of
config 3, the oracle's force at the full 16^4.  Seeded synthetic fields stand
in for HiRep's ranlux ones (hot start: Haar SU(N); smooth: exp(i eps H))."""
import numpy as np
import pytest

import oracle as O
from hirep_b200 import fields as F
from hirep_b200 import hrgpu as G

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_config1_wilson_8x8x8x8_against_the_oracle():
    """SU(3) fundamental, Wilson, 8^4, hot start, m0 = 0.1: Dphi and Dphi_eopre,
    then CG on g5Dphi_sq to err2 = 1e-28; fields and iteration count against
    the oracle."""
    o = O.Oracle(8, 8, 8, 8, 3, O.FUND)
    u = F.hot_gauge(1234, o.V, 3)
    o.set_gauge(o.represent_gauge_field(u, True))
    lat = G.Lattice(8, 8, 8, 8, 3, G.FUND, ipt=o.geometry()[0])
    lat.set_gauge(u)
    lat.represent_gauge_field(True)
    m = 0.1
    o.set_mass(m)
    src = F.gaussian_spinor(1234, o.V, o.nf) * np.sqrt(2)  # unit variance per real component
    fs, out = lat.field(O.FULL, host=src), lat.field(O.FULL)
    lat.Dphi(m, out, fs)
    assert rel(out.download(), o.Dphi(m, src)) < 1e-13
    e = src[: o.VH].copy()
    fe, oe = lat.field(O.EVEN, host=e), lat.field(O.EVEN)
    lat.Dphi_eopre(m, oe, fe)
    assert rel(oe.download(), o.Dphi_eopre(m, e)) < 1e-13
    xo, it_o = o.cg_mshift(G.OP_G5DPHI_SQ, [0.0], 1e-28, src)
    x = lat.field(O.FULL)
    it_g, ok = lat.cg_mshift(G.OP_G5DPHI_SQ, m, [0.0], 1e-28, fs, [x])
    assert ok
    assert rel(x.download(), xo[0]) < 1e-12
    assert abs(it_g - it_o) <= 3
    r = o.g5Dphi_sq(m, x.download()) - src
    assert o.sqnorm(r) / o.sqnorm(src) < 1e-28


@pytest.fixture(scope="module")
def config2():
    """SU(3) fundamental, clover csw = 1.0, m0 = -0.2, 16^3 x 32, U = exp(i 0.3 H) seed 7."""
    lat = G.Lattice(32, 16, 16, 16, 3, G.FUND)
    lat.set_gauge(F.smooth_gauge(7, lat.V, 3, 0.3))
    lat.represent_gauge_field(True)
    lat.clover_init(1.0)
    return lat


def test_config2_operator_properties(config2):
    lat, m = config2, -0.2
    x = lat.field(O.EVEN, host=F.gaussian_spinor(1, lat.VH, lat.nf))
    y = lat.field(O.EVEN, host=F.gaussian_spinor(2, lat.VH, lat.nf))
    hx, hy, t = lat.field(O.EVEN), lat.field(O.EVEN), lat.field(O.EVEN)
    lat.g5Cphi_eopre(m, hx, x)
    lat.g5Cphi_eopre(m, hy, y)
    a, b = lat.prod(x, hy), lat.prod(hx, y)  # H = g5 Cphi_eopre is Hermitian
    assert abs(a - b) < 1e-13 * abs(a)
    # linearity: H(x + 0.3i y) = Hx + 0.3i Hy
    lat.la("copy", t, x)
    lat.la("mulc_add_assign", t, 0.3j, y)
    lat.g5Cphi_eopre(m, hx, t)
    h1 = hx.download()
    lat.g5Cphi_eopre(m, hx, x)
    lat.g5Cphi_eopre(m, hy, y)
    assert rel(h1, hx.download() + 0.3j * hy.download()) < 1e-14
    # FP32 operator against FP64
    xs = x.download()
    x32, h32 = lat.field(O.EVEN, G.FLOAT, host=xs.astype(np.complex64)), lat.field(O.EVEN, G.FLOAT)
    lat.g5Cphi_eopre_flt(m, h32, x32)
    assert rel(h32.download().astype(complex), hx.download()) < 2e-6


def test_config2_mixed_solve_and_host_path(config2):
    """The mixed-precision solve reaches |r|/|b| < 1e-12 (true FP64 residual),
    agrees with the FP64 solve, and the pipelined host-field operator is
    bit-identical to the device operator at the full size."""
    lat, m = config2, -0.2
    bh = F.gaussian_spinor(3, lat.VH, lat.nf)
    b = lat.field(O.EVEN, host=bh)
    xm, xd, r = lat.field(O.EVEN), lat.field(O.EVEN), lat.field(O.EVEN)
    _, ok = lat.cg_mshift(G.OP_G5CPHI_EOPRE_SQ, m, [0.0], 1e-24, b, [xm], flt=True)
    assert ok
    _, ok = lat.cg_mshift(G.OP_G5CPHI_EOPRE_SQ, m, [0.0], 1e-24, b, [xd])
    assert ok
    lat.g5Cphi_eopre_sq(m, r, xm)
    lat.la("sub_assign", r, b)
    assert np.sqrt(lat.sqnorm(r) / lat.sqnorm(b)) < 1e-12
    assert rel(xm.download(), xd.download()) < 1e-10
    out = lat.field(O.EVEN)
    lat.Cphi_eopre(m, out, b)
    assert np.array_equal(lat.apply_op_host(G.OP_CPHI_EOPRE, m, bh), out.download())


def test_config3_force_against_the_oracle_at_16x16x16x16():
    """SU(4) two-index antisymmetric (NF = 6), Wilson m0 = -0.1, 16^4, links
    exp(i 0.25 H) seed 11: force_fermion_core (with the odd-site fill) and
    fermion_force_end against the oracle at the full size."""
    dims, ng = (16, 16, 16, 16), 4
    o = O.Oracle(*dims, ng, O.ASYM)
    u = F.smooth_gauge(11, o.V, ng, 0.25)
    o.set_gauge(o.represent_gauge_field(u, True))
    lat = G.Lattice(*dims, ng, G.ASYM, ipt=o.geometry()[0])
    lat.set_gauge(u)
    lat.represent_gauge_field(True)
    m = -0.1
    o.set_mass(m)
    lat.set_dirac_mass(m)
    X = F.gaussian_spinor(31, o.V, o.nf)
    Y = F.gaussian_spinor(32, o.V, o.nf)
    o.fermion_force_begin()
    o.force_fermion_core(X, Y, 1, 0.3, 1.0)
    lat.fermion_force_begin()
    lat.force_fermion_core(lat.field(O.FULL, host=X), lat.field(O.FULL, host=Y), 1, 0.3, 1.0)
    zero = np.zeros((o.V, 4, o.dimg))
    assert rel(lat.fermion_force_end(0.3, zero.copy()), o.fermion_force_end(0.3, zero.copy())) < 1e-12


def test_config4_batch_against_single_fields_at_24x24x24x48():
    """SU(3) two-index symmetric (NF = 6), clover csw = 1.0, m0 = -0.3,
    24^3 x 48, links exp(i 0.3 H) seed 21: the batched g5Cphi_eopre on the 12
    point sources (colours 0-2 x 4 spins at the origin) equals the single-field
    operator field by field (FP64 to 1e-13, FP32 to 2e-6)."""
    lat = G.Lattice(48, 24, 24, 24, 3, G.SYM)
    lat.set_gauge(F.smooth_gauge(21, lat.V, 3, 0.3))
    lat.represent_gauge_field(True)
    lat.clover_init(1.0)
    m = -0.3
    srcs = [F.point_source(lat.VH, lat.nf, s, c) for c in range(3) for s in range(4)]
    for prec, tol in ((G.DOUBLE, 1e-13), (G.FLOAT, 2e-6)):
        dt = np.complex128 if prec == G.DOUBLE else np.complex64
        fs = [lat.field(O.EVEN, prec, host=s.astype(dt)) for s in srcs]
        bi, bo = lat.batch(12, prec, fields=fs), lat.batch(12, prec)
        lat.apply_op_batch(G.OP_G5CPHI_EOPRE, m, bo, bi)
        outs = [lat.field(O.EVEN, prec) for _ in range(12)]
        bo.unpack(outs)
        single = lat.field(O.EVEN, prec)
        for k in (0, 5, 11):
            (lat.g5Cphi_eopre if prec == G.DOUBLE else lat.g5Cphi_eopre_flt)(m, single, fs[k])
            assert rel(outs[k].download(), single.download()) < tol


def test_config5_adjoint_32x32x32x64_operator():
    """SU(2) adjoint (NF = 3, real links), Wilson m0 = -1.0, 32^3 x 64, links
    exp(i 0.2 H) seed 99: g5Dphi_eopre is Hermitian, H^2 positive, and the FP32
    operator agrees with FP64, at the full size."""
    lat = G.Lattice(64, 32, 32, 32, 2, G.ADJ)
    lat.set_gauge(F.smooth_gauge(99, lat.V, 2, 0.2))
    lat.represent_gauge_field(True)
    m = -1.0
    x = lat.field(O.EVEN, host=F.gaussian_spinor(5, lat.VH, lat.nf))
    y = lat.field(O.EVEN, host=F.gaussian_spinor(6, lat.VH, lat.nf))
    hx, hy = lat.field(O.EVEN), lat.field(O.EVEN)
    lat.g5Dphi_eopre(m, hx, x)
    lat.g5Dphi_eopre(m, hy, y)
    a, b = lat.prod(x, hy), lat.prod(hx, y)
    assert abs(a - b) < 1e-13 * abs(a)
    lat.g5Dphi_eopre_sq(m, hy, x)
    assert lat.prod_re(x, hy) > 0.0 and abs(lat.prod_re(x, hy) - lat.sqnorm(hx)) < 1e-12 * lat.sqnorm(hx)
    x32, h32 = lat.field(O.EVEN, G.FLOAT, host=x.download().astype(np.complex64)), lat.field(O.EVEN, G.FLOAT)
    lat.g5Dphi_eopre_flt(m, h32, x32)
    assert rel(h32.download().astype(complex), hx.download()) < 2e-6
