"""Pins the CPU oracle (oracle/hr_oracle.c) and the library's host geometry to
HiRep itself: the reference's own library, compiled from its sources by
oracle/ref/Makefile and driven through oracle/ref/hr_ref.c (CPU only).

Same seeded inputs on both sides, compared field by field:
  geometry        ipt / iup / idn (geometry_mpi_eo.c)          bit-exact, also hrgpu_geometry
  representation  represent_gauge_field + BCs                   1e-15
  Wilson          Dphi_, Dphi, g5Dphi(_sq), (g5)Dphi_eopre(_sq), Dphi_oepre   1e-13
  clover          cl_term, cl_ldl, Cphi*, Cphi_diag(_inv)      1e-13
  exp. clover     Cphi*                                         1e-13
  cg_mshift       check_inverters_1's shifts: MVM count equal, solutions 1e-12
  cg_mshift_flt   MVM count within 10 %, solutions 1e-10
  force           force_fermion_core + fermion_force_end       1e-13
  config 1        HiRep's own hot start (ranlux seed 1234) and Gaussian source on 8^4

HiRep's clover builds run with one OpenMP thread here: HiRep's Cphi_
(LibHR/Update/Dphi.c:1092-1146) declares its temporaries (v1, v2, tmp, in, out,
s0..s3) outside the `_MASTER_FOR` parallel loop, so with more than one thread
they are shared and its results change from call to call.
"""
import os

import numpy as np
import pytest

import hirep_ref as H
import oracle as O
from hirep_b200 import fields as F
from hirep_b200 import hrgpu

REP = {"FUND": O.FUND, "ADJ": O.ADJ, "SYM": O.SYM, "ASYM": O.ASYM}
WILSON = ["su2_fund", "su2_adj", "su3_fund", "su3_adj", "su4_fund", "su4_asym"]
CLOVER = ["su3_fund_clover", "su3_sym_clover", "su3_asym_clover"]
REF_SOURCES = os.path.isdir("/root/reference/LibHR")


@pytest.fixture(scope="module", autouse=True)
def hirep_built():
    missing = [c for c in H.CONFIGS if not H.available(c)]
    if missing and REF_SOURCES:
        H.build()
    missing = [c for c in H.CONFIGS if not H.available(c)]
    if missing:
        pytest.skip(f"HiRep builds missing ({missing}) and no reference sources to build them")


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def pair(cfg, dims, seed=7, eps=0.3, threads=None):
    """The same smooth gauge field in HiRep and in the oracle."""
    ng, rep, clover = H.CONFIGS[cfg]
    h = H.HiRep(cfg, *dims, threads=threads if threads is not None else (1 if clover else None))
    o = O.Oracle(*dims, ng, REP[rep])
    u = F.smooth_gauge(seed, o.V, ng, eps)
    h.set_gauge(u)
    o.set_gauge(o.represent_gauge_field(u, True))
    return h, o, u


@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (8, 8, 8, 8), (6, 4, 4, 4), (4, 6, 2, 8), (16, 4, 4, 8)])
def test_geometry_is_hireps(dims):
    with H.HiRep("su3_fund", *dims) as h:
        ipt, iup, idn = h.geometry()
    oi, ou, od = O.Oracle(*dims, 3, O.FUND).geometry()
    li, lu, ld = hrgpu.geometry(*dims)
    for a, b, c in ((ipt, oi, li), (iup, ou, lu), (idn, od, ld)):
        assert np.array_equal(a, b)
        assert np.array_equal(a, c)


@pytest.mark.parametrize("cfg", WILSON + CLOVER)
def test_represented_links_are_hireps(cfg):
    h, o, u = pair(cfg, (4, 4, 4, 4))
    with h:
        uf = h.gauge_f()
    ng, rep, _ = H.CONFIGS[cfg]
    assert rel(uf, O.Oracle(4, 4, 4, 4, ng, REP[rep]).represent_gauge_field(u, True)) < 1e-15


@pytest.mark.parametrize("cfg", WILSON)
def test_wilson_operators_are_hireps(cfg):
    h, o, _ = pair(cfg, (4, 4, 4, 4))
    e = F.gaussian_spinor(1, o.VH, o.nf)
    od = F.gaussian_spinor(2, o.VH, o.nf)
    f = F.gaussian_spinor(3, o.V, o.nf)
    m = -0.1
    with h:
        assert rel(h.Dphi_(e, H.EVEN, H.ODD), o.Dphi_(e, O.EVEN, O.ODD)) < 1e-13
        assert rel(h.Dphi_(od, H.ODD, H.EVEN), o.Dphi_(od, O.ODD, O.EVEN)) < 1e-13
        assert rel(h.Dphi_(f, H.FULL, H.FULL), o.Dphi_(f, O.FULL, O.FULL)) < 1e-13
        for name in ("Dphi", "g5Dphi", "g5Dphi_sq"):
            assert rel(getattr(h, name)(m, f), getattr(o, name)(m, f)) < 1e-13, name
        for name in ("Dphi_eopre", "g5Dphi_eopre", "g5Dphi_eopre_sq"):
            assert rel(getattr(h, name)(m, e), getattr(o, name)(m, e)) < 1e-13, name
        assert rel(h.Dphi_oepre(m, od), o.Dphi_oepre(m, od)) < 1e-13


@pytest.mark.parametrize("cfg", CLOVER)
def test_clover_is_hireps(cfg):
    h, o, _ = pair(cfg, (4, 4, 4, 4))
    csw, m = 1.0, -0.2
    o.clover_init(csw)
    o.compute_clover_term()
    e = F.gaussian_spinor(1, o.VH, o.nf)
    f = F.gaussian_spinor(3, o.V, o.nf)
    with h:
        h.set_csw(csw)
        assert rel(h.clover_term(), o.clover_term()) < 1e-14
        o.compute_ldl_decomp(4.0 + m)
        assert rel(h.clover_ldl(m), o.clover_ldl()) < 1e-13
        for name in ("Cphi", "g5Cphi", "g5Cphi_sq"):
            assert rel(getattr(h, name)(m, f), getattr(o, name)(m, f)) < 1e-13, name
        for name in ("Cphi_eopre", "g5Cphi_eopre", "g5Cphi_eopre_sq"):
            assert rel(getattr(h, name)(m, e), getattr(o, name)(m, e)) < 1e-13, name
        for par, hp in ((O.EVEN, H.EVEN), (O.ODD, H.ODD)):
            assert rel(h.Cphi_diag(m, e, hp), o.Cphi_diag(m, e, par)) < 1e-13
            assert rel(h.Cphi_diag_inv(m, e, hp), o.Cphi_diag_inv(m, e, par)) < 1e-13


def test_hireps_clover_races_under_openmp():
    """The reason the clover builds run single-threaded: with 8 threads HiRep's
    own Cphi_diag gives a different answer from call to call."""
    h, o, _ = pair("su3_fund_clover", (4, 4, 4, 4), threads=8)
    e = F.gaussian_spinor(1, o.VH, o.nf)
    with h:
        h.set_csw(1.0)
        outs = [h.Cphi_diag(-0.2, e, H.EVEN) for _ in range(6)]
    o.clover_init(1.0)
    o.compute_clover_term()
    want = o.Cphi_diag(-0.2, e, O.EVEN)
    if h.threads > 1:
        assert max(rel(x, want) for x in outs) > 1e-3


def test_expclover_is_hireps():
    h, o, _ = pair("su3_fund_expclover", (4, 4, 4, 4), threads=1)
    csw, m = 1.0, -0.2
    o.expclover_init(csw)
    o.compute_clover_term()
    e = F.gaussian_spinor(1, o.VH, o.nf)
    f = F.gaussian_spinor(3, o.V, o.nf)
    with h:
        h.set_csw(csw)
        assert rel(h.clover_term(), o.clover_term()) < 1e-14
        for name in ("Cphi", "g5Cphi_sq"):
            assert rel(getattr(h, name)(m, f), getattr(o, name)(m, f)) < 1e-13, name
        for name in ("Cphi_eopre", "g5Cphi_eopre_sq"):
            assert rel(getattr(h, name)(m, e), getattr(o, name)(m, e)) < 1e-13, name
        for par, hp in ((O.EVEN, H.EVEN), (O.ODD, H.ODD)):
            assert rel(h.Cphi_diag(m, e, hp), o.Cphi_diag(m, e, par)) < 1e-13
            assert rel(h.Cphi_diag_inv(m, e, hp), o.Cphi_diag_inv(m, e, par)) < 1e-13


# check_inverters_1.c:86-91: its six shifts and err2 1e-28, here on the even-odd H^2
SHIFTS = [0.1, -0.21, 0.05, -0.01, -0.15, -0.05]


@pytest.mark.parametrize("cfg,op", [("su3_fund", "g5Dphi_eopre_sq"), ("su4_asym", "g5Dphi_eopre_sq"),
                                    ("su2_adj", "g5Dphi_eopre_sq"), ("su3_fund_clover", "g5Cphi_eopre_sq")])
def test_cg_mshift_is_hireps(cfg, op):
    h, o, _ = pair(cfg, (8, 8, 4, 4))
    m = 0.1
    if H.CONFIGS[cfg][2]:
        h.set_csw(1.0)
        o.clover_init(1.0)
        o.compute_clover_term()
    o.set_mass(m)
    e = F.gaussian_spinor(1, o.VH, o.nf)
    opcode = {"g5Dphi_eopre_sq": O.OP_G5DPHI_EOPRE_SQ, "g5Cphi_eopre_sq": O.OP_G5CPHI_EOPRE_SQ}[op]
    with h:
        xh, mvm_h = h.cg_mshift(op, m, SHIFTS, 1e-28, e, H.EVEN, max_iter=5000)
    xo, mvm_o = o.cg_mshift(opcode, SHIFTS, 1e-28, e, max_iter=5000)
    assert mvm_h == mvm_o
    for k in range(len(SHIFTS)):
        assert rel(xo[k], xh[k]) < 1e-12


@pytest.mark.parametrize("cfg", ["su3_fund", "su4_asym", "su2_adj"])
def test_cg_mshift_flt_is_hireps(cfg):
    h, o, _ = pair(cfg, (8, 8, 4, 4))
    m = 0.1
    o.set_mass(m)
    e = F.gaussian_spinor(1, o.VH, o.nf)
    shifts = [0.1, -0.21, 0.05]
    with h:
        xh, mvm_h = h.cg_mshift("g5Dphi_eopre_sq", m, shifts, 1e-20, e, H.EVEN, flt=True, max_iter=5000)
    xo, mvm_o = o.cg_mshift(O.OP_G5DPHI_EOPRE_SQ, shifts, 1e-20, e, flt=True, max_iter=5000)
    assert abs(mvm_h - mvm_o) <= 0.1 * mvm_h
    for k in range(len(shifts)):
        assert rel(xo[k], xh[k]) < 1e-9


@pytest.mark.parametrize("cfg", ["su3_fund", "su4_asym", "su2_adj", "su3_fund_clover", "su3_sym_clover"])
def test_force_is_hireps(cfg):
    h, o, _ = pair(cfg, (4, 4, 4, 4))
    m, dt, res = -0.1, 0.37, 1.3
    clover = H.CONFIGS[cfg][2]
    if clover:
        h.set_csw(1.0)
        o.clover_init(1.0)
        o.compute_clover_term()
    X = F.gaussian_spinor(11, o.V, o.nf)
    Y = F.gaussian_spinor(12, o.V, o.nf)
    o.set_mass(m)
    o.fermion_force_begin()
    o.force_fermion_core(X, Y, 1, dt, res)
    fo = o.fermion_force_end(dt, np.zeros((o.V, 4, o.dimg)))
    with h:
        fh = h.force(m, dt, res, X, Y, True)
    assert rel(fh, fo) < 1e-13


def test_config1_hot_start_from_hireps_ranlux():
    """Config 1 as specified: SU(3) fundamental 8^4, random_u after rlxd_init(1,1234),
    Dphi / Dphi_eopre at m0=0.1, and CG on g5Dphi_sq to |r|/|b| < 1e-14."""
    dims, m = (8, 8, 8, 8), 0.1
    with H.HiRep("su3_fund", *dims, seed=1234, threads=1) as h:
        u = h.random_u()
        plaq = h.plaquette()
        f = h.gaussian_spinor_field(H.FULL)
        e = f[: h.VH].copy()
        d_h = h.Dphi(m, f)
        eo_h = h.Dphi_eopre(m, e)
        x_h, mvm_h = h.cg_mshift("g5Dphi_sq", m, [0.0], 1e-28, f, H.FULL, max_iter=5000)
    o = O.Oracle(*dims, 3, O.FUND)
    # in the fundamental representation u_gauge_f is u_gauge, so the links read
    # back already carry the antiperiodic sign (archive.c:238-242)
    o.set_gauge(o.represent_gauge_field(u, False))
    o.set_mass(m)
    # a hot start: the average plaquette of Haar links is ~0; one thread draws
    # the fixture's field (ranlxd keeps a stream per OpenMP thread)
    assert abs(plaq) < 0.02
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "hirep_config1.npz"))
    assert abs(plaq - float(g["plaquette"])) < 1e-14
    assert abs(o.avr_plaquette(u) - plaq) < 1e-12
    assert rel(o.Dphi(m, f), d_h) < 1e-13
    assert rel(o.Dphi_eopre(m, e), eo_h) < 1e-13
    x_o, mvm_o = o.cg_mshift(O.OP_G5DPHI_SQ, [0.0], 1e-28, f, max_iter=5000)
    assert mvm_o == mvm_h
    assert rel(x_o[0], x_h[0]) < 1e-12


# ---------------------------------------------------------------------------
# the "next" rows: g5QMR and MINRES, the gauge force and the link update
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("cfg", ["su3_fund", "su4_asym", "su2_adj"])
def test_g5qmr_is_hireps(cfg):
    """g5QMR_mshift (g5QMR_mshift.c:481-542) on Dphi_eopre with three shifts: the
    oracle's MVM count equals HiRep's, solutions to 1e-10 (the solver's accuracy)."""
    h, o, _ = pair(cfg, (8, 8, 4, 4))
    m, shifts, err2 = 0.1, [0.0, -0.1, 0.05], 1e-26
    o.set_mass(m)
    e = F.gaussian_spinor(5, o.VH, o.nf)
    with h:
        xh, mvm_h = h.g5QMR_mshift("Dphi_eopre", m, shifts, err2, e, H.EVEN, max_iter=5000)
    xo, mvm_o = o.g5QMR_mshift(O.OP_DPHI_EOPRE, shifts, err2, e, max_iter=5000)
    assert mvm_o == mvm_h
    for k in range(len(shifts)):
        assert rel(xo[k], xh[k]) < 1e-10


def test_minres_is_hireps():
    """MINRES (MINRES.c:160-172) on the hermitian g5Dphi_eopre."""
    h, o, _ = pair("su3_fund", (8, 8, 4, 4))
    m, err2 = 0.1, 1e-26
    o.set_mass(m)
    e = F.gaussian_spinor(6, o.VH, o.nf)
    with h:
        xh, mvm_h = h.MINRES("g5Dphi_eopre", m, err2, e, H.EVEN, max_iter=5000)
    xo, mvm_o = o.MINRES(O.OP_G5DPHI_EOPRE, err2, e, max_iter=5000)
    assert mvm_o == mvm_h
    assert rel(xo, xh) < 1e-10


@pytest.mark.parametrize("cfg", ["su3_fund", "su2_adj", "su4_asym"])
def test_gauge_force_and_link_update_are_hireps(cfg):
    """force0 (force0.c:22-99) into given momenta, and update_gauge_field
    (field_update.c:18-66, ExpX), on the links HiRep holds (in a fundamental build
    the antiperiodic sign sits on u_gauge itself)."""
    h, o, _ = pair(cfg, (4, 4, 4, 4))
    ng = H.CONFIGS[cfg][0]
    rng = np.random.default_rng(41)
    mom = rng.standard_normal((o.V, 4, ng * ng - 1))
    with h:
        uh = h.gauge()
        h.momenta_set(mom)
        h.force0(0.23, 2.25)
        assert rel(h.momenta_get(), o.force0(0.23, 2.25, uh, mom)) < 1e-13
        h.momenta_set(mom)
        h.update_gauge_field(0.05)
        assert rel(h.gauge(), o.update_gauge_field(0.05, uh, mom)) < 1e-13
