"""Parity of the B200 library (through its C ABI) with the CPU oracle.

FP64 results must agree to 1e-13 relative (max-norm of the difference over the
max-norm of the result), FP32 results to 2e-6, index maps exactly.  Inputs are
seeded synthetic fields on lattices the oracle finishes in seconds.
"""
import numpy as np
import pytest

import oracle as O
from hirep_b200 import fields as F
from hirep_b200 import hrgpu as G

pytestmark = pytest.mark.gpu

TOL64 = 1e-13
TOL32 = 2e-6
REPS = [(3, O.FUND), (2, O.ADJ), (3, O.SYM), (4, O.ASYM), (2, O.FUND), (3, O.ADJ)]


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def setup(dims, ng, rep, seed=1, smooth=0.4, bc=True, gpu_represent=False):
    o = O.Oracle(*dims, ng, rep)
    ipt, _, _ = o.geometry()
    u = F.smooth_gauge(seed, o.V, ng, smooth) if smooth else F.hot_gauge(seed, o.V, ng)
    uf = o.represent_gauge_field(u, bc)
    o.set_gauge(uf)
    lat = G.Lattice(*dims, ng, rep, ipt=ipt)
    if gpu_represent:
        lat.set_gauge(u)
        lat.represent_gauge_field(bc)
    else:
        lat.set_gauge_f(uf)
    return o, lat, u, uf


@pytest.mark.parametrize("ng,rep", REPS)
def test_represent_gauge_field(ng, rep):
    o, lat, u, uf = setup((4, 4, 4, 4), ng, rep, gpu_represent=True, smooth=None)
    got = lat.gauge_f()
    assert rel(got, uf) < TOL64


@pytest.mark.parametrize("ng,rep", REPS)
def test_spinor_roundtrip_and_layout(ng, rep):
    o, lat, _, _ = setup((4, 4, 2, 6), ng, rep)
    for par in (O.EVEN, O.ODD, O.FULL):
        s = F.gaussian_spinor(3 + par, o.nsites(par), o.nf)
        assert np.array_equal(lat.field(par, host=s).download(), s)
        s32 = s.astype(np.complex64)
        assert np.array_equal(lat.field(par, G.FLOAT, host=s32).download(), s32)


@pytest.mark.parametrize("ng,rep", REPS)
def test_hopping_and_wilson_operators(ng, rep):
    o, lat, _, _ = setup((4, 4, 4, 6), ng, rep, seed=3)
    m = -0.15
    e = F.gaussian_spinor(1, o.VH, o.nf)
    od = F.gaussian_spinor(2, o.VH, o.nf)
    full = F.gaussian_spinor(3, o.V, o.nf)
    fe, fo, ff = lat.field(O.EVEN, host=e), lat.field(O.ODD, host=od), lat.field(O.FULL, host=full)
    out_e, out_o, out_f = lat.field(O.EVEN), lat.field(O.ODD), lat.field(O.FULL)
    lat.Dphi_(out_o, fe)
    assert rel(out_o.download(), o.Dphi_(e, O.EVEN, O.ODD)) < TOL64
    lat.Dphi_(out_e, fo)
    assert rel(out_e.download(), o.Dphi_(od, O.ODD, O.EVEN)) < TOL64
    lat.Dphi_(out_f, ff)
    assert rel(out_f.download(), o.Dphi_(full, O.FULL, O.FULL)) < TOL64
    for name in ("Dphi", "g5Dphi", "g5Dphi_sq"):
        getattr(lat, name)(m, out_f, ff)
        assert rel(out_f.download(), getattr(o, name)(m, full)) < TOL64, name
    for name in ("Dphi_eopre", "g5Dphi_eopre", "g5Dphi_eopre_sq"):
        getattr(lat, name)(m, out_e, fe)
        assert rel(out_e.download(), getattr(o, name)(m, e)) < TOL64, name
    lat.Dphi_oepre(m, out_o, fo)
    assert rel(out_o.download(), o.Dphi_oepre(m, od)) < TOL64


@pytest.mark.parametrize("ng,rep", [(3, O.FUND), (2, O.ADJ), (3, O.SYM)])
def test_float_operators(ng, rep):
    o, lat, _, _ = setup((4, 4, 4, 4), ng, rep, seed=4)
    m = 0.1
    e = F.gaussian_spinor(1, o.VH, o.nf).astype(np.complex64)
    full = F.gaussian_spinor(3, o.V, o.nf).astype(np.complex64)
    fe, ff = lat.field(O.EVEN, G.FLOAT, host=e), lat.field(O.FULL, G.FLOAT, host=full)
    out_o, out_e, out_f = lat.field(O.ODD, G.FLOAT), lat.field(O.EVEN, G.FLOAT), lat.field(O.FULL, G.FLOAT)
    lat.Dphi_flt_(out_o, fe)
    assert rel(out_o.download(), o.Dphi_flt_(e, O.EVEN, O.ODD)) < TOL32
    lat.Dphi_flt(m, out_f, ff)
    assert rel(out_f.download(), o.Dphi_flt(m, full)) < TOL32
    for name in ("Dphi_eopre_flt", "g5Dphi_eopre_flt", "g5Dphi_eopre_sq_flt"):
        getattr(lat, name)(m, out_e, fe)
        assert rel(out_e.download(), getattr(o, name)(m, e)) < 10 * TOL32, name
    # float operator against the double one
    lat.g5Dphi_eopre_flt(m, out_e, fe)
    d = o.g5Dphi_eopre(m, e.astype(np.complex128))
    assert rel(out_e.download(), d) < 1e-5


@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (4, 6, 6, 6)])
@pytest.mark.parametrize("ng,rep", [(2, O.FUND), (3, O.FUND), (4, O.FUND), (2, O.ADJ), (3, O.ADJ), (4, O.ADJ),
                                    (3, O.SYM), (4, O.SYM), (4, O.ASYM), (5, O.ASYM)])
def test_clover_term_every_representation(dims, ng, rep):
    """compute_clover_term (one thread per site, plane and row; several sites per
    block) against the oracle element by element for every NF the library builds,
    complex and real, on a lattice whose last block is ragged (4^4) and one with
    padding sites (half volume 432)."""
    o, lat, _, _ = setup(dims, ng, rep, seed=5, smooth=0.3)
    o.clover_init(1.0)
    o.compute_clover_term()
    lat.clover_init(1.0)
    assert rel(lat.clover_term(), o.clover_term()) < TOL64


@pytest.mark.parametrize("ng,rep", [(3, O.FUND), (2, O.ADJ), (3, O.SYM), (2, O.FUND)])
def test_clover_operators(ng, rep):
    o, lat, _, _ = setup((4, 4, 4, 4), ng, rep, seed=5, smooth=0.3)
    o.clover_init(1.0)
    o.compute_clover_term()
    lat.clover_init(1.0)
    assert rel(lat.clover_term(), o.clover_term()) < TOL64
    m = -0.2
    e = F.gaussian_spinor(1, o.VH, o.nf)
    od = F.gaussian_spinor(2, o.VH, o.nf)
    full = F.gaussian_spinor(3, o.V, o.nf)
    fe, fo, ff = lat.field(O.EVEN, host=e), lat.field(O.ODD, host=od), lat.field(O.FULL, host=full)
    out_e, out_o, out_f = lat.field(O.EVEN), lat.field(O.ODD), lat.field(O.FULL)
    for name in ("Cphi_eopre", "g5Cphi_eopre", "g5Cphi_eopre_sq"):
        getattr(lat, name)(m, out_e, fe)
        assert rel(out_e.download(), getattr(o, name)(m, e)) < TOL64, name
    for name in ("Cphi", "g5Cphi", "g5Cphi_sq"):
        getattr(lat, name)(m, out_f, ff)
        assert rel(out_f.download(), getattr(o, name)(m, full)) < TOL64, name
    lat.Cphi_diag(m, out_o, fo)
    assert rel(out_o.download(), o.Cphi_diag(m, od, O.ODD)) < TOL64
    lat.Cphi_diag_inv(m, out_o, fo)
    assert rel(out_o.download(), o.Cphi_diag_inv(m, od, O.ODD)) < TOL64
    # in place, as HiRep allows for Cphi_diag_inv
    lat.Cphi_diag_inv(m, fo, fo)
    assert rel(fo.download(), o.Cphi_diag_inv(m, od, O.ODD)) < TOL64
    # float clover operator against the double one
    fe32, oe32 = lat.field(O.EVEN, G.FLOAT, host=e.astype(np.complex64)), lat.field(O.EVEN, G.FLOAT)
    lat.g5Cphi_eopre_flt(m, oe32, fe32)
    assert rel(oe32.download(), o.g5Cphi_eopre(m, e.astype(np.complex64).astype(complex))) < 1e-5


def test_linear_algebra():
    o, lat, _, _ = setup((4, 4, 4, 4), 3, O.FUND)
    a = F.gaussian_spinor(1, o.VH, o.nf)
    b = F.gaussian_spinor(2, o.VH, o.nf)
    c = F.gaussian_spinor(3, o.VH, o.nf)
    fa, fb, fc, r = (lat.field(O.EVEN, host=x) for x in (a, b, c, a))
    assert lat.sqnorm(fa) == pytest.approx(o.sqnorm(a), rel=1e-14)
    assert lat.prod_re(fa, fb) == pytest.approx(o.prod_re(a, b), rel=1e-13)
    assert lat.prod_im(fa, fb) == pytest.approx(o.prod_im(a, b), rel=1e-13)
    assert lat.g5_prod_re(fa, fb) == pytest.approx(o.g5_prod_re(a, b), rel=1e-12)
    assert lat.g5_prod_im(fa, fb) == pytest.approx(o.g5_prod_im(a, b), rel=1e-12)
    p = lat.prod(fa, fb)
    assert p == pytest.approx(np.vdot(a, b), rel=1e-13)
    g5 = np.array([1, 1, -1, -1])[None, :, None]
    cases = [
        ("mul_add_assign", (r, 0.3, fb), a + 0.3 * b),
        ("mulc_add_assign", (r, 0.3 - 0.7j, fb), a + (0.3 - 0.7j) * b),
        ("g5_mulc_add_assign", (r, 0.3 - 0.7j, fb), a + (0.3 - 0.7j) * g5 * b),
        ("mul", (r, -1.5, fb), -1.5 * b),
        ("mulc", (r, 0.5 + 2j, fb), (0.5 + 2j) * b),
        ("add", (r, fb, fc), b + c),
        ("sub", (r, fb, fc), b - c),
        ("add_assign", (r, fb), a + b),
        ("sub_assign", (r, fb), a - b),
        ("copy", (r, fb), b),
        ("minus", (r, fb), -b),
        ("lc", (r, 0.2, fb, -0.4, fc), 0.2 * b - 0.4 * c),
        ("lc_add_assign", (r, 0.2, fb, -0.4, fc), a + 0.2 * b - 0.4 * c),
        ("clc", (r, 0.2j, fb, 1 - 1j, fc), 0.2j * b + (1 - 1j) * c),
        ("clc_add_assign", (r, 0.2j, fb, 1 - 1j, fc), a + 0.2j * b + (1 - 1j) * c),
        ("g5", (r, fb), g5 * b),
        ("g0", (r, fb), o.gamma(0, b)),
        ("g1", (r, fb), o.gamma(1, b)),
        ("g2", (r, fb), o.gamma(2, b)),
        ("g3", (r, fb), o.gamma(3, b)),
        ("lc1", (0.7, r, fb), a + 0.7 * b),
        ("lc2", (0.7, -0.2, r, fb), 0.7 * a - 0.2 * b),
    ]
    for name, args, expect in cases:
        r.upload(a)
        lat.la(name, *args)
        assert rel(r.download(), expect) < 1e-15 * 10, name
    r.upload(a)
    lat.la("g5_assign", r)
    assert rel(r.download(), g5 * a) == 0
    r.upload(c)
    lat.la("lc3", 0.7, -0.2, fa, fb, r)
    assert rel(r.download(), -(c - 0.7 * a + 0.2 * b)) < 1e-14
    lat.la("zero", r)
    assert np.abs(r.download()).max() == 0
    # float variants and conversions
    fa32 = lat.field(O.EVEN, G.FLOAT)
    lat.assign_sd2s(fa32, fa)
    assert np.array_equal(fa32.download(), a.astype(np.complex64))
    back = lat.field(O.EVEN)
    lat.assign_s2sd(back, fa32)
    assert np.array_equal(back.download(), a.astype(np.complex64).astype(complex))
    assert lat.sqnorm(fa32) == pytest.approx(float(np.vdot(a.astype(np.complex64), a.astype(np.complex64)).real), rel=1e-6)


@pytest.mark.parametrize("ng,rep,op", [(3, O.FUND, G.OP_G5DPHI_EOPRE_SQ), (2, O.ADJ, G.OP_G5DPHI_EOPRE_SQ),
                                       (3, O.FUND, G.OP_G5DPHI_SQ), (4, O.ASYM, G.OP_G5DPHI_EOPRE_SQ)])
def test_cg_mshift(ng, rep, op):
    o, lat, _, _ = setup((4, 4, 4, 4), ng, rep, seed=6, smooth=None)
    m = -0.1 if op == G.OP_G5DPHI_SQ else 0.2
    o.set_mass(m)
    shifts = [0.1, -0.21, 0.05, -0.01, -0.15, -0.05] if op == G.OP_G5DPHI_SQ else [0.0, -0.1, 0.3]
    err2 = 1e-26
    par = O.FULL if op == G.OP_G5DPHI_SQ else O.EVEN
    b = F.gaussian_spinor(8, o.nsites(par), o.nf)
    xo, it_o = o.cg_mshift(op, shifts, err2, b)
    fb = lat.field(par, host=b)
    outs = [lat.field(par) for _ in shifts]
    it_g, ok = lat.cg_mshift(op, m, shifts, err2, fb, outs)
    assert ok
    apply = o.g5Dphi_sq if op == G.OP_G5DPHI_SQ else o.g5Dphi_eopre_sq
    for i, s in enumerate(shifts):
        x = outs[i].download()
        res = apply(m, x) - s * x - b
        assert o.sqnorm(res) / o.sqnorm(b) < err2
        assert rel(x, xo[i]) < 1e-10
    assert abs(it_g - it_o) <= 3


def test_cg_single_shift_initial_guess_and_max_iter():
    o, lat, _, _ = setup((4, 4, 4, 4), 3, O.FUND, seed=7)
    m = 0.1
    o.set_mass(m)
    b = F.gaussian_spinor(9, o.VH, o.nf)
    fb = lat.field(O.EVEN, host=b)
    # exact solution as the guess: converged at once
    xo, _ = o.cg_mshift(O.OP_G5DPHI_EOPRE_SQ, [0.0], 1e-26, b)
    out = lat.field(O.EVEN, host=xo[0])
    it, ok = lat.cg_mshift(G.OP_G5DPHI_EOPRE_SQ, m, [0.0], 1e-20, fb, [out])
    assert ok and it <= 4
    # max_iter stops early and reports non-convergence
    out2 = lat.field(O.EVEN)
    it2, ok2 = lat.cg_mshift(G.OP_G5DPHI_EOPRE_SQ, m, [0.0], 1e-60, fb, [out2], max_iter=5)
    assert not ok2


@pytest.mark.parametrize("clover", [False, True])
def test_cg_mshift_flt_reaches_double_precision(clover):
    o, lat, _, _ = setup((4, 4, 4, 8), 3, O.FUND, seed=8, smooth=0.3)
    m = -0.2 if clover else 0.1
    o.set_mass(m)
    if clover:
        o.clover_init(1.0)
        o.compute_clover_term()
        lat.clover_init(1.0)
    op = G.OP_G5CPHI_EOPRE_SQ if clover else G.OP_G5DPHI_EOPRE_SQ
    apply = o.g5Cphi_eopre_sq if clover else o.g5Dphi_eopre_sq
    shifts = [0.0, 0.05, 0.3]
    err2 = 1e-24
    b = F.gaussian_spinor(10, o.VH, o.nf)
    fb = lat.field(O.EVEN, host=b)
    outs = [lat.field(O.EVEN) for _ in shifts]
    it, ok = lat.cg_mshift(op, m, shifts, err2, fb, outs, flt=True)
    assert ok and it > 0
    for i, s in enumerate(shifts):
        x = outs[i].download()
        r = apply(m, x) - s * x - b
        assert o.sqnorm(r) / o.sqnorm(b) < err2


@pytest.mark.parametrize("ng,rep,clover", [(3, O.FUND, False), (2, O.ADJ, False), (4, O.ASYM, False),
                                            (3, O.SYM, False), (3, O.FUND, True), (2, O.ADJ, True)])
def test_force_matches_oracle(ng, rep, clover):
    o, lat, _, _ = setup((4, 4, 4, 4), ng, rep, seed=9, smooth=0.3)
    m = -0.1
    o.set_mass(m)
    lat.set_dirac_mass(m)
    if clover:
        o.clover_init(1.0)
        o.compute_clover_term()
        lat.clover_init(1.0)
    X = F.gaussian_spinor(11, o.V, o.nf)
    Y = F.gaussian_spinor(12, o.V, o.nf)
    o.fermion_force_begin()
    Xo, Yo = o.force_fermion_core(X, Y, 1, 0.7, 1.3)
    lat.fermion_force_begin()
    fX, fY = lat.field(O.FULL, host=X), lat.field(O.FULL, host=Y)
    lat.force_fermion_core(fX, fY, 1, 0.7, 1.3)
    assert rel(fX.download(), Xo) < TOL64
    assert rel(fY.download(), Yo) < TOL64
    assert rel(lat.force_sum(), o.force_sum()) < 1e-12
    if clover:
        o.force_clover_logdet(m, 0.4)
        lat.force_clover_logdet(m, 0.4)
    mom = F.gaussian_spinor(13, o.V, 1).real.reshape(-1)[: o.V].repeat(4 * o.dimg).reshape(o.V, 4, o.dimg)
    fo = o.fermion_force_end(0.7, mom)
    fg = lat.fermion_force_end(0.7, mom)
    assert rel(fg - mom, fo - mom) < 1e-12


@pytest.mark.parametrize("variant", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("ng,rep", [(2, O.FUND), (3, O.FUND), (2, O.ADJ), (4, O.ASYM), (3, O.SYM), (4, O.FUND),
                                    (5, O.FUND), (6, O.FUND)])
def test_force_variants(variant, ng, rep):
    """Every kernel of the hopping force (one lane per link; two lanes per link in two
    warps with the constant-memory projection table, padded to 2, 3 or 5 entries per
    element, without and with L2 prefetches, with the NF = 6 two-index links
    built from the fundamental ones, and with the link, or the link and the
    spinor at x, staged in shared memory by cp.async) gives the oracle's force, on a
    4x6x6x6 lattice whose half volume (432) is not a multiple of 32, so the last
    block holds padding sites that compute and write nothing."""
    o, lat, _, _ = setup((4, 6, 6, 6), ng, rep, seed=19, smooth=0.3, gpu_represent=True)
    if variant == 4 and rep in (O.SYM, O.ASYM) and lat.nf == 6:
        assert lat.link_recon() == 4  # variant 4 builds the links from the fundamental ones
    G._check(lat.L.hrgpu_set_force_variant(variant), "set_force_variant")
    try:
        m = -0.1
        o.set_mass(m)
        lat.set_dirac_mass(m)
        X = F.gaussian_spinor(31, o.V, o.nf)
        Y = F.gaussian_spinor(32, o.V, o.nf)
        o.fermion_force_begin()
        o.force_fermion_core(X, Y, 1, 0.7, 1.3)
        lat.fermion_force_begin()
        lat.force_fermion_core(lat.field(O.FULL, host=X), lat.field(O.FULL, host=Y), 1, 0.7, 1.3)
        assert rel(lat.force_sum(), o.force_sum()) < 1e-12
    finally:
        G._check(lat.L.hrgpu_set_force_variant(0), "set_force_variant")


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("ng,rep", [(3, O.FUND), (2, O.ADJ), (3, O.SYM)])
def test_hop_variants(variant, ng, rep):
    """Every variant of the hopping kernel the autotuner can pick gives the oracle's
    result (4x16x8x4: a time slab of one parity is 256 sites, as variant 5 needs)."""
    o, lat, _, _ = setup((4, 16, 8, 4), ng, rep, seed=21, smooth=0.3)
    G._check(lat.L.hrgpu_set_hop_variant(variant), "set_hop_variant")
    try:
        m = -0.2
        e = F.gaussian_spinor(5, o.VH, o.nf)
        fe, out = lat.field(O.EVEN, host=e), lat.field(O.EVEN)
        try:
            lat.g5Dphi_eopre(m, out, fe)
        except G.HRGPUError as exc:
            if "not built" in str(exc):
                pytest.skip(f"variant {variant} is not built for NF={o.nf}")
            raise
        assert rel(out.download(), o.g5Dphi_eopre(m, e)) < TOL64
        full = F.gaussian_spinor(6, o.V, o.nf)
        ff, outf = lat.field(O.FULL, host=full), lat.field(O.FULL)
        lat.g5Dphi(m, outf, ff)
        assert rel(outf.download(), o.g5Dphi(m, full)) < TOL64
        o.clover_init(1.0)
        o.compute_clover_term()
        lat.clover_init(1.0)
        lat.g5Cphi_eopre(m, out, fe)
        assert rel(out.download(), o.g5Cphi_eopre(m, e)) < TOL64
        e32 = e.astype(np.complex64)
        fe32, out32 = lat.field(O.EVEN, G.FLOAT, host=e32), lat.field(O.EVEN, G.FLOAT)
        lat.g5Dphi_eopre_flt(m, out32, fe32)
        assert rel(out32.download(), o.g5Dphi_eopre_flt(m, e32)) < 10 * TOL32
    finally:
        G._check(lat.L.hrgpu_set_hop_variant(-1), "set_hop_variant")


def test_programmatic_dependent_launch_changes_no_result():
    """FP64 hops with and without programmatic dependent launch: the same
    kernels, so bit-identical operators and solves."""
    o, lat, _, _ = setup((4, 4, 4, 4), 3, O.FUND, seed=31, smooth=0.3)
    lat.clover_init(1.0)
    m = -0.2
    e = F.gaussian_spinor(8, o.VH, o.nf)
    fin, fout = lat.field(O.EVEN, host=e), lat.field(O.EVEN)
    res = {}
    try:
        for pdl in (1, 0):
            G._check(lat.L.hrgpu_set_hop_pdl(pdl), "set_hop_pdl")
            lat.g5Cphi_eopre_sq(m, fout, fin)
            x = lat.field(O.EVEN)
            lat.cg_mshift(G.OP_G5CPHI_EOPRE_SQ, m, [0.0], 1e-24, fin, [x])
            res[pdl] = (fout.download(), x.download())
    finally:
        G._check(lat.L.hrgpu_set_hop_pdl(1), "set_hop_pdl")
    assert np.array_equal(res[0][0], res[1][0])
    assert np.array_equal(res[0][1], res[1][1])


def test_spin_structure_gamma_matrices():
    """TestProgram/DiracOperator/check_diracoperator_4 restated: with every link
    zero but U(g, mu) = 1 (periodic BCs) and a constant source in spin beta,
    colour ic, Dphi_ gives out(g) - out(g+mu) = gamma_mu column beta.  The
    extracted gammas are the same for every site and colour (1e-14, as the
    reference requires), Hermitian, satisfy {g_mu, g_nu} = 2 delta, and
    diag(1,1,-1,-1) (the gamma_5 of g5Dphi) anticommutes with them and equals
    +-g0 g1 g2 g3."""
    dims = (4, 4, 4, 4)
    T, X, Y, Z = dims
    ng = 3
    o = O.Oracle(*dims, ng, O.FUND)
    ipt = o.geometry()[0]
    lat = G.Lattice(*dims, ng, G.FUND, ipt=ipt)
    V, nf = lat.V, lat.nf

    def idx(t, x, y, z):
        return ipt[((t % T * X + x % X) * Y + y % Y) * Z + z % Z]

    ref = None
    inp, out = lat.field(O.FULL), lat.field(O.FULL)
    for g in [(0, 0, 0, 0), (3, 3, 3, 3), (1, 2, 3, 0), (2, 0, 1, 3)]:
        for ic in (0, nf - 1):
            gam = np.zeros((4, 4, 4), complex)
            for mu in range(4):
                u = np.zeros((V, 4, ng, ng), complex)
                u[idx(*g), mu] = np.eye(ng)
                lat.set_gauge(u)
                lat.represent_gauge_field(False)
                sh = [0, 0, 0, 0]
                sh[mu] = 1
                gp = idx(*(c + s for c, s in zip(g, sh)))
                for beta in range(4):
                    src = np.zeros((V, 4, nf), complex)
                    src[:, beta, ic] = 1.0
                    inp.upload(src)
                    lat.Dphi_(out, inp)
                    r = out.download()
                    gam[mu, :, beta] = r[idx(*g), :, ic] - r[gp, :, ic]
                    others = np.ones(V, bool)
                    others[[idx(*g), gp]] = False
                    assert np.all(r[others] == 0.0)
            if ref is None:
                ref = gam
            assert np.sum(np.abs(gam - ref) ** 2) < 1e-14
    eye = np.eye(4)
    g5 = np.diag([1.0, 1.0, -1.0, -1.0])
    for mu in range(4):
        assert np.allclose(ref[mu], ref[mu].conj().T, atol=1e-15)
        assert np.allclose(g5 @ ref[mu] + ref[mu] @ g5, 0.0, atol=1e-15)
        for nu in range(4):
            assert np.allclose(ref[mu] @ ref[nu] + ref[nu] @ ref[mu], 2.0 * eye * (mu == nu), atol=1e-15)
    prod = ref[0] @ ref[1] @ ref[2] @ ref[3]
    assert np.allclose(prod, g5, atol=1e-15) or np.allclose(prod, -g5, atol=1e-15)


@pytest.mark.parametrize("ng,rep", [(3, O.FUND), (2, O.ADJ)])
@pytest.mark.parametrize("bc", [True, False])
def test_link_reconstruction(ng, rep, bc):
    """SU(3) fundamental and SU(2) adjoint links represented on the device pass
    the row-2 check, and the hopping kernels then rebuild row 2 (mode 2 with
    the antiperiodic sign, 1 without); links uploaded already represented
    (hrgpu_gauge_set_f) are checked the same way.  Wilson and clover eopre
    operators, FP64 and FP32, for the variants 0-2 and 5 (0 and 2 rebuild),
    against the oracle and against the full-link kernels.  A field that is not
    unitary fails the check and the kernels read full links."""
    dims = (4, 8, 8, 4)  # a time slab of 128 sites, so variant 5 applies
    m = -0.2
    o, lat, u, uf = setup(dims, ng, rep, seed=12, smooth=0.4, bc=bc, gpu_represent=True)
    assert lat.link_recon() == (2 if bc else 1)
    e = F.gaussian_spinor(21, o.VH, o.nf)
    e32 = e.astype(np.complex64)
    fin, out = lat.field(O.EVEN, host=e), lat.field(O.EVEN)
    f32, out32 = lat.field(O.EVEN, G.FLOAT, host=e32), lat.field(O.EVEN, G.FLOAT)
    ref, ref32 = o.g5Dphi_eopre(m, e), o.g5Dphi_eopre_flt(m, e32)
    try:
        for v in (0, 1, 2, 5):
            G._check(lat.L.hrgpu_set_hop_variant(v), "set_hop_variant")
            lat.g5Dphi_eopre(m, out, fin)
            assert rel(out.download(), ref) < TOL64, v
            lat.g5Dphi_eopre_flt(m, out32, f32)
            assert rel(out32.download(), ref32) < 10 * TOL32, v
        G._check(lat.L.hrgpu_set_hop_variant(0), "set_hop_variant")
        lat.g5Dphi_eopre(m, out, fin)
        rebuilt = out.download()
        lat.clover_init(1.0)
        o.clover_init(1.0)
        o.compute_clover_term()
        lat.g5Cphi_eopre(m, out, fin)
        assert rel(out.download(), o.g5Cphi_eopre(m, e)) < TOL64
    finally:
        G._check(lat.L.hrgpu_set_hop_variant(-1), "set_hop_variant")
    # the same links uploaded already represented: the check finds the mode
    # again; with reconstruction forbidden the kernels read all three rows
    lat2 = G.Lattice(*dims, ng, rep, ipt=o.geometry()[0])
    lat2.set_gauge_f(uf)
    assert lat2.link_recon() == (2 if bc else 1)
    out2 = lat2.field(O.EVEN)
    try:
        G._check(lat2.L.hrgpu_set_link_recon(0), "set_link_recon")
        assert lat2.link_recon() == 0
        lat2.g5Dphi_eopre(m, out2, lat2.field(O.EVEN, host=e))
    finally:
        G._check(lat2.L.hrgpu_set_link_recon(1), "set_link_recon")
    assert rel(rebuilt, out2.download()) < 1e-14
    # links that are not SU(3): no reconstruction, and still the oracle's operator
    ub = u * 1.05
    o.set_gauge(o.represent_gauge_field(ub, bc))
    o.clover_init(1.0)
    o.compute_clover_term()
    lat3 = G.Lattice(*dims, ng, rep, ipt=o.geometry()[0])
    lat3.set_gauge(ub)
    lat3.represent_gauge_field(bc)
    assert lat3.link_recon() == 0
    lat3.clover_init(1.0)
    out3 = lat3.field(O.EVEN)
    lat3.g5Cphi_eopre(m, out3, lat3.field(O.EVEN, host=e))
    assert rel(out3.download(), o.g5Cphi_eopre(m, e)) < TOL64
