"""Pins the CPU oracle against HiRep's own tests for this path (CPU only).

Each test restates one of the reference's self-checking programs, with the
tolerance that program uses:
  TestProgram/DiracOperator/check_diracoperator_1.c  gauge covariance      < 1e-14
  TestProgram/DiracOperator/check_diracoperator_2.c  plane waves (free)    known answer
  TestProgram/DiracOperator/check_diracoperator_3.c  hermiticity g5D^2     < 1e-14
  TestProgram/DiracOperator/check_diracoperator_6.c  FP32 vs FP64 Dphi     < 1e-6
  TestProgram/Inverters/check_inverters_1.c          cg_mshift, 6 shifts   true residual < err2
  TestProgram/Inverters/check_inverters_6.c          cg_mshift_flt vs cg   < 10 err2
plus the geometry walk (first even sites of the serial 8^4 walk as printed by a
probe of the reference build) and the autosun generator conventions.
"""
import numpy as np
import pytest

import oracle as O
from hirep_b200 import fields as F

REPS = [(3, O.FUND), (2, O.ADJ), (3, O.SYM), (4, O.ASYM), (2, O.FUND), (3, O.ADJ)]


def _setup(dims, ng, rep, seed=1, smooth=None, bc=True):
    o = O.Oracle(*dims, ng, rep)
    u = F.hot_gauge(seed, o.V, ng) if smooth is None else F.smooth_gauge(seed, o.V, ng, smooth)
    uf = o.represent_gauge_field(u, bc)
    o.set_gauge(uf)
    return o, u, uf


def test_geometry_walk_pins():
    o = O.Oracle(8, 8, 8, 8, 3, O.FUND)
    ipt, iup, idn = o.geometry()
    V = o.V
    # serial walk puts even sites first and odd sites second
    coords = {}
    for t in range(8):
        for x in range(8):
            for y in range(8):
                for z in range(8):
                    ix = ipt[((t * 8 + x) * 8 + y) * 8 + z]
                    coords[ix] = (t, x, y, z)
                    assert (ix < V // 2) == ((t + x + y + z) % 2 == 0)
    assert sorted(coords) == list(range(V))
    # first even sites of the reference walk on 8^4: (0,0,0,0), (0,1,1,0), (0,1,0,1)
    assert coords[0] == (0, 0, 0, 0)
    assert coords[1] == (0, 1, 1, 0)
    assert coords[2] == (0, 1, 0, 1)
    # neighbours (check_geometry_1 style)
    for ix in range(V):
        c = coords[ix]
        for mu in range(4):
            up = list(c)
            up[mu] = (up[mu] + 1) % 8
            assert coords[iup[4 * ix + mu]] == tuple(up)
            assert idn[4 * iup[4 * ix + mu] + mu] == ix


@pytest.mark.parametrize("ng,rep", REPS)
def test_representation_conventions(ng, rep):
    o = O.Oracle(2, 2, 2, 2, ng, rep)
    rng = np.random.default_rng(3)
    u = F.haar_su_n(rng, 2, ng)
    Ra, Rb, Rab = (o.group_represent(m) for m in (u[0], u[1], u[0] @ u[1]))
    assert np.abs(Ra @ Rb - Rab).max() < 1e-13
    assert np.abs(Ra @ Ra.conj().T - np.eye(o.nf)).max() < 1e-13
    gT, rT, norms = o.generators()
    assert norms[0] == 0.5
    expect = {O.FUND: 0.5, O.ADJ: ng, O.SYM: (ng + 2) / 2, O.ASYM: (ng - 2) / 2}[rep]
    assert norms[1] == pytest.approx(expect)
    # Tr T_A T_B = delta_AB / 2
    tr = np.einsum("aij,bji->ab", gT, gT)
    assert np.abs(tr - 0.5 * np.eye(o.dimg)).max() < 1e-14
    # R(exp(eps X)) = 1 + eps R(X) + O(eps^2): _group_represent2 agrees with the generators
    h = rng.standard_normal(o.dimg)
    eps = 1e-6
    Xf = np.einsum("a,aij->ij", h, 1j * gT)
    Xr = np.einsum("a,aij->ij", h, rT)
    E = F.exp_i_hermitian((-1j * eps * Xf)[None])[0]
    assert np.abs((o.group_represent(E) - np.eye(o.nf)) / eps - Xr).max() < 1e-5
    assert np.abs(o.algebra_project(Xr.real if o.real else Xr) - h).max() < 1e-13


def _plane_wave_case(o, rng, hmass):
    T, X, Y, Z = o.dims
    ipt, _, _ = o.geometry()
    n = [rng.integers(0, L) for L in (T, X, Y, Z)]
    p = [2 * np.pi * n[k] / L for k, L in enumerate((T, X, Y, Z))]
    s = rng.standard_normal((4, o.nf)) + 1j * rng.standard_normal((4, o.nf))
    psi = np.zeros((o.V, 4, o.nf), complex)
    tt, xx, yy, zz = np.meshgrid(range(T), range(X), range(Y), range(Z), indexing="ij")
    ph = np.exp(1j * (p[0] * tt + p[1] * xx + p[2] * yy + p[3] * zz))
    psi[ipt.reshape(T, X, Y, Z)] = ph[..., None, None] * s
    mp = hmass + sum(1 - np.cos(q) for q in p)
    expect = mp * psi
    for mu in range(4):
        expect = expect + 1j * np.sin(p[mu]) * o.gamma(mu, psi)
    return psi, expect


def test_plane_waves_free_field():
    """check_diracoperator_2: Dphi on plane waves, unit links, periodic BCs."""
    for ng, rep in [(3, O.FUND), (2, O.ADJ)]:
        o = O.Oracle(4, 4, 4, 4, ng, rep)
        unit = np.broadcast_to(np.eye(ng, dtype=complex), (o.V, 4, ng, ng)).copy()
        o.set_gauge(o.represent_gauge_field(unit, bc_t_antiperiodic=False))
        rng = np.random.default_rng(7)
        for _ in range(5):
            psi, expect = _plane_wave_case(o, rng, 0.1)
            got = o.Dphi(0.1, psi)
            assert np.abs(got - expect).max() < 1e-13 * np.abs(expect).max() + 1e-14


def _gauge_transform(o, u, g):
    """U'(x,mu) = g(x) U(x,mu) g(x+mu)^+ on fundamental links."""
    _, iup, _ = o.geometry()
    up = np.empty_like(u)
    for mu in range(4):
        gy = g[iup[mu::4]]
        up[:, mu] = g @ u[:, mu] @ np.conj(np.swapaxes(gy, 1, 2))
    return up


@pytest.mark.parametrize("ng,rep", REPS)
def test_gauge_covariance(ng, rep):
    """check_diracoperator_1: ||D[U^g](g psi) - g D[U] psi|| < 1e-14 (normalised psi)."""
    o, u, uf = _setup((4, 4, 4, 4), ng, rep, seed=11)
    psi = F.gaussian_spinor(5, o.V, o.nf)
    psi /= np.sqrt(o.sqnorm(psi))
    d1 = o.Dphi(0.1, psi)
    g = F.haar_su_n(np.random.default_rng(9), o.V, ng)
    Rg = np.stack([o.group_represent(m) for m in g])
    o.set_gauge(o.represent_gauge_field(_gauge_transform(o, u, g), True))
    gpsi = np.einsum("xij,xsj->xsi", Rg, psi)
    d2 = o.Dphi(0.1, gpsi)
    diff = d2 - np.einsum("xij,xsj->xsi", Rg, d1)
    assert np.sqrt(o.sqnorm(diff)) < 1e-14 * 10


@pytest.mark.parametrize("ng,rep", REPS)
def test_hermiticity_eopre_sq(ng, rep):
    """check_diracoperator_3: <a, g5D_eo^2 b> = <g5D_eo^2 a, b>."""
    o, _, _ = _setup((4, 4, 4, 4), ng, rep, seed=2)
    a = F.gaussian_spinor(1, o.VH, o.nf)
    b = F.gaussian_spinor(2, o.VH, o.nf)
    Ma, Mb = o.g5Dphi_eopre_sq(0.1, a), o.g5Dphi_eopre_sq(0.1, b)
    lhs = np.vdot(a, Mb)
    rhs = np.vdot(Ma, b)
    assert abs(lhs - rhs) / abs(lhs) < 1e-14 * 10
    # g5 D is hermitian on the full lattice
    a = F.gaussian_spinor(3, o.V, o.nf)
    b = F.gaussian_spinor(4, o.V, o.nf)
    assert abs(np.vdot(a, o.g5Dphi(0.2, b)) - np.vdot(o.g5Dphi(0.2, a), b)) < 1e-11


def test_eopre_schur_complement():
    """Dphi_eopre = (4+m)^2 - D_eo D_oe on even sites, checked against the full operator."""
    o, _, _ = _setup((4, 4, 4, 4), 3, O.FUND, seed=4)
    m = -0.3
    e = F.gaussian_spinor(6, o.VH, o.nf)
    full = np.zeros((o.V, 4, o.nf), complex)
    full[: o.VH] = e
    # D_oe e, then D_eo of it, using the full-lattice hopping term
    h1 = o.Dphi_(full, O.FULL, O.FULL)
    h1[: o.VH] = 0
    h2 = o.Dphi_(h1, O.FULL, O.FULL)[: o.VH]
    expect = (4 + m) ** 2 * e - h2
    got = o.Dphi_eopre(m, e)
    assert np.abs(got - expect).max() < 1e-12


def test_float_vs_double_dphi():
    """check_diracoperator_6: FP32 Dphi agrees with FP64 to 1e-6 (relative norm)."""
    o, _, _ = _setup((4, 4, 4, 4), 3, O.FUND, seed=5)
    psi = F.gaussian_spinor(3, o.V, o.nf)
    d = o.Dphi(0.1, psi)
    f = o.Dphi_flt(0.1, psi.astype(np.complex64))
    assert np.sqrt(o.sqnorm(d - f) / o.sqnorm(d)) < 1e-6


def test_cg_mshift_six_shifts():
    """check_inverters_1: 6 shifts on g5Dphi_sq(-0.1), each true residual < err2."""
    o, _, _ = _setup((4, 4, 4, 4), 3, O.FUND, seed=6)
    o.set_mass(-0.1)
    shifts = [0.1, -0.21, 0.05, -0.01, -0.15, -0.05]
    err2 = 1e-28
    b = F.gaussian_spinor(8, o.V, o.nf) / np.sqrt(2.0)
    out, it = o.cg_mshift(O.OP_G5DPHI_SQ, shifts, err2, b)
    assert it > 0
    for i, s in enumerate(shifts):
        r = o.g5Dphi_sq(-0.1, out[i]) - s * out[i] - b
        assert o.sqnorm(r) / o.sqnorm(b) < err2


def test_cg_mshift_flt_vs_double():
    """check_inverters_6: mixed precision vs double on g5Dphi_eopre_sq(-1.2), err2 1e-20."""
    o, _, _ = _setup((4, 4, 4, 4), 3, O.FUND, seed=7)
    o.set_mass(-1.2)
    shifts = [-0.0, -0.1, -0.2, 0.1, 0.2, 0.3]
    err2 = 1e-20
    b = F.gaussian_spinor(9, o.VH, o.nf)
    x_f, _ = o.cg_mshift(O.OP_G5DPHI_EOPRE_SQ, shifts, err2, b, flt=True)
    x_d, _ = o.cg_mshift(O.OP_G5DPHI_EOPRE_SQ, shifts, err2, b)
    for i, s in enumerate(shifts):
        for x in (x_f[i], x_d[i]):
            r = o.g5Dphi_eopre_sq(-1.2, x) - s * x - b
            assert o.sqnorm(r) / o.sqnorm(b) < err2
        r = o.g5Dphi_eopre_sq(-1.2, x_f[i] - x_d[i]) - s * (x_f[i] - x_d[i])
        assert o.sqnorm(r) / o.sqnorm(b) < 10 * err2


@pytest.mark.parametrize("ng,rep", [(3, O.FUND), (2, O.ADJ), (3, O.SYM)])
def test_clover_inverse_and_hermiticity(ng, rep):
    o, _, _ = _setup((4, 4, 4, 4), ng, rep, seed=12, smooth=0.3)
    o.clover_init(1.0)
    o.compute_clover_term()
    m = -0.2
    psi = F.gaussian_spinor(1, o.VH, o.nf)
    back = o.Cphi_diag_inv(m, o.Cphi_diag(m, psi, O.ODD), O.ODD)
    assert np.abs(back - psi).max() < 1e-13
    a = F.gaussian_spinor(2, o.VH, o.nf)
    b = F.gaussian_spinor(3, o.VH, o.nf)
    lhs = np.vdot(a, o.g5Cphi_eopre_sq(m, b))
    rhs = np.vdot(o.g5Cphi_eopre_sq(m, a), b)
    assert abs(lhs - rhs) / abs(lhs) < 1e-13
    # the clover term is hermitian in each chiral block
    cl = o.clover_term()
    for blk in (0, 2):
        assert np.abs(cl[:, blk] - np.conj(np.swapaxes(cl[:, blk], 1, 2))).max() < 1e-14
    # clover eopre is the Schur complement of the full clover operator
    full = np.zeros((o.V, 4, o.nf), complex)
    full[: o.VH] = psi
    h = o.Dphi_(full, O.FULL, O.FULL)
    h[: o.VH] = 0
    h[o.VH:] = o.Cphi_diag_inv(m, h[o.VH:], O.ODD)
    h2 = o.Dphi_(h, O.FULL, O.FULL)[: o.VH]
    expect = o.Cphi_diag(m, psi, O.EVEN) - h2
    assert np.abs(o.Cphi_eopre(m, psi) - expect).max() < 1e-12


def test_smooth_field_plaquette():
    """exp(i 0.3 H) links give an average plaquette near 0.8 (config 2's field)."""
    o = O.Oracle(4, 4, 4, 4, 3, O.FUND)
    u = F.smooth_gauge(7, o.V, 3, 0.3)
    p = o.avr_plaquette(u)
    assert 0.7 < p < 0.9


# ---- g5QMR_mshift, MINRES, MRE (LibHR/Inverters/g5QMR_mshift.c, MINRES.c, LibHR/Update/mre.c)
SHIFTS6 = [0.1, -0.21, 0.05, -0.01, -0.15, -0.05]  # check_inverters_2.c:83-88, check_inverters_3.c:73-78


@pytest.mark.parametrize("op", [O.OP_DPHI_EOPRE, O.OP_DPHI])
def test_g5qmr_six_shifts(op):
    """check_inverters_3.c: g5QMR_mshift on D with six shifts, |D x - s x - b|^2/|b|^2 < err2."""
    o = O.Oracle(4, 4, 4, 4, 3, O.FUND)
    o.set_gauge(o.represent_gauge_field(F.hot_gauge(1234, o.V, 3), True))
    o.set_mass(0.1)
    par = O.FULL if op == O.OP_DPHI else O.EVEN
    b = F.gaussian_spinor(5, o.nsites(par), o.nf)
    err2 = 1e-26
    x, it = o.g5QMR_mshift(op, SHIFTS6, err2, b)
    D = o.Dphi if op == O.OP_DPHI else o.Dphi_eopre
    for i, s in enumerate(SHIFTS6):
        r = D(0.1, x[i]) - s * x[i] - b
        assert o.sqnorm(r) / o.sqnorm(b) < err2, (i, s)
    assert it > 0


def test_minres_hermitian_g5D():
    """check_inverters_2.c:111-141: MINRES on H = g5 D(m) with the mass moved by -shift,
    i.e. g5 (D - shift), each solve started from the previous solution."""
    o = O.Oracle(4, 4, 4, 4, 3, O.FUND)
    o.set_gauge(o.represent_gauge_field(F.hot_gauge(1234, o.V, 3), True))
    o.set_mass(0.1)
    b = F.gaussian_spinor(6, o.VH, o.nf)
    err2 = 1e-26
    prev = None
    for s in [0.0] + SHIFTS6[:-1]:
        x, it = o.MINRES(O.OP_DPHI_EOPRE, err2, b, trial=prev, g5=True, sh=s)
        r = o.gamma(5, o.Dphi_eopre(0.1, x) - s * x) - b
        assert o.sqnorm(r) / o.sqnorm(b) < err2
        prev = x


def _mre_numpy(o, D, sols, pf):
    """HiRep's mre_guess formula restated with numpy (Gram-Schmidt, A[j][i] = <D v_i, v_j>,
    b_i = <v_i, pf>, A y = conj(b), out = sum y_i v_i)."""
    v = [s.copy() for s in sols]
    for i in range(len(v)):
        v[i] = v[i] / np.sqrt(np.vdot(v[i], v[i]).real)
        for j in range(i + 1, len(v)):
            v[j] = v[j] - np.vdot(v[i], v[j]) * v[i]
    n = len(v)
    A = np.empty((n, n), complex)
    bb = np.empty(n, complex)
    for i in range(n):
        Dv = D(v[i])
        for j in range(n):
            A[j, i] = np.vdot(Dv, v[j])
        bb[i] = np.vdot(v[i], pf)
    y = np.linalg.solve(A, np.conj(bb))
    return sum(y[i] * v[i] for i in range(n))


def test_mre_guess_formula():
    o = O.Oracle(4, 4, 4, 4, 3, O.FUND)
    o.set_gauge(o.represent_gauge_field(F.smooth_gauge(3, o.V, 3, 0.3), True))
    o.set_mass(0.1)
    sols = [F.gaussian_spinor(20 + k, o.VH, o.nf) for k in range(5)]
    pf = F.gaussian_spinor(30, o.VH, o.nf)
    g = o.mre_guess(O.OP_DPHI_EOPRE, sols, pf)
    ref = _mre_numpy(o, lambda s: o.Dphi_eopre(0.1, s), sols, pf)
    assert np.abs(g - ref).max() / np.abs(ref).max() < 1e-12


# ---- HMC pieces (LibHR/Update/force0.c, field_update.c, local_action.c, suN_utils.c)
def _perturb(o, u, w, eps):
    gT = o.generators()[0]
    X = np.einsum("xma,aij->xmij", eps * w, gT)
    E = F.exp_i_hermitian(X.reshape(-1, o.ng, o.ng)).reshape(u.shape)
    return np.einsum("xmij,xmjk->xmik", E, u)


@pytest.mark.parametrize("ng", [2, 3])
def test_force0_is_minus_twice_gauge_action_derivative(ng):
    o = O.Oracle(4, 4, 4, 4, ng, O.FUND)
    u = F.smooth_gauge(4, o.V, ng, 0.4)
    beta = 2.25
    dimg = ng * ng - 1
    zero = np.zeros((o.V, 4, dimg))
    f = o.force0(1.0, beta, u, zero)
    w = np.random.default_rng(5).standard_normal((o.V, 4, dimg))
    S = lambda uu: o.local_hmc_action(beta, uu, zero).sum()
    eps = 1e-5
    fd = (S(_perturb(o, u, w, eps)) - S(_perturb(o, u, w, -eps))) / (2 * eps)
    an = -0.5 * np.sum(w * f)
    assert abs(fd - an) < 1e-7 * abs(an)


def test_update_exponential_and_projection():
    o = O.Oracle(4, 4, 4, 4, 3, O.FUND)
    u = F.smooth_gauge(6, o.V, 3, 0.3)
    mom = np.random.default_rng(7).standard_normal((o.V, 4, 8))
    dt = 0.05
    u2 = o.update_gauge_field(dt, u, mom)
    gT = o.generators()[0]
    X = np.einsum("xma,aij->xmij", dt * mom, gT)
    ref = np.einsum("xmij,xmjk->xmik", F.exp_i_hermitian(X.reshape(-1, 3, 3)).reshape(u.shape), u)
    assert np.abs(u2 - ref).max() < 1e-14
    # projection: SU(3) result, the identity on SU(3) input, a fix of a perturbed link
    p = o.project_gauge_field(u2)
    assert np.abs(p - u2).max() < 1e-13
    noisy = u2 + 1e-3 * np.random.default_rng(8).standard_normal(u2.shape)
    q = o.project_gauge_field(noisy).reshape(-1, 3, 3)
    assert np.abs(np.einsum("kij,klj->kil", q, q.conj()) - np.eye(3)).max() < 1e-14
    assert np.abs(np.linalg.det(q) - 1).max() < 1e-14


def test_local_action_is_momenta_plus_plaquette_action():
    o = O.Oracle(4, 4, 4, 4, 2, O.FUND)
    u = F.smooth_gauge(9, o.V, 2, 0.5)
    mom = np.random.default_rng(10).standard_normal((o.V, 4, 3))
    beta = 2.25
    loc = o.local_hmc_action(beta, u, mom)
    expect = 0.25 * np.sum(mom * mom) - beta / 2 * 6 * 2 * o.V * o.avr_plaquette(u)
    assert abs(loc.sum() - expect) < 1e-9 * abs(expect)


def test_pure_gauge_leapfrog_energy_violation_scales_as_dt_squared():
    o = O.Oracle(4, 4, 4, 4, 2, O.FUND)
    u0 = F.smooth_gauge(11, o.V, 2, 0.4)
    p0 = np.random.default_rng(12).standard_normal((o.V, 4, 3))
    beta, tau = 2.25, 0.5

    def dH(nsteps):
        dt = tau / nsteps
        u, p = u0.copy(), p0.copy()
        H0 = o.local_hmc_action(beta, u, p).sum()
        p = o.force0(dt / 2, beta, u, p)
        for s in range(nsteps):
            u = o.update_gauge_field(dt, u, p)
            p = o.force0(dt if s < nsteps - 1 else dt / 2, beta, u, p)
        return o.local_hmc_action(beta, u, p).sum() - H0

    d1, d2 = dH(10), dH(20)
    assert 3.5 < d1 / d2 < 4.5, (d1, d2)  # leapfrog: dH = O(dt^2)


# ---- exponential clover (Dphi.c:1292-1482, LibHR/Utils/clover_exp.c)
def _expclover_oracle(csw=1.0, ng=3, rep=O.FUND):
    o = O.Oracle(4, 4, 4, 4, ng, rep)
    o.set_gauge(o.represent_gauge_field(F.smooth_gauge(5, o.V, ng, 0.4), True))
    o.expclover_init(csw)
    o.compute_clover_term()
    return o


def test_expclover_diag_times_inverse_is_identity_and_matches_expm():
    import scipy.linalg as sl

    o = _expclover_oracle()
    m = -0.2
    e = F.gaussian_spinor(1, o.VH, o.nf)
    back = o.Cphi_diag_inv(m, o.Cphi_diag(m, e, O.EVEN), O.EVEN)
    assert np.abs(back - e).max() < 1e-13
    # site 0, chiral block 0 against scipy's expm of [[s0, s1], [s1^+, -s0]] / (4+m)
    cl = o.clover_term()[0]
    nf = o.nf
    A = np.block([[cl[0], cl[1]], [cl[1].conj().T, -cl[0]]])
    E = (4 + m) * sl.expm(A / (4 + m))
    v = np.zeros((o.VH, 4, nf), complex)
    v[0, 0, 0] = 1.0
    col = o.Cphi_diag(m, v, O.EVEN)[0, :2].reshape(-1)
    assert np.abs(col - E[:, 0]).max() < 1e-13


def test_expclover_is_the_clover_operator_at_small_csw():
    m = -0.2
    e = F.gaussian_spinor(2, 128, 3)
    out = {}
    for exp_, csw in ((True, 1e-4), (False, 1e-4)):
        o = O.Oracle(4, 4, 4, 4, 3, O.FUND)
        o.set_gauge(o.represent_gauge_field(F.smooth_gauge(5, o.V, 3, 0.4), True))
        (o.expclover_init if exp_ else o.clover_init)(csw)
        o.compute_clover_term()
        out[exp_] = o.Cphi_eopre(m, e)
    assert 0 < np.abs(out[True] - out[False]).max() / np.abs(out[False]).max() < 1e-8


def test_expclover_eopre_sq_hermitian():
    o = _expclover_oracle()
    m = -0.2
    a, b = F.gaussian_spinor(3, o.VH, o.nf), F.gaussian_spinor(4, o.VH, o.nf)
    lhs = np.vdot(a, o.g5Cphi_eopre_sq(m, b))
    rhs = np.vdot(o.g5Cphi_eopre_sq(m, a), b)
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)


def test_expclover_hmc_energy_violation_scales_as_dt_squared():
    """An oracle HMC trajectory with Nf=2 exponential clover fermions (csw=1.2,
    SU(3) fundamental, 4^4): dH falls as dt^2 (8 -> 16 steps: 3.95), so the
    exponential clover force is the derivative of the exponential clover action."""
    from hmc_oracle import oracle_trajectory
    from hirep_b200 import fields as F

    dh = {}
    for n in (8, 16):
        o = O.Oracle(4, 4, 4, 4, 3, O.FUND)
        u0 = F.smooth_gauge(98, o.V, 3, 0.2)
        dh[n], _ = oracle_trajectory(o, u0, 5.6, -0.3, 0.5, n, np.random.default_rng(15), 1e-26, 1e-28,
                                     expclover_csw=1.2)
    assert 3.5 < dh[8] / dh[16] < 4.5, dh


def test_clover_logdet_hmc_energy_violation_scales_as_dt_squared():
    """An oracle HMC trajectory with Nf=2 standard clover fermions, log-det terms
    included (clover_la_logdet in the action, force_clover_logdet in the force):
    dH falls as dt^2, so the log-det force is the derivative of the log-det action."""
    from hmc_oracle import oracle_trajectory
    from hirep_b200 import fields as F

    dh = {}
    for n in (8, 16):
        o = O.Oracle(4, 4, 4, 4, 3, O.FUND)
        u0 = F.smooth_gauge(97, o.V, 3, 0.2)
        dh[n], _ = oracle_trajectory(o, u0, 5.6, -0.3, 0.5, n, np.random.default_rng(16), 1e-26, 1e-28,
                                     clover_csw=1.2)
    assert 3.5 < dh[8] / dh[16] < 4.5, dh


def test_clover_la_logdet_is_log_det_of_the_odd_diagonal():
    """clover_la_logdet subtracts nf log det((4+m) + A) on every odd site
    (clover_tools.c:312-331), the determinant of the dense 2NF x 2NF blocks."""
    o = O.Oracle(4, 4, 4, 4, 2, O.FUND)
    from hirep_b200 import fields as F

    o.set_gauge(o.represent_gauge_field(F.smooth_gauge(3, o.V, 2, 0.4), True))
    o.clover_init(1.3)
    o.compute_clover_term()
    m = -0.4
    la = o.clover_la_logdet(2.0, m, np.zeros(o.V))
    assert np.all(la[: o.VH] == 0.0)
    cl = o.clover_term().reshape(o.V, 4, o.nf, o.nf)
    nf = o.nf
    for ix in (o.VH, o.VH + 7, o.V - 1):
        det = 1.0
        for b in range(2):
            s0, s1 = cl[ix, 2 * b], cl[ix, 2 * b + 1]
            blk = np.block([[s0, s1], [s1.conj().T, -s0]]) + (4 + m) * np.eye(2 * nf)
            det *= np.linalg.det(blk).real
        assert abs(la[ix] + 2.0 * np.log(det)) < 1e-12 * abs(la[ix])


@pytest.mark.parametrize("kind,ratio", [("o4mn", (14.0, 19.0)), ("leapfrog", (3.5, 4.5))])
def test_integrator_orders(kind, ratio):
    """Oracle trajectories with HiRep's O4MN (integrators.c:95-132) and leapfrog
    (:30-52) integrators: halving dt divides dH by 2^4 (measured 16.6 from 8 to
    16 steps) and by 2^2 (4.1), which pins their coefficients."""
    from hmc_oracle import oracle_trajectory
    from hirep_b200 import fields as F

    dh = {}
    for n in (8, 16):
        o = O.Oracle(4, 4, 4, 4, 2, O.ADJ)
        u0 = F.smooth_gauge(7, o.V, 2, 0.3)
        dh[n], _ = oracle_trajectory(o, u0, 2.25, -1.0, 0.5, n, np.random.default_rng(8), 1e-28, 1e-28,
                                     levels=[(kind, n, ("gauge", "fermion"))])
    assert ratio[0] < dh[8] / dh[16] < ratio[1], dh
