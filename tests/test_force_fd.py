"""Pseudofermion force against finite differences of the action.

S = phi^+ (H^2)^-1 phi with H = g5 D_eopre (Wilson or clover).  HiRep's force
(force_rhmc.c:79-94 with one pole b=0, a=1: X = (H^2)^-1 phi, Y = H X,
force_fermion_core(Y, X, 1, dt, 1)) is the momentum update of HiRep's MD, whose
kinetic term is 1/2 * C(F) * sum p^2 = 1/4 sum p^2 (local_action.c:63), and whose
link update is U -> exp(dt sum_A p_A iT_A) U (field_update.c:37, autosun ExpX).
Energy conservation then fixes F_A(x,mu) = -2 dS/d eps_A(x,mu) for
U(x,mu) -> exp(eps_A iT_A) U(x,mu).  The tests check that relation by central
differences along random algebra directions (step 1e-5; the GPU test uses the
fourth-order stencil, whose truncation error is far below the 1e-8 bound).

The GPU tests run the config-3 setup (SU(4), two-index antisymmetric, NF=6,
Wilson m0=-0.1, links exp(i 0.25 H), phi = D^+ eta) on a 4^4 lattice, through a
thin torch.autograd.Function whose backward is the GPU force kernel.
"""
import numpy as np
import pytest

import oracle as O
from hirep_b200 import fields as F


def perturbed(u, gT, w, eps):
    """exp(eps * sum_A w_A iT_A) U on every link."""
    ng = u.shape[-1]
    X = np.einsum("xma,aij->xmij", eps * w, gT)  # Hermitian
    E = F.exp_i_hermitian(X.reshape(-1, ng, ng)).reshape(u.shape)
    return np.einsum("xmij,xmjk->xmik", E, u)


@pytest.mark.parametrize("ng,rep,clover", [(2, O.FUND, False), (2, O.ADJ, False), (3, O.FUND, True),
                                            (3, O.SYM, False), (4, O.ASYM, False), (3, O.FUND, "exp"),
                                            (2, O.ADJ, "exp")])
def test_oracle_force_is_minus_twice_action_derivative(ng, rep, clover):
    o = O.Oracle(4, 4, 4, 4, ng, rep)
    m = -0.1
    o.set_mass(m)
    if clover == "exp":
        o.expclover_init(1.0)
    elif clover:
        o.clover_init(1.0)
    u = F.smooth_gauge(5, o.V, ng, 0.3)
    phi = F.gaussian_spinor(3, o.VH, o.nf)
    op = O.OP_G5CPHI_EOPRE_SQ if clover else O.OP_G5DPHI_EOPRE_SQ

    def action(links):
        o.set_gauge(o.represent_gauge_field(links, True))
        if clover:
            o.compute_clover_term()
        x, _ = o.cg_mshift(op, [0.0], 1e-30, phi)
        return np.vdot(phi, x[0]).real, x[0]

    _, X = action(u)
    Y = (o.g5Cphi_eopre if clover else o.g5Dphi_eopre)(m, X)
    Xs = np.zeros((o.V, 4, o.nf), complex)
    Ys = np.zeros_like(Xs)
    Xs[: o.VH], Ys[: o.VH] = Y, X
    o.fermion_force_begin()
    o.force_fermion_core(Xs, Ys, 1, 1.0, 1.0)
    force = o.fermion_force_end(1.0, np.zeros((o.V, 4, o.dimg)))
    gT, _, _ = o.generators()
    w = np.random.default_rng(1).standard_normal((o.V, 4, o.dimg))
    eps = 1e-5
    fd = (action(perturbed(u, gT, w, eps))[0] - action(perturbed(u, gT, w, -eps))[0]) / (2 * eps)
    an = -0.5 * np.sum(w * force)
    assert abs(fd - an) <= 1e-7 * abs(an)


class _Model:
    """GPU pseudofermion action S(U) = phi^+ (H^2)^-1 phi and its force, around links u0."""

    def __init__(self, lat, o, u0, phi, mass, err2, flt=False):
        from hirep_b200 import hrgpu as G

        self.G, self.lat, self.o = G, lat, o
        self.u0, self.mass, self.err2, self.flt = u0, mass, err2, flt
        self.gT = o.generators()[0]
        self.phi = lat.field(G.EVEN, host=phi)
        self.x = lat.field(G.EVEN)
        self.y = lat.field(G.EVEN)

    def links(self, omega):
        return perturbed(self.u0, self.gT, omega, 1.0)

    def action(self, omega):
        G, lat = self.G, self.lat
        lat.set_gauge(self.links(omega))
        lat.represent_gauge_field(True)
        lat.la("zero", self.x)
        _, ok = lat.cg_mshift(G.OP_G5DPHI_EOPRE_SQ, self.mass, [0.0], self.err2, self.phi, [self.x], flt=self.flt)
        assert ok
        return lat.prod_re(self.phi, self.x)

    def force(self):
        """HiRep force at the links of the last action() call (X = last solution)."""
        G, lat, o = self.G, self.lat, self.o
        lat.set_dirac_mass(self.mass)
        lat.g5Dphi_eopre(self.mass, self.y, self.x)
        xe, ye = self.x.download(), self.y.download()
        Xs = np.zeros((o.V, 4, o.nf), complex)
        Ys = np.zeros_like(Xs)
        Xs[: o.VH], Ys[: o.VH] = ye, xe
        fX, fY = lat.field(G.FULL, host=Xs), lat.field(G.FULL, host=Ys)
        lat.fermion_force_begin()
        lat.force_fermion_core(fX, fY, 1, 1.0, 1.0)
        return lat.fermion_force_end(1.0, np.zeros((o.V, 4, o.dimg)))


def _autograd_action():
    import torch

    class PseudofermionAction(torch.autograd.Function):
        """S(omega) = phi^+ (H^2)^-1 phi at links exp(omega iT) u0; backward = -F/2 (GPU force kernel).

        The backward is exact at omega = 0, which is where the test evaluates it."""

        @staticmethod
        def forward(ctx, omega, model):
            ctx.model = model
            return torch.tensor(model.action(omega.detach().cpu().numpy()), dtype=torch.float64)

        @staticmethod
        def backward(ctx, g):
            force = ctx.model.force()
            return g * torch.from_numpy(-0.5 * force), None

    return PseudofermionAction


def _config3_setup(flt=False):
    from hirep_b200 import hrgpu as G

    dims, ng, m = (4, 4, 4, 4), 4, -0.1
    o = O.Oracle(*dims, ng, O.ASYM)
    ipt, _, _ = o.geometry()
    u0 = F.smooth_gauge(11, o.V, ng, 0.25)
    lat = G.Lattice(*dims, ng, G.ASYM, ipt=ipt)
    lat.set_gauge(u0)
    lat.represent_gauge_field(True)
    # phi = D^+ eta = g5 D g5 eta on the even sites
    eta = F.gaussian_spinor(11, o.VH, o.nf)
    g5 = np.array([1, 1, -1, -1])[None, :, None]
    fe, tmp = lat.field(G.EVEN, host=g5 * eta), lat.field(G.EVEN)
    lat.Dphi_eopre(m, tmp, fe)
    phi = g5 * tmp.download()
    return _Model(lat, o, u0, phi, m, 1e-28 if not flt else 1e-26, flt=flt), o


@pytest.mark.gpu
def test_gpu_force_matches_finite_differences_su4_antisymmetric():
    import torch

    model, o = _config3_setup()
    Action = _autograd_action()
    omega = torch.zeros((o.V, 4, o.dimg), dtype=torch.float64, requires_grad=True)
    S = Action.apply(omega, model)
    S.backward()
    grad = omega.grad.numpy()
    rng = np.random.default_rng(32)
    eps = 1e-5
    worst = 0.0
    for _ in range(32):
        d = rng.standard_normal((o.V, 4, o.dimg))
        # central differences with step 1e-5, fourth-order stencil so that the
        # eps^2 truncation term does not mask the comparison
        s1 = model.action(eps * d) - model.action(-eps * d)
        s2 = model.action(2 * eps * d) - model.action(-2 * eps * d)
        fd = (8 * s1 - s2) / (12 * eps)
        an = float(np.sum(grad * d))
        worst = max(worst, abs(fd - an) / abs(an))
    assert worst < 1e-8, worst


@pytest.mark.gpu
def test_gpu_force_matches_oracle_force_su4_antisymmetric():
    model, o = _config3_setup()
    model.action(np.zeros((o.V, 4, o.dimg)))
    fg = model.force()
    uf = o.represent_gauge_field(model.u0, True)
    o.set_gauge(uf)
    o.set_mass(model.mass)
    xe = model.x.download()
    ye = o.g5Dphi_eopre(model.mass, xe)
    Xs = np.zeros((o.V, 4, o.nf), complex)
    Ys = np.zeros_like(Xs)
    Xs[: o.VH], Ys[: o.VH] = ye, xe
    o.fermion_force_begin()
    o.force_fermion_core(Xs, Ys, 1, 1.0, 1.0)
    fo = o.fermion_force_end(1.0, np.zeros((o.V, 4, o.dimg)))
    assert np.abs(fg - fo).max() / np.abs(fo).max() < 1e-12


@pytest.mark.gpu
def test_gpu_force_mixed_precision_solve():
    """Force from an X solved by the FP32-inner defect-correction CG: error against the FP64 force."""
    model64, o = _config3_setup()
    model64.action(np.zeros((o.V, 4, o.dimg)))
    f64 = model64.force()
    model32, _ = _config3_setup(flt=True)
    model32.action(np.zeros((o.V, 4, o.dimg)))
    f32 = model32.force()
    err = np.abs(f32 - f64).max() / np.abs(f64).max()
    assert err < 1e-9, err


@pytest.mark.gpu
def test_library_generators_are_the_oracle_basis():
    from hirep_b200 import hrgpu as G

    for ng, rep in ((2, O.ADJ), (3, O.FUND), (4, O.ASYM)):
        o = O.Oracle(4, 4, 4, 4, ng, rep)
        lat = G.Lattice(4, 4, 4, 4, ng, {O.FUND: G.FUND, O.ADJ: G.ADJ, O.ASYM: G.ASYM}[rep], ipt=o.geometry()[0])
        assert np.abs(lat.generators() - o.generators()[0]).max() < 1e-15
