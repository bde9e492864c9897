"""The CPU oracle against golden fixtures written by HiRep itself
(tests/golden/make_golden.py, from the reference's own library built by
oracle/ref/Makefile).  Runs without the HiRep build: the fixtures hold HiRep's
outputs, the inputs are regenerated from their seeds."""
import os

import numpy as np
import pytest

import oracle as O
from hirep_b200 import fields as F

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = {
    "su3_fund": (3, O.FUND, False),
    "su3_fund_clover": (3, O.FUND, True),
    "su4_asym": (4, O.ASYM, False),
    "su2_adj": (2, O.ADJ, False),
    "su3_sym_clover": (3, O.SYM, True),
}
DIMS = (4, 4, 4, 4)
MASS, CSW, DT, RES = -0.1, 1.0, 0.37, 1.3


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def golden_inputs(cfg):
    """The fixture's inputs and an oracle set up on them, clover term included."""
    ng, rep, clover = CASES[cfg]
    g = np.load(os.path.join(GOLDEN, f"hirep_{cfg}.npz"))
    o = O.Oracle(*DIMS, ng, rep)
    u = F.smooth_gauge(7, o.V, ng, 0.3)
    uf = o.represent_gauge_field(u, True)
    o.set_gauge(uf)
    o.set_mass(MASS)
    if clover:
        o.clover_init(CSW)
        o.compute_clover_term()
    src = {"e": F.gaussian_spinor(1, o.VH, o.nf), "X": F.gaussian_spinor(11, o.V, o.nf),
           "Y": F.gaussian_spinor(12, o.V, o.nf), "u": u, "uf": uf}
    return g, o, src


@pytest.mark.parametrize("cfg", list(CASES))
def test_oracle_matches_hirep_fixture(cfg):
    g, o, s = golden_inputs(cfg)
    clover = CASES[cfg][2]
    assert rel(s["uf"][:2], g["gauge_f_head"]) < 1e-15
    eo = o.Cphi_eopre(MASS, s["e"]) if clover else o.Dphi_eopre(MASS, s["e"])
    assert rel(eo, g["eopre"]) < 1e-13
    if clover:
        cl = o.clover_term()
        assert rel(cl[:2], g["cl_term_head"]) < 1e-14
        assert abs((np.abs(cl) ** 2).sum() / g["cl_term_sqnorm"] - 1) < 1e-13
    op = O.OP_G5CPHI_EOPRE_SQ if clover else O.OP_G5DPHI_EOPRE_SQ
    x, mvm = o.cg_mshift(op, [0.1], 1e-28, s["e"], max_iter=5000)
    assert mvm == int(g["cg_mvm"])
    assert rel(x[0], g["cg"][0]) < 1e-12
    o.fermion_force_begin()
    o.force_fermion_core(s["X"], s["Y"], 1, DT, RES)
    f = o.fermion_force_end(DT, np.zeros((o.V, 4, o.dimg)))
    assert rel(f, g["force"]) < 1e-13


def test_oracle_geometry_matches_hirep_fixture():
    g = np.load(os.path.join(GOLDEN, "hirep_geometry_4x6x2x8.npz"))
    ipt, iup, idn = O.Oracle(4, 6, 2, 8, 3, O.FUND).geometry()
    assert np.array_equal(ipt, g["ipt"])
    assert np.array_equal(iup, g["iup"])
    assert np.array_equal(idn, g["idn"])
