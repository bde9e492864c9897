"""FP32 operators reading BF16 links (an experiment of this library; HiRep has
no reduced-precision link storage).  The operator result must differ from the
FP64 oracle at the BF16 rounding level (well above FP32 rounding, well below
1e-2), and the FP64 defect correction of cg_mshift_flt must still reach the
FP64 tolerance with it."""
import numpy as np
import pytest

import oracle as O
from hirep_b200 import fields as F
from hirep_b200 import hrgpu as G

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("ng,rep,clover", [(3, O.FUND, True), (2, O.ADJ, False), (3, O.SYM, False)])
def test_bf16_link_operator_error_band(ng, rep, clover):
    o = O.Oracle(4, 4, 4, 4, ng, rep)
    u = F.smooth_gauge(3, o.V, ng, 0.3)
    o.set_gauge(o.represent_gauge_field(u, True))
    lat = G.Lattice(4, 4, 4, 4, ng, rep, ipt=o.geometry()[0])
    lat.set_gauge(u)
    lat.represent_gauge_field(True)
    m = -0.2 if clover else 0.1
    if clover:
        o.clover_init(1.0)
        o.compute_clover_term()
        lat.clover_init(1.0)
    e = F.gaussian_spinor(4, o.VH, o.nf).astype(np.complex64)
    ref = (o.g5Cphi_eopre if clover else o.g5Dphi_eopre)(m, e.astype(complex))
    fi, fo = lat.field(O.EVEN, G.FLOAT, host=e), lat.field(O.EVEN, G.FLOAT)
    op = lat.g5Cphi_eopre_flt if clover else lat.g5Dphi_eopre_flt
    op(m, fo, fi)
    err32 = rel(fo.download(), ref)
    G._check(lat.L.hrgpu_set_flt_link_storage(G.LINKS_BF16), "set_flt_link_storage")
    try:
        op(m, fo, fi)
        err16 = rel(fo.download(), ref)
    finally:
        G._check(lat.L.hrgpu_set_flt_link_storage(G.LINKS_F32), "set_flt_link_storage")
    assert err32 < 1e-5
    assert 1e-4 < err16 < 1e-2, err16
    assert lat.L.hrgpu_set_flt_link_storage(7) == 2


@pytest.mark.parametrize("clover", [False, True])
def test_mixed_solve_with_bf16_links_reaches_fp64_tolerance(clover):
    o = O.Oracle(4, 4, 4, 8, 3, O.FUND)
    u = F.smooth_gauge(8, o.V, 3, 0.3)
    o.set_gauge(o.represent_gauge_field(u, True))
    lat = G.Lattice(4, 4, 4, 8, 3, G.FUND, ipt=o.geometry()[0])
    lat.set_gauge(u)
    lat.represent_gauge_field(True)
    m = -0.2 if clover else 0.1
    o.set_mass(m)
    if clover:
        o.clover_init(1.0)
        o.compute_clover_term()
        lat.clover_init(1.0)
    op = G.OP_G5CPHI_EOPRE_SQ if clover else G.OP_G5DPHI_EOPRE_SQ
    apply = o.g5Cphi_eopre_sq if clover else o.g5Dphi_eopre_sq
    b = F.gaussian_spinor(10, o.VH, o.nf)
    fb = lat.field(O.EVEN, host=b)
    shifts, err2 = [0.0, 0.05], 1e-24
    outs = [lat.field(O.EVEN) for _ in shifts]
    G._check(lat.L.hrgpu_set_flt_link_storage(G.LINKS_BF16), "set_flt_link_storage")
    try:
        it, ok = lat.cg_mshift(op, m, shifts, err2, fb, outs, flt=True)
    finally:
        G._check(lat.L.hrgpu_set_flt_link_storage(G.LINKS_F32), "set_flt_link_storage")
    assert ok
    xo, _ = o.cg_mshift(op, shifts, err2, b)
    for i, s in enumerate(shifts):
        x = outs[i].download()
        r = apply(m, x) - s * x - b
        assert o.sqnorm(r) / o.sqnorm(b) < err2
        assert rel(x, xo[i]) < 1e-9
