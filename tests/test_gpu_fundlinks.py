"""The NF = 6 two-index representations (SU(3) symmetric, SU(4) antisymmetric)
with the hopping kernels building each represented link from the fundamental
one (link modes 3 and 4; FP64, and FP32 from a float copy): every even-odd operator against the oracle
and against the kernels that read the stored represented links, for both
boundary conditions, with and without a clover term, and the rule that the mode
ends as soon as the fundamental links are written without a new
represent_gauge_field (HiRep's operators read u_gauge_f, which only
represent_gauge_field changes).
"""
import numpy as np
import pytest

import oracle as O
from hirep_b200 import fields as F
from hirep_b200 import hrgpu as G

pytestmark = pytest.mark.gpu

TOL64 = 1e-13


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def make(ng, rep, bc, dims=(4, 6, 4, 6), seed=23):
    o = O.Oracle(*dims, ng, rep)
    ipt, _, _ = o.geometry()
    u = F.smooth_gauge(seed, o.V, ng, 0.3)
    o.set_gauge(o.represent_gauge_field(u, bc))
    lat = G.Lattice(*dims, ng, rep, ipt=ipt)
    lat.set_gauge(u)
    lat.represent_gauge_field(bc)
    return o, u, lat


OPS = ["Dphi_eopre", "g5Dphi_eopre", "g5Dphi_eopre_sq"]
COPS = ["Cphi_eopre", "g5Cphi_eopre", "g5Cphi_eopre_sq"]


@pytest.mark.parametrize("bc", [True, False])
@pytest.mark.parametrize("ng,rep", [(3, O.SYM), (4, O.ASYM)])
def test_links_from_fundamental_match_oracle(bc, ng, rep):
    """Hop variant 6 (links built from the fundamental ones) against the oracle,
    and against variant 0 reading the stored links."""
    o, u, lat = make(ng, rep, bc)
    assert lat.link_recon() == (4 if bc else 3)
    G._check(lat.L.hrgpu_set_hop_variant(6), "set_hop_variant")
    try:
        m = -0.2
        e = F.gaussian_spinor(5, o.VH, o.nf)
        fe, out = lat.field(O.EVEN, host=e), lat.field(O.EVEN)
        got = {}
        for name in OPS:
            getattr(lat, name)(m, out, fe)
            got[name] = out.download()
            assert rel(got[name], getattr(o, name)(m, e)) < TOL64, name
        o.clover_init(1.0)
        o.compute_clover_term()
        lat.clover_init(1.0)
        for name in COPS:
            getattr(lat, name)(m, out, fe)
            got[name] = out.download()
            assert rel(got[name], getattr(o, name)(m, e)) < TOL64, name
        # the same operators reading the stored represented links
        G._check(lat.L.hrgpu_set_hop_variant(0), "set_hop_variant")
        for name in COPS:
            getattr(lat, name)(m, out, fe)
            assert rel(got[name], out.download()) < 1e-14, name
        # without the mode variant 6 is not built
        G._check(lat.L.hrgpu_set_link_recon(0), "set_link_recon")
        assert lat.link_recon() == 0
        G._check(lat.L.hrgpu_set_hop_variant(6), "set_hop_variant")
        with pytest.raises(G.HRGPUError, match="not built"):
            lat.Cphi_eopre(m, out, fe)
    finally:
        G._check(lat.L.hrgpu_set_link_recon(1), "set_link_recon")
        G._check(lat.L.hrgpu_set_hop_variant(-1), "set_hop_variant")


@pytest.mark.parametrize("bc", [True, False])
@pytest.mark.parametrize("ng,rep", [(3, O.SYM), (4, O.ASYM)])
def test_links_from_fundamental_fp32(bc, ng, rep):
    """The FP32 operators with variant 6 (the links built in FP32 from a float copy
    of the fundamental links) against the oracle's FP32 operators and against
    variant 0 reading the stored FP32 links, within the FP32 tolerance."""
    o, u, lat = make(ng, rep, bc)
    m = -0.2
    e = F.gaussian_spinor(5, o.VH, o.nf).astype(np.complex64)
    fe, out = lat.field(O.EVEN, G.FLOAT, host=e), lat.field(O.EVEN, G.FLOAT)
    try:
        got = {}
        for v in (6, 0):
            G._check(lat.L.hrgpu_set_hop_variant(v), "set_hop_variant")
            for name in ("Dphi_eopre_flt", "g5Dphi_eopre_flt", "g5Dphi_eopre_sq_flt"):
                getattr(lat, name)(m, out, fe)
                got[(v, name)] = out.download()
        for name in ("Dphi_eopre_flt", "g5Dphi_eopre_flt", "g5Dphi_eopre_sq_flt"):
            assert rel(got[(6, name)], getattr(o, name)(m, e)) < 2e-5, name
            assert rel(got[(6, name)], got[(0, name)]) < 2e-6, name
        o.clover_init(1.0)
        o.compute_clover_term()
        lat.clover_init(1.0)
        for v in (6, 0):
            G._check(lat.L.hrgpu_set_hop_variant(v), "set_hop_variant")
            lat.g5Cphi_eopre_flt(m, out, fe)
            got[(v, "c")] = out.download()
        assert rel(got[(6, "c")], got[(0, "c")]) < 2e-6
        assert rel(got[(6, "c")].astype(complex), o.g5Cphi_eopre(m, e.astype(complex))) < 2e-5
    finally:
        G._check(lat.L.hrgpu_set_hop_variant(-1), "set_hop_variant")


@pytest.mark.parametrize("ng,rep", [(3, O.SYM), (4, O.ASYM)])
def test_fundamental_write_ends_the_mode(ng, rep):
    """After new fundamental links without represent_gauge_field the operator still
    applies the represented links of the last represent_gauge_field."""
    o, u, lat = make(ng, rep, True)
    m = -0.2
    e = F.gaussian_spinor(7, o.VH, o.nf)
    fe, out = lat.field(O.EVEN, host=e), lat.field(O.EVEN)
    G._check(lat.L.hrgpu_set_hop_variant(6), "set_hop_variant")
    try:
        lat.Dphi_eopre(m, out, fe)
        before = out.download()
        lat.set_gauge(F.smooth_gauge(99, o.V, ng, 0.3))  # hrgpu_gauge_set only
        assert lat.link_recon() == 0
        G._check(lat.L.hrgpu_set_hop_variant(0), "set_hop_variant")
        lat.Dphi_eopre(m, out, fe)
        assert rel(out.download(), before) < 1e-14
        assert rel(out.download(), o.Dphi_eopre(m, e)) < TOL64
        lat.represent_gauge_field(True)  # the new links, and the mode again
        assert lat.link_recon() == 4
    finally:
        G._check(lat.L.hrgpu_set_hop_variant(-1), "set_hop_variant")


def test_tuned_variant_survives_the_end_of_the_mode():
    """The autotuner picks variant 6; after new fundamental links without
    represent_gauge_field the operator runs on the stored links (variant 0)."""
    o, u, lat = make(4, O.ASYM, True, dims=(4, 8, 8, 8))
    m = -0.2
    e = F.gaussian_spinor(9, o.VH, o.nf)
    fe, out = lat.field(O.EVEN, host=e), lat.field(O.EVEN)
    lat.Dphi_eopre(m, out, fe)  # tunes the FP64 hops
    ref = o.Dphi_eopre(m, e)
    assert rel(out.download(), ref) < TOL64
    lat.set_gauge(F.smooth_gauge(98, o.V, 4, 0.3))  # hrgpu_gauge_set only: the mode ends
    assert lat.link_recon() == 0
    lat.Dphi_eopre(m, out, fe)
    assert rel(out.download(), ref) < TOL64


def test_uploaded_represented_links_use_the_stored_form():
    """Links uploaded already represented (hrgpu_gauge_set_f) give mode 0."""
    o = O.Oracle(4, 4, 4, 4, 3, O.SYM)
    ipt, _, _ = o.geometry()
    u = F.smooth_gauge(3, o.V, 3, 0.3)
    uf = o.represent_gauge_field(u, True)
    lat = G.Lattice(4, 4, 4, 4, 3, O.SYM, ipt=ipt)
    lat.set_gauge(u)
    lat.represent_gauge_field(True)
    assert lat.link_recon() == 4
    lat.set_gauge_f(uf)
    assert lat.link_recon() == 0
