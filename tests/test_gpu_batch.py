"""Batched (multi-right-hand-side) operators and inverter against the CPU oracle.

The batch entry points have no HiRep counterpart of their own: each field of a
batch must give what HiRep's single-field function gives for it (Dphi.c for the
operators; cg_mshift.c / cg_mshift_flt.c per source for the solver).  FP64 to
1e-13 relative, FP32 to 1e-5; solver residuals below err2 as HiRep checks them.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from hirep_b200 import fields as F
from hirep_b200 import hrgpu as G

pytestmark = pytest.mark.gpu

TOL64 = 1e-13


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def setup(dims, ng, rep, seed=1, smooth=0.3, clover=None):
    o = O.Oracle(*dims, ng, rep)
    ipt, _, _ = o.geometry()
    u = F.smooth_gauge(seed, o.V, ng, smooth)
    uf = o.represent_gauge_field(u, True)
    o.set_gauge(uf)
    lat = G.Lattice(*dims, ng, rep, ipt=ipt)
    lat.set_gauge(u)
    lat.represent_gauge_field(True)
    if clover is not None:
        o.clover_init(clover)
        o.compute_clover_term()
        lat.clover_init(clover)
    return o, lat


def test_batch_layout_and_roundtrip():
    o, lat = setup((4, 4, 4, 4), 3, O.FUND)
    nb = 5
    hs = [F.gaussian_spinor(10 + i, o.VH, o.nf) for i in range(nb)]
    fs = [lat.field(O.EVEN, host=h) for h in hs]
    b = lat.batch(nb, fields=fs)
    # tiles of 4 fields, blocks of 8 sites: element (c, n, f) of the batch at
    # (((f//4)*ld/8 + n//8)*4NF + c)*32 + (n%8)*4 + f%4 is element (c, n) of field f,
    # stored at c*ld + n
    ncomp = 4 * o.nf
    ld = fs[0].nbytes // 16 // ncomp
    ntile = (nb + 3) // 4
    assert b.nbytes == ntile * 4 * fs[0].nbytes
    raw = b.buf.cpu().numpy().view(np.complex128).reshape(ntile, ld // 8, ncomp, 8, 4)
    for f in range(nb):
        single = fs[f].buf.cpu().numpy().view(np.complex128).reshape(ncomp, ld // 8, 8)
        assert np.array_equal(raw[f // 4, :, :, :, f % 4].transpose(1, 0, 2), single)
    # the padding field of the last tile stays zero
    assert not raw[ntile - 1, :, :, :, nb % 4:].any()
    back = [lat.field(O.EVEN) for _ in range(nb)]
    b.unpack(back)
    for f in range(nb):
        assert np.array_equal(back[f].download(), hs[f])
    # float batch
    f32 = [lat.field(O.EVEN, G.FLOAT, host=h.astype(np.complex64)) for h in hs]
    b32 = lat.batch(nb, G.FLOAT, fields=f32)
    back32 = [lat.field(O.EVEN, G.FLOAT) for _ in range(nb)]
    b32.unpack(back32)
    for f in range(nb):
        assert np.array_equal(back32[f].download(), hs[f].astype(np.complex64))


OPS_W = [(G.OP_DPHI_EOPRE, "Dphi_eopre"), (G.OP_G5DPHI_EOPRE, "g5Dphi_eopre"),
         (G.OP_G5DPHI_EOPRE_SQ, "g5Dphi_eopre_sq")]
OPS_C = [(G.OP_CPHI_EOPRE, "Cphi_eopre"), (G.OP_G5CPHI_EOPRE, "g5Cphi_eopre"),
         (G.OP_G5CPHI_EOPRE_SQ, "g5Cphi_eopre_sq")]


@pytest.mark.parametrize("nb", [1, 3, 12])
@pytest.mark.parametrize("ng,rep,clover", [(3, O.FUND, False), (2, O.ADJ, False), (4, O.ASYM, False),
                                           (3, O.SYM, True), (2, O.FUND, True)])
def test_batch_operators_match_oracle(ng, rep, clover, nb):
    o, lat = setup((4, 4, 4, 4), ng, rep, seed=3, clover=1.0 if clover else None)
    m = -0.2 if clover else 0.1
    hs = [F.gaussian_spinor(20 + i, o.VH, o.nf) for i in range(nb)]
    fs = [lat.field(O.EVEN, host=h) for h in hs]
    bin_, bout = lat.batch(nb, fields=fs), lat.batch(nb)
    outs = [lat.field(O.EVEN) for _ in range(nb)]
    for op, name in (OPS_C if clover else OPS_W):
        lat.apply_op_batch(op, m, bout, bin_)
        bout.unpack(outs)
        for f in range(nb):
            assert rel(outs[f].download(), getattr(o, name)(m, hs[f])) < TOL64, (name, f)
    # the FP32 batch against the oracle on the rounded inputs
    f32 = [lat.field(O.EVEN, G.FLOAT, host=h.astype(np.complex64)) for h in hs]
    b32, o32 = lat.batch(nb, G.FLOAT, fields=f32), lat.batch(nb, G.FLOAT)
    outs32 = [lat.field(O.EVEN, G.FLOAT) for _ in range(nb)]
    op, name = (OPS_C if clover else OPS_W)[1]
    lat.apply_op_batch(op, m, o32, b32)
    o32.unpack(outs32)
    for f in range(nb):
        ref = getattr(o, name)(m, hs[f].astype(np.complex64).astype(complex))
        assert rel(outs32[f].download(), ref) < 1e-5


def test_batch_operator_equals_single_field_operator():
    """Same per-site arithmetic as the one-thread-per-site single-field kernel."""
    o, lat = setup((4, 4, 4, 8), 3, O.FUND, seed=4, clover=1.0)
    G._check(lat.L.hrgpu_set_hop_variant(0), "set_hop_variant")
    try:
        m, nb = -0.2, 4
        hs = [F.gaussian_spinor(30 + i, o.VH, o.nf) for i in range(nb)]
        fs = [lat.field(O.EVEN, host=h) for h in hs]
        bin_, bout = lat.batch(nb, fields=fs), lat.batch(nb)
        lat.apply_op_batch(G.OP_G5CPHI_EOPRE, m, bout, bin_)
        outs = [lat.field(O.EVEN) for _ in range(nb)]
        bout.unpack(outs)
        one = lat.field(O.EVEN)
        for f in range(nb):
            lat.g5Cphi_eopre(m, one, fs[f])
            assert rel(outs[f].download(), one.download()) < 1e-15
    finally:
        G._check(lat.L.hrgpu_set_hop_variant(-1), "set_hop_variant")


def _residual_ok(o, apply, m, x, s, b, err2):
    r = apply(m, x) - s * x - b
    return o.sqnorm(r) / o.sqnorm(b) < err2


@pytest.mark.parametrize("flt", [False, True])
@pytest.mark.parametrize("clover", [False, True])
def test_cg_mshift_batch_matches_per_source_cg(clover, flt):
    o, lat = setup((4, 4, 4, 8), 3, O.FUND, seed=8, clover=1.0 if clover else None)
    m = -0.2 if clover else 0.1
    o.set_mass(m)
    op = G.OP_G5CPHI_EOPRE_SQ if clover else G.OP_G5DPHI_EOPRE_SQ
    apply = o.g5Cphi_eopre_sq if clover else o.g5Dphi_eopre_sq
    shifts = [[0.0, -0.05, -0.4], [0.0], [-0.01, 0.0]]
    err2 = 1e-24
    hs = [F.gaussian_spinor(40 + i, o.VH, o.nf) for i in range(len(shifts))]
    srcs = [lat.field(O.EVEN, host=h) for h in hs]
    outs = [lat.field(O.EVEN) for s in shifts for _ in s]
    its, ok = lat.cg_mshift_batch(op, m, srcs, shifts, err2, outs, flt=flt)
    assert ok
    j = 0
    for s, sh in enumerate(shifts):
        xo, it_o = o.cg_mshift(op, sh, err2, hs[s])
        for i, sig in enumerate(sh):
            x = outs[j].download()
            assert _residual_ok(o, apply, m, x, sig, hs[s], err2), (s, i)
            assert rel(x, xo[i]) < 1e-9
            j += 1
        if not flt:
            assert abs(int(its[s]) - it_o) <= 3, (its, it_o)


def test_cg_mshift_batch_point_sources_sextet_clover():
    """Config-4 shape on a small lattice: SU(3) two-index symmetric (NF=6), clover,
    12 spin-colour point sources at the origin (colours 0-2 x 4 spins), source 0
    also solved for 10 shifts log-spaced 1e-4..10 (HiRep passes shift = -sigma)."""
    o, lat = setup((4, 4, 4, 8), 3, O.SYM, seed=21, clover=1.0)
    m = -0.3
    o.set_mass(m)
    sig = np.logspace(-4, 1, 10)
    shifts = [[0.0] + list(-sig)] + [[0.0] for _ in range(11)]
    hs = [F.point_source(o.VH, o.nf, spin=b, col=c) for c in range(3) for b in range(4)]
    srcs = [lat.field(O.EVEN, host=h) for h in hs]
    outs = [lat.field(O.EVEN) for s in shifts for _ in s]
    err2 = 1e-24
    its, ok = lat.cg_mshift_batch(G.OP_G5CPHI_EOPRE_SQ, m, srcs, shifts, err2, outs, flt=True)
    assert ok
    j = 0
    for s, sh in enumerate(shifts):
        for sg in sh:
            x = outs[j].download()
            assert _residual_ok(o, o.g5Cphi_eopre_sq, m, x, sg, hs[s], err2), (s, sg)
            j += 1
    # against HiRep's sequential FP64 solves (oracle) for source 0's shifts
    xo, _ = o.cg_mshift(G.OP_G5CPHI_EOPRE_SQ, shifts[0], err2, hs[0])
    for i in range(len(shifts[0])):
        assert rel(outs[i].download(), xo[i]) < 1e-9


def test_cg_mshift_batch_edge_cases():
    o, lat = setup((4, 4, 4, 4), 2, O.ADJ, seed=9)
    m = 0.1
    o.set_mass(m)
    op = G.OP_G5DPHI_EOPRE_SQ
    h = F.gaussian_spinor(50, o.VH, o.nf)
    zero = lat.field(O.EVEN)
    src = lat.field(O.EVEN, host=h)
    outs = [lat.field(O.EVEN, host=h) for _ in range(3)]  # non-zero junk: the solver starts from zero
    its, ok = lat.cg_mshift_batch(op, m, [zero, src], [[0.0, -0.2], [0.0]], 1e-24, outs, flt=True)
    assert ok
    assert np.abs(outs[0].download()).max() == 0 and np.abs(outs[1].download()).max() == 0
    assert _residual_ok(o, o.g5Dphi_eopre_sq, m, outs[2].download(), 0.0, h, 1e-24)
    # max_iter reached: reported, not fatal
    its, ok = lat.cg_mshift_batch(op, m, [src], [[0.0]], 1e-60, outs[:1], max_iter=5)
    assert not ok
    # argument errors
    L = lat.L
    one = (ctypes.c_void_p * 1)(src.ptr.value)
    o1 = (ctypes.c_void_p * 1)(outs[0].ptr.value)
    it = np.zeros(64, np.int32)
    nsh = np.ones(64, np.int32)
    sh = np.zeros(128, np.float64)
    D = ctypes.c_double
    assert L.hrgpu_cg_mshift_batch(G.OP_G5DPHI_SQ, D(m), 1, G._ptr(nsh), G._ptr(sh), D(1e-20), 0, one, o1, 0,
                                   G._ptr(it)) == 2  # full-lattice operator: no batched form
    assert L.hrgpu_cg_mshift_batch(op, D(m), 33, G._ptr(nsh), G._ptr(sh), D(1e-20), 0, one, o1, 0,
                                   G._ptr(it)) == 2  # too many sources
    big = np.full(1, 65, np.int32)
    assert L.hrgpu_cg_mshift_batch(op, D(m), 1, G._ptr(big), G._ptr(sh), D(1e-20), 0, one, o1, 0,
                                   G._ptr(it)) == 2  # too many systems
    alias = (ctypes.c_void_p * 1)(src.ptr.value)
    assert L.hrgpu_cg_mshift_batch(op, D(m), 1, G._ptr(nsh), G._ptr(sh), D(1e-20), 0, one, alias, 0,
                                   G._ptr(it)) == 2  # output aliases the source
    assert "alias" in L.hrgpu_last_error().decode()
    b1 = lat.batch(2)
    assert L.hrgpu_apply_op_batch(G.OP_G5DPHI_SQ, 0, D(m), b1.ptr, b1.ptr, 2) == 2


@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("ng,rep,clover", [(3, O.FUND, True), (2, O.ADJ, False), (3, O.SYM, True)])
def test_batch_variants(variant, ng, rep, clover):
    o, lat = setup((4, 4, 4, 4), ng, rep, seed=12, clover=1.0 if clover else None)
    G._check(lat.L.hrgpu_set_batch_variant(variant), "set_batch_variant")
    try:
        m, nb = (-0.2 if clover else 0.1), 5
        hs = [F.gaussian_spinor(60 + i, o.VH, o.nf) for i in range(nb)]
        fs = [lat.field(O.EVEN, host=h) for h in hs]
        bin_, bout = lat.batch(nb, fields=fs), lat.batch(nb)
        outs = [lat.field(O.EVEN) for _ in range(nb)]
        op, name = (OPS_C if clover else OPS_W)[2]
        lat.apply_op_batch(op, m, bout, bin_)
        bout.unpack(outs)
        for f in range(nb):
            assert rel(outs[f].download(), getattr(o, name)(m, hs[f])) < TOL64
    finally:
        G._check(lat.L.hrgpu_set_batch_variant(-1), "set_batch_variant")


@pytest.mark.parametrize("ng,rep,clover", [(3, O.FUND, True), (3, O.SYM, True), (4, O.ASYM, False), (2, O.FUND, False)])
def test_batch_packed_fma_variant(ng, rep, clover):
    """Variant 5, the link products in packed FP32 FMAs (fma.rn.f32x2), for the
    complex representations in FP32: every field against the FP32 single-field
    operator (2e-6) and the oracle's FP64 operator (1e-5); in FP64 and for the
    real representations the variant is not built."""
    o, lat = setup((4, 4, 4, 8), ng, rep, seed=17, clover=1.0 if clover else None)
    G._check(lat.L.hrgpu_set_batch_variant(5), "set_batch_variant")
    try:
        m, nb = (-0.3 if clover else -0.1), 7
        ops = OPS_C[1:] if clover else OPS_W
        hs = [F.gaussian_spinor(90 + i, o.VH, o.nf) for i in range(nb)]
        fs = [lat.field(O.EVEN, G.FLOAT, host=h.astype(np.complex64)) for h in hs]
        bin_, bout = lat.batch(nb, G.FLOAT, fields=fs), lat.batch(nb, G.FLOAT)
        outs = [lat.field(O.EVEN, G.FLOAT) for _ in range(nb)]
        single = lat.field(O.EVEN, G.FLOAT)
        for op, name in ops:
            lat.apply_op_batch(op, m, bout, bin_)
            bout.unpack(outs)
            for f in (0, nb // 2, nb - 1):
                getattr(lat, name + "_flt")(m, single, fs[f])
                assert rel(outs[f].download(), single.download()) < 2e-6, (name, f)
                assert rel(outs[f].download().astype(complex), getattr(o, name)(m, hs[f])) < 1e-5, (name, f)
        b64i, b64o = lat.batch(nb), lat.batch(nb)
        with pytest.raises(G.HRGPUError, match="not built"):
            lat.apply_op_batch(ops[0][0], m, b64o, b64i)
    finally:
        G._check(lat.L.hrgpu_set_batch_variant(-1), "set_batch_variant")


def test_batch_autotuner_reports_its_choice():
    o, lat = setup((4, 4, 4, 4), 3, O.FUND, seed=13, clover=1.0)
    nb = 7
    bi, bo = lat.batch(nb), lat.batch(nb)
    lat.apply_op_batch(G.OP_G5CPHI_EOPRE, -0.2, bo, bi)
    chosen = ctypes.c_int(-2)
    ms = (ctypes.c_float * 6)()
    for ep in (1, 2):  # the two clover epilogues ran
        G._check(lat.L.hrgpu_batch_tuning(G.DOUBLE, ep, nb, ctypes.byref(chosen), ms), "batch_tuning")
        assert 0 <= chosen.value < 3
        assert all(t > 0 for t in ms[:3]) and ms[3] == ms[4] == -1.0  # the tensor-core variants run only when pinned
        assert ms[5] == -1.0  # the packed-FMA variant is FP32 only
    G._check(lat.L.hrgpu_batch_tuning(G.FLOAT, 0, nb, ctypes.byref(chosen), ms), "batch_tuning")
    assert chosen.value == -1  # not tuned: never ran


@pytest.mark.parametrize("variant,nb", [(3, 5), (3, 12), (3, 32), (4, 5), (4, 12), (4, 16)])
@pytest.mark.parametrize("ng,rep,clover", [(3, O.SYM, True), (4, O.ASYM, False)])
def test_batch_tensor_core_variant(variant, nb, ng, rep, clover):
    """Variants 3 and 4, the link products on the tensor cores (tcgen05, kind::tf32,
    three products for FP32 accuracy), for the NF = 6 representations: every field
    of the FP32 batched operator against the FP32 single-field operator (2e-6, the
    FP32 operators' tolerance) and against the oracle's FP64 operator; a batch of
    more than 32 (variant 3) or 16 (variant 4) fields is refused."""
    o, lat = setup((4, 4, 4, 8), ng, rep, seed=17, clover=1.0 if clover else None)
    G._check(lat.L.hrgpu_set_batch_variant(variant), "set_batch_variant")
    try:
        m = -0.3 if clover else -0.1
        ops = OPS_C[1:] if clover else OPS_W  # (the clover operators have FP32 forms with gamma_5)
        hs = [F.gaussian_spinor(80 + i, o.VH, o.nf) for i in range(nb)]
        fs = [lat.field(O.EVEN, G.FLOAT, host=h.astype(np.complex64)) for h in hs]
        bin_, bout = lat.batch(nb, G.FLOAT, fields=fs), lat.batch(nb, G.FLOAT)
        outs = [lat.field(O.EVEN, G.FLOAT) for _ in range(nb)]
        single = lat.field(O.EVEN, G.FLOAT)
        for op, name in ops:
            lat.apply_op_batch(op, m, bout, bin_)
            bout.unpack(outs)
            for f in sorted({0, nb // 2, nb - 1}):
                getattr(lat, name + "_flt")(m, single, fs[f])
                assert rel(outs[f].download(), single.download()) < 2e-6, (name, f)
                assert rel(outs[f].download().astype(complex), getattr(o, name)(m, hs[f])) < 2e-6, (name, f)
        if nb == (32 if variant == 3 else 16):
            big_in, big_out = lat.batch(nb + 1, G.FLOAT), lat.batch(nb + 1, G.FLOAT)
            with pytest.raises(G.HRGPUError, match="not built"):
                lat.apply_op_batch(ops[0][0], m, big_out, big_in)
    finally:
        G._check(lat.L.hrgpu_set_batch_variant(-1), "set_batch_variant")
