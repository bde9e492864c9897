"""hrgpu_apply_op_host: an even-odd preconditioned operator on a host field
(HiRep layout and site order) with the copies overlapped slab by slab.  Every
site is computed by the whole-lattice kernels, so the result must be
bit-identical to upload + operator + download, for any chunking and any
even-first site order; and it matches the oracle (Dphi.c:874-985, :1240-1261)."""
import numpy as np
import pytest

import oracle as O
from hirep_b200 import fields as F
from hirep_b200 import hrgpu as G

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def random_even_first_ipt(dims, seed):
    """A random site order with the even sites first (any permutation HiRep's
    lattice_init accepts), so chunks of host order touch arbitrary time slabs."""
    T, X, Y, Z = dims
    rng = np.random.default_rng(seed)
    coords = [(t, x, y, z) for t in range(T) for x in range(X) for y in range(Y) for z in range(Z)]
    even = [c for c in coords if sum(c) % 2 == 0]
    odd = [c for c in coords if sum(c) % 2 == 1]
    order = [even[i] for i in rng.permutation(len(even))] + [odd[i] for i in rng.permutation(len(odd))]
    ipt = np.empty(T * X * Y * Z, np.int32)
    for h, (t, x, y, z) in enumerate(order):
        ipt[((t * X + x) * Y + y) * Z + z] = h
    return ipt


def make(dims, ng, rep, ipt=None, clover=True):
    o = O.Oracle(*dims, ng, rep)
    u = F.smooth_gauge(3, o.V, ng, 0.3)
    if ipt is None:
        ipt = o.geometry()[0]
    lat = G.Lattice(*dims, ng, rep, ipt=ipt)
    lat.set_gauge(u)
    lat.represent_gauge_field(True)
    if clover:
        lat.clover_init(1.0)
    return o, u, lat


OPS = {G.OP_DPHI_EOPRE: "Dphi_eopre", G.OP_G5DPHI_EOPRE: "g5Dphi_eopre", G.OP_CPHI_EOPRE: "Cphi_eopre",
       G.OP_G5CPHI_EOPRE: "g5Cphi_eopre"}


@pytest.mark.parametrize("chunks", [1, 3, 8, 64])
@pytest.mark.parametrize("dims,ng,rep,order", [((8, 4, 4, 4), 3, O.FUND, "hirep"), ((6, 4, 2, 4), 2, O.ADJ, "random"),
                                               ((4, 4, 4, 4), 3, O.SYM, "hirep"), ((2, 4, 4, 2), 3, O.FUND, "random")])
def test_apply_op_host_is_bit_identical(chunks, dims, ng, rep, order):
    ipt = random_even_first_ipt(dims, 5) if order == "random" else None
    o, u, lat = make(dims, ng, rep, ipt)
    lat.set_host_chunks(chunks)
    m = -0.2
    e = F.gaussian_spinor(7, lat.VH, lat.nf)
    fin, fout = lat.field(G.EVEN, host=e), lat.field(G.EVEN)
    for op, name in OPS.items():
        ref = (getattr(lat, name)(m, fout, fin), fout.download())[1]
        got = lat.apply_op_host(op, m, e)
        assert np.array_equal(got, ref), (name, np.abs(got - ref).max())
    # FP32: the float operators on a complex64 host field
    e32 = e.astype(np.complex64)
    f32, o32 = lat.field(G.EVEN, G.FLOAT, host=e32), lat.field(G.EVEN, G.FLOAT)
    lat.g5Cphi_eopre_flt(m, o32, f32)
    got = lat.apply_op_host(G.OP_G5CPHI_EOPRE, m, e32, prec=G.FLOAT)
    assert np.array_equal(got, o32.download())


def test_apply_op_host_matches_oracle_and_counts():
    o, u, lat = make((8, 4, 4, 4), 3, O.FUND, clover=False)
    o.set_gauge(o.represent_gauge_field(u, True))
    m = 0.1
    e = F.gaussian_spinor(9, lat.VH, lat.nf)
    lat.getMVM()
    got = lat.apply_op_host(G.OP_DPHI_EOPRE, m, e)
    assert lat.getMVM() == 1  # one even-odd application (two hops), as Dphi_eopre counts it
    assert rel(got, o.Dphi_eopre(m, e)) < 1e-13


def test_apply_op_host_refuses_other_ops_and_missing_clover():
    o, u, lat = make((4, 4, 4, 4), 2, O.FUND, clover=False)
    e = F.gaussian_spinor(1, lat.VH, lat.nf)
    with pytest.raises(G.HRGPUError, match="not an even-odd"):
        lat.apply_op_host(G.OP_G5DPHI_EOPRE_SQ, 0.1, e)
    with pytest.raises(G.HRGPUError, match="no clover term"):
        lat.apply_op_host(G.OP_CPHI_EOPRE, 0.1, e)
    with pytest.raises(G.HRGPUError, match="chunks"):
        lat.set_host_chunks(0)


def test_apply_op_host_graph_path_with_pinned_buffers():
    """Pinned host buffers take the captured-graph path: repeated calls, new input
    data, a new gauge field and a new mass all give the eager result."""
    import torch

    o, u, lat = make((8, 4, 4, 4), 3, O.FUND)
    lat.set_host_chunks(4)
    n = lat.VH * 4 * lat.nf
    t_in = torch.empty(2 * n, dtype=torch.float64).pin_memory()
    t_out = torch.empty(2 * n, dtype=torch.float64).pin_memory()
    h_in = t_in.numpy().view(np.complex128).reshape(lat.VH, 4, lat.nf)
    h_out = t_out.numpy().view(np.complex128).reshape(lat.VH, 4, lat.nf)
    fin, fout = lat.field(G.EVEN), lat.field(G.EVEN)
    # before any whole-lattice launch the kernel variants are not tuned: the
    # pipelined call then runs eagerly (zero-copy, default variant, no graph)
    h_in[...] = F.gaussian_spinor(11, lat.VH, lat.nf)
    first = lat.apply_op_host(G.OP_CPHI_EOPRE, -0.2, h_in, out=h_out).copy()
    fin.upload(h_in.copy())
    lat.Cphi_eopre(-0.2, fout, fin)
    assert rel(first, fout.download()) < 1e-14

    def check(m, seed):
        h_in[...] = F.gaussian_spinor(seed, lat.VH, lat.nf)
        fin.upload(h_in.copy())
        lat.Cphi_eopre(m, fout, fin)
        got = lat.apply_op_host(G.OP_CPHI_EOPRE, m, h_in, out=h_out)
        assert got is h_out
        assert np.array_equal(h_out, fout.download())

    check(-0.2, 1)
    check(-0.2, 2)  # cached graph, new data
    u2 = F.smooth_gauge(8, lat.V, 3, 0.3)
    lat.set_gauge(u2)
    lat.represent_gauge_field(True)  # rebuilds the clover term
    check(-0.2, 3)
    check(-0.1, 4)  # a new mass: a new graph


@pytest.mark.parametrize("form", [0, 1, 2])
def test_apply_op_host_forms_are_bit_identical(form):
    """Form 0 times the pipelined form against the plain sequence when it makes a
    graph, alternates them over its first 32 calls and again after every 1024,
    and keeps the faster; 1 and 2 pin one.  Every form gives the device
    operator's field bit for bit, through the rounds of trials too, and the
    choice is reported."""
    import torch

    o, u, lat = make((8, 4, 4, 4), 3, O.FUND)
    G._check(lat.L.hrgpu_set_host_form(form), "set_host_form")
    try:
        n = lat.VH * 4 * lat.nf
        t_in = torch.empty(2 * n, dtype=torch.float64).pin_memory()
        t_out = torch.empty(2 * n, dtype=torch.float64).pin_memory()
        h_in = t_in.numpy().view(np.complex128).reshape(lat.VH, 4, lat.nf)
        h_out = t_out.numpy().view(np.complex128).reshape(lat.VH, 4, lat.nf)
        h_in[...] = F.gaussian_spinor(21, lat.VH, lat.nf)
        fin, fout = lat.field(G.EVEN, host=h_in.copy()), lat.field(G.EVEN)
        lat.Cphi_eopre(-0.2, fout, fin)  # settles the kernel variants: the graph path
        ref = fout.download()
        for k in range(34 + (1024 + 34 if form == 0 else 0)):
            # form 0: calls 1-32 alternate the two forms, then the kept one runs;
            # after 1024 more calls 32 calls alternate them again
            h_out[...] = 0
            lat.apply_op_host(G.OP_CPHI_EOPRE, -0.2, h_in, out=h_out)
            if k < 34 or k >= 1024 + 30:
                assert np.array_equal(h_out, ref)
        chosen, ms_p, ms_s = G.ctypes.c_int(), G.ctypes.c_float(), G.ctypes.c_float()
        G._check(lat.L.hrgpu_host_form(G.ctypes.byref(chosen), G.ctypes.byref(ms_p), G.ctypes.byref(ms_s)), "form")
        if form == 0:
            assert chosen.value in (1, 2) and ms_p.value > 0 and ms_s.value > 0
            assert chosen.value == (2 if ms_s.value < ms_p.value else 1)
        else:
            assert chosen.value == form
    finally:
        G._check(lat.L.hrgpu_set_host_form(0), "set_host_form")
    with pytest.raises(G.HRGPUError, match="set_host_form"):
        G._check(lat.L.hrgpu_set_host_form(3), "set_host_form")
