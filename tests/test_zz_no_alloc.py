"""The allocation-free even-odd operator entry point (hrgpu_Dphi_eopre_noalloc).

Some callers cannot let the library cudaMalloc its temporaries, because a host
framework owns the GPU's memory through its own pool.  For them the library
offers hrgpu_Dphi_eopre_noalloc, which keeps the odd-parity temporary in a
static device array of 32 MiB.  This test calls it through the C ABI and checks
it against hrgpu_Dphi_eopre on two calls in a row (the array keeps the previous
call's contents, which must not matter); that its first call on a fresh lattice,
made before any allocating operator, leaves the device's free memory unchanged
and agrees with hrgpu_Dphi_eopre called afterwards; and that a lattice too
large for the array is refused with a clear error.  It sits in a file of its
own, collected last.
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
    return np.abs(a - b).max() / np.abs(b).max()


def _entry():
    lib = G.lib()
    fn = lib.hrgpu_Dphi_eopre_noalloc
    fn.argtypes = [ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return lib, fn


def test_noalloc_eopre_matches_allocating_entry_point():
    dims = (8, 8, 8, 16)
    o = O.Oracle(*dims, 3, O.FUND)
    ipt, _, _ = o.geometry()
    lat = G.Lattice(*dims, 3, G.FUND, ipt=ipt)
    lat.set_gauge(F.smooth_gauge(3, o.V, 3, 0.3))
    lat.represent_gauge_field(True)
    lib, fn = _entry()
    for call, (seed, m) in enumerate([(1, 0.1), (2, -0.35)]):
        src = F.gaussian_spinor(seed, o.VH, o.nf)
        fin, ref, out = lat.field(G.EVEN, host=src), lat.field(G.EVEN), lat.field(G.EVEN)
        lat.Dphi_eopre(m, ref, fin)
        rc = fn(m, out.ptr, fin.ptr)
        assert rc == 0, lib.hrgpu_last_error().decode()
        assert rel(out.download(), ref.download()) < TOL64, f"call {call}"


def test_noalloc_first_call_on_a_fresh_lattice_allocates_nothing():
    """The first call in a process loads the library's module for the entry
    point (which reserves the static array) and looks up its address: that
    happens on a small lattice first.  Then, on a fresh lattice whose fields are
    already allocated, the entry point's first call (it also times the
    hopping-kernel variants) must leave the device's free memory where it was;
    an allocating operator would need a 6.3 MB odd temporary here."""
    import torch

    lib, fn = _entry()
    warm = G.Lattice(4, 4, 4, 4, 3, G.FUND)
    warm.set_gauge(F.smooth_gauge(5, warm.V, 3, 0.3))
    warm.represent_gauge_field(True)
    wi, wo = warm.field(G.EVEN, host=F.gaussian_spinor(5, warm.VH, 3)), warm.field(G.EVEN)
    assert fn(0.1, wo.ptr, wi.ptr) == 0, lib.hrgpu_last_error().decode()

    dims, m = (16, 16, 16, 16), -0.2
    lat = G.Lattice(*dims, 3, G.FUND)
    lat.set_gauge(F.smooth_gauge(6, lat.V, 3, 0.3))
    lat.represent_gauge_field(True)
    src = F.gaussian_spinor(6, lat.VH, lat.nf)
    fin, out, ref = lat.field(G.EVEN, host=src), lat.field(G.EVEN), lat.field(G.EVEN)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    rc = fn(m, out.ptr, fin.ptr)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert rc == 0, lib.hrgpu_last_error().decode()
    assert abs(free1 - free0) < (1 << 20), (free0, free1)
    lat.Dphi_eopre(m, ref, fin)  # the allocating entry point, afterwards
    assert rel(out.download(), ref.download()) < TOL64


def test_noalloc_rejects_lattice_beyond_scratch():
    dims = (32, 24, 24, 24)  # odd FP64 field of 42 MB > 32 MiB
    ipt, _, _ = G.geometry(*dims)
    lat = G.Lattice(*dims, 3, G.FUND, ipt=ipt)
    lib, fn = _entry()
    fin, out = lat.field(G.EVEN), lat.field(G.EVEN)
    rc = fn(0.1, out.ptr, fin.ptr)
    assert rc == 2  # HRGPU_E_ARG
    assert b"static scratch" in lib.hrgpu_last_error()
