"""The allocation-free even-odd operator entry point (hrgpu_Dphi_eopre_noalloc).

Some callers cannot let the library cudaMalloc its temporaries, because a host
framework owns the GPU's memory through its own pool.  For them the library
offers hrgpu_Dphi_eopre_noalloc, which keeps the odd-parity temporary in a
static device array of 32 MiB.  This test calls it through the C ABI and checks
it against hrgpu_Dphi_eopre on two calls in a row (the array keeps the previous
call's contents, which must not matter), and that a lattice too large for the
array is refused with a clear error.  It sits in a file of its own, collected
last.
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


def test_noalloc_rejects_lattice_beyond_scratch():
    dims = (32, 24, 24, 24)  # odd FP64 field of 42 MB > 32 MiB
    ipt, _, _ = G.geometry(*dims)
    lat = G.Lattice(*dims, 3, G.FUND, ipt=ipt)
    lib, fn = _entry()
    fin, out = lat.field(G.EVEN), lat.field(G.EVEN)
    rc = fn(0.1, out.ptr, fin.ptr)
    assert rc == 2  # HRGPU_E_ARG
    assert b"static scratch" in lib.hrgpu_last_error()
