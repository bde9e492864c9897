"""CPU-side checks of the C-ABI library: it loads, exports every symbol the
headers declare, and its host-side geometry equals HiRep's serial walk (the
oracle's restatement of LibHR/Geometry/geometry_mpi_eo.c) bit for bit."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle as O
from hirep_b200 import hrgpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[a-z_ ]+\**\s*\**(hrgpu_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = hrgpu.lib()
    names = declared_symbols()
    assert len(names) > 80
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []


@pytest.mark.parametrize("dims", [(8, 8, 8, 8), (4, 6, 2, 8), (16, 4, 4, 8), (2, 2, 2, 2)])
def test_geometry_bit_exact(dims):
    ipt, iup, idn = hrgpu.geometry(*dims)
    o = O.Oracle(*dims, 3, O.FUND)
    oi, ou, od = o.geometry()
    assert np.array_equal(ipt, oi)
    assert np.array_equal(iup, ou)
    assert np.array_equal(idn, od)


def test_errors_are_reported_not_fatal():
    lib = hrgpu.lib()
    rc = lib.hrgpu_geometry(0, 4, 4, 4, None, None, None)
    assert rc == 2
    assert b"bad arguments" in lib.hrgpu_last_error()


@pytest.mark.parametrize("setter,good,bad,default", [
    ("hrgpu_set_hop_variant", [-1, 0, 6], [-2, 7], -1),
    ("hrgpu_set_batch_variant", [-1, 0, 5], [-2, 6], -1),
    ("hrgpu_set_force_variant", [0, 5, 6], [-1, 7], 0),
    ("hrgpu_set_host_form", [0, 1, 2], [-1, 3], 0),
    ("hrgpu_set_host_chunks", [1, 10], [0, -3], 10),
])
def test_tuning_controls_check_their_arguments(setter, good, bad, default):
    """The tuning controls are host state: each accepts its documented range and
    refuses anything else with HRGPU_E_ARG (2) and a message naming the call,
    without a GPU."""
    lib = hrgpu.lib()
    fn = getattr(lib, setter)
    try:
        for v in good:
            assert fn(v) == 0
        for v in bad:
            assert fn(v) == 2
            assert setter[len("hrgpu_"):].encode() in lib.hrgpu_last_error()
    finally:
        assert fn(default) == 0
