"""The reference's linear-algebra consistency checks (TestProgram/SpinorField/
check_spinorfield_1.c) restated on the device BLAS: prod against an explicit
sum, prod_re and sqnorm; |k + z l|^2 from prod and sqnorm after
mulc_add_assign; project + normalize; a 5-field rotation built from mulc and
mulc_add_assign undone again; g5 twice is the identity and preserves prod.
Every check has the reference's bound, 1e-14."""
import numpy as np
import pytest

from hirep_b200 import fields as F
from hirep_b200 import hrgpu as G

pytestmark = pytest.mark.gpu
EPS = 1e-14


@pytest.fixture(scope="module")
def lat():
    lat = G.Lattice(8, 8, 8, 8, 3, G.FUND)
    lat.set_gauge(F.smooth_gauge(1, lat.V, 3, 0.3))
    lat.represent_gauge_field(True)
    return lat


def fields(lat, n, seed):
    hs = [F.gaussian_spinor(seed + i, lat.V, lat.nf) for i in range(n)]
    return hs, [lat.field(G.FULL, host=h) for h in hs]


def test_prod_prod_re_sqnorm(lat):
    hs, ws = fields(lat, 10, 100)
    dmax = 0.0
    for i in range(10):
        k, l = ws[i], ws[9 - i]
        w = np.vdot(hs[i], hs[9 - i])  # the explicit sum over sites and components
        zd = lat.prod(k, l)
        rd = lat.sqnorm(k) * lat.sqnorm(l)
        dmax = max(dmax, abs(zd - w) / np.sqrt(rd))
        dmax = max(dmax, abs(zd.real / lat.prod_re(k, l) - 1.0))
        zd = lat.prod(k, k)
        rd = lat.sqnorm(k)
        dmax = max(dmax, abs(zd.imag / rd), abs(zd.real / rd - 1.0))
    assert dmax < EPS, dmax


def test_mulc_add_assign_norm(lat):
    _, ws = fields(lat, 10, 200)
    zd = 0.345 - 0.876j
    zsq = abs(zd) ** 2
    dmax = 0.0
    for i in range(9):
        k, l = ws[i], ws[i + 1]
        wd = lat.prod(k, l)
        rd = lat.sqnorm(k) + zsq * lat.sqnorm(l) + 2.0 * (zd * wd).real
        lat.la("mulc_add_assign", k, zd, l)
        dmax = max(dmax, abs(rd / lat.sqnorm(k) - 1.0))
    assert dmax < EPS, dmax


def test_project_and_normalize(lat):
    _, ws = fields(lat, 10, 300)
    dmax = 0.0
    for i in range(10):
        k = ws[i]
        if i > 0:
            l = ws[i - 1]
            lat.la("mulc_add_assign", k, -lat.prod(l, k), l)  # project out l
            zd = lat.prod(k, l)
            dmax = max(dmax, (abs(zd.real) + abs(zd.imag)) / np.sqrt(lat.sqnorm(k)))
        lat.la("mul", k, 1.0 / np.sqrt(lat.sqnorm(k)), k)
        dmax = max(dmax, abs(lat.sqnorm(k) - 1.0))
    assert dmax < EPS, dmax


def test_rotate_and_undo(lat):
    hs, ws = fields(lat, 5, 400)
    copies = [lat.field(G.FULL, host=h) for h in hs]
    v = np.empty(25, complex)
    for i in range(5):
        for j in range(5):
            v[5 * i + j] = (float(np.float32(0.1234)) * (i ^ 2) - float(np.float32(0.8976)) * j
                            + 1j * (float(np.float32(0.2231)) * i + float(np.float32(0.9922)) * (j ^ 2)))
    # rotate: new_k = sum_j v[k + 5 j] p_j (the reference's rotate_ptr)
    rot = [lat.field(G.FULL) for _ in range(5)]
    for k in range(5):
        lat.la("mulc", rot[k], complex(v[k]), copies[0])
        for j in range(1, 5):
            lat.la("mulc_add_assign", rot[k], complex(v[k + 5 * j]), copies[j])
    dmax = 0.0
    for k in range(5):
        for j in range(5):
            lat.la("mulc_add_assign", rot[k], complex(-v[5 * j + k]), ws[j])
        dmax = max(dmax, abs(lat.sqnorm(rot[k])))
    dmax = np.sqrt(dmax / lat.sqnorm(ws[0]))
    assert dmax < EPS, dmax


def test_g5(lat):
    _, ws = fields(lat, 10, 500)
    tmp = lat.field(G.FULL)
    dmax = 0.0
    for i in range(5):
        k, l = ws[i], ws[9 - i]
        lat.la("copy", l, k)
        lat.la("g5", tmp, k)
        lat.la("g5", k, tmp)
        lat.la("mulc_add_assign", l, -1.0 + 0j, k)
        dmax = max(dmax, np.sqrt(lat.sqnorm(l) / lat.sqnorm(k)))
        l.upload(F.gaussian_spinor(600 + i, lat.V, lat.nf))
        zd = lat.prod(k, l)
        lat.la("g5", tmp, k)
        lat.la("copy", k, tmp)
        lat.la("g5", tmp, l)
        lat.la("copy", l, tmp)
        wd = lat.prod(k, l)
        dmax = max(dmax, (abs((zd - wd).real) + abs((zd - wd).imag)) / (abs(zd.real) + abs(zd.imag)))
    assert dmax < EPS, dmax
