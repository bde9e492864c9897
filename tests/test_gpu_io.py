"""Gauge configuration files in HiRep's format (LibHR/IO/archive.c,
archive_su2quat.c), decoded here independently with numpy: big-endian header
(NG, T, X, Y, Z, plaquette) and links in (t, x, y, z) order, SU(2) as
quaternions."""
import numpy as np
import pytest

import oracle as O
from hirep_b200 import fields as F
from hirep_b200 import hrgpu as G

pytestmark = pytest.mark.gpu
DIMS = (4, 4, 4, 6)  # T, X, Y, Z: all different orders would show


def _lattice(ng, seed=3):
    o = O.Oracle(*DIMS, ng, O.FUND)
    ipt = o.geometry()[0]
    u = F.smooth_gauge(seed, o.V, ng, 0.4)
    lat = G.Lattice(*DIMS, ng, G.FUND, ipt=ipt)
    lat.set_gauge(u)
    lat.represent_gauge_field(True)
    return o, lat, u, ipt


def _decode(path, ng):
    raw = open(path, "rb").read()
    hdr = np.frombuffer(raw[:20], ">i4")
    plaq = np.frombuffer(raw[20:28], ">f8")[0]
    body = np.frombuffer(raw[28:], ">f8")
    return hdr, plaq, body


def test_write_then_decode_su3(tmp_path):
    o, lat, u, ipt = _lattice(3)
    f = tmp_path / "conf_su3"
    lat.write_gauge_field(f)
    hdr, plaq, body = _decode(f, 3)
    assert list(hdr) == [3, *DIMS]
    assert plaq == pytest.approx(o.avr_plaquette(u), rel=1e-14)
    m = body.reshape(-1, 4, 3, 3, 2)
    links = m[..., 0] + 1j * m[..., 1]
    assert np.array_equal(links, u[ipt])  # file site ((t*X+x)*Y+y)*Z+z = HiRep ipt order
    # and back into a new lattice
    lat2 = G.Lattice(*DIMS, 3, G.FUND, ipt=ipt)
    pf, pr = lat2.read_gauge_field(f)
    assert pf == plaq and abs(pr - pf) < 1e-14
    assert np.array_equal(lat2.gauge_get(), u)


def test_su2_quaternions_both_ways(tmp_path):
    o, lat, u, ipt = _lattice(2, seed=5)
    f = tmp_path / "conf_su2"
    lat.write_gauge_field(f)
    hdr, plaq, body = _decode(f, 2)
    q = body.reshape(-1, 4, 4)
    m = np.empty(q.shape[:2] + (2, 2), complex)
    m[..., 0, 0] = q[..., 0] + 1j * q[..., 3]
    m[..., 0, 1] = -q[..., 2] + 1j * q[..., 1]
    m[..., 1, 0] = q[..., 2] + 1j * q[..., 1]
    m[..., 1, 1] = q[..., 0] - 1j * q[..., 3]
    assert np.abs(m - u[ipt]).max() < 1e-15
    lat2 = G.Lattice(*DIMS, 2, G.FUND, ipt=ipt)
    lat2.read_gauge_field(f)
    assert np.abs(lat2.gauge_get() - u).max() < 1e-15
    # an SU(2) file in matrix form is recognised and read exactly
    g = tmp_path / "conf_su2_matrix"
    with open(g, "wb") as fh:
        fh.write(np.array([2, *DIMS], ">i4").tobytes())
        fh.write(np.array([plaq], ">f8").tobytes())
        fh.write(np.stack([u[ipt].real, u[ipt].imag], axis=-1).astype(">f8").tobytes())
    lat3 = G.Lattice(*DIMS, 2, G.FUND, ipt=ipt)
    lat3.read_gauge_field(g)
    assert np.array_equal(lat3.gauge_get(), u)


def test_read_refuses_mismatches(tmp_path):
    o, lat, u, ipt = _lattice(3)
    f = tmp_path / "conf"
    lat.write_gauge_field(f)
    other = G.Lattice(4, 4, 4, 4, 3, G.FUND)
    with pytest.raises(G.HRGPUError, match="lattice is NG=3 4x4x4x4"):
        other.read_gauge_field(f)
    short = tmp_path / "short"
    short.write_bytes(open(f, "rb").read()[:1000])
    lat2 = G.Lattice(*DIMS, 3, G.FUND, ipt=ipt)
    with pytest.raises(G.HRGPUError, match="bytes"):
        lat2.read_gauge_field(short)
    with pytest.raises(G.HRGPUError, match="cannot open"):
        lat2.read_gauge_field(tmp_path / "missing")
