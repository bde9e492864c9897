"""Random draws on the device (hrgpu_random_seed, hrgpu_gaussian_momenta,
hrgpu_gaussian_spinor_field; HiRep's rlxd_init, gaussian_momenta in
LibHR/Update/random_momenta.c:18-38 and gaussian_spinor_field in
LibHR/Update/random_spinor_field.c:14-36).  The generator is Philox4x32-10
with Box-Muller Gaussians: the numpy restatement below is pinned to the
published known-answer vectors of Philox4x32-10 (Random123, Salmon et al.,
SC11), and the device field must equal it element by element."""
import numpy as np
import pytest

from hirep_b200 import hrgpu as G

M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Philox4x32-10 on uint64 arrays holding 32-bit words."""
    c0, c1, c2, c3 = (np.asarray(x, np.uint64) & MASK for x in (c0, c1, c2, c3))
    k0, k1 = np.uint64(k0), np.uint64(k1)
    for _ in range(10):
        p0, p1 = np.uint64(M0) * c0, np.uint64(M1) * c2
        c0, c1, c2, c3 = ((p1 >> np.uint64(32)) ^ c1 ^ k0, p1 & MASK, (p0 >> np.uint64(32)) ^ c3 ^ k1, p0 & MASK)
        k0, k1 = (k0 + np.uint64(W0)) & MASK, (k1 + np.uint64(W1)) & MASK
    return c0, c1, c2, c3


def gauss_pairs(q, stream, seed):
    """The two Gaussians of Philox block q of a stream (the device's gauss_pair)."""
    q = np.asarray(q, np.uint64)
    k0, k1 = seed & 0xFFFFFFFF, seed >> 32
    c = philox4x32_10(q & MASK, q >> np.uint64(32), np.full_like(q, stream & 0xFFFFFFFF),
                      np.full_like(q, stream >> 32), k0, k1)
    u1 = (((c[0] << np.uint64(32)) | c[1]) >> np.uint64(11)).astype(np.float64)
    u2 = (((c[2] << np.uint64(32)) | c[3]) >> np.uint64(11)).astype(np.float64)
    u1, u2 = (u1 + 0.5) * 2.0**-53, (u2 + 0.5) * 2.0**-53
    r = np.sqrt(-2.0 * np.log(u1))
    return r * np.cos(2 * np.pi * u2), r * np.sin(2 * np.pi * u2)


def test_philox_known_answers():
    """The published Philox4x32-10 known-answer vectors."""
    kat = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
           ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
           ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
            (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]
    for ctr, key, want in kat:
        got = philox4x32_10(*[np.array([x], np.uint64) for x in ctr], *key)
        assert tuple(int(x[0]) for x in got) == want


def device_layout(f, lat):
    """The raw device buffer of an even field: [4 NF][ld] complex."""
    dt = np.complex128 if f.prec == G.DOUBLE else np.complex64
    a = f.buf.cpu().numpy().view(dt)
    return a.reshape(4 * lat.nf, -1)


@pytest.fixture(scope="module")
def lat():
    lat = G.Lattice(6, 6, 2, 2, 3, G.FUND)  # VH = 72: 24 padding sites per plane (ld = 96)
    return lat


@pytest.mark.gpu
def test_spinor_draw_matches_the_restatement(lat):
    seed = 0x0123456789ABCDEF
    lat.random_seed(seed)
    f = lat.gaussian_spinor_field(lat.field(G.EVEN))
    dev = device_layout(f, lat)
    ncomp, ld = dev.shape
    assert ld > lat.VH
    e = np.arange(ncomp * ld, dtype=np.uint64)
    z0, z1 = gauss_pairs(e, 0, seed)
    want = ((z0 + 1j * z1) / np.sqrt(2)).reshape(ncomp, ld)
    want[:, lat.VH:] = 0.0
    assert np.abs(dev - want).max() < 1e-12
    assert np.all(dev[:, lat.VH:] == 0)


@pytest.mark.gpu
def test_draws_reproduce_and_advance(lat):
    lat.random_seed(11)
    a = lat.gaussian_spinor_field(lat.field(G.FULL)).download()
    b = lat.gaussian_spinor_field(lat.field(G.FULL)).download()
    lat.random_seed(11)
    a2 = lat.gaussian_spinor_field(lat.field(G.FULL)).download()
    assert np.array_equal(a, a2)  # a seed replays its draws
    assert np.abs(a - b).max() > 1.0  # the next draw is another one
    lat.random_seed(11)
    d = lat.gaussian_spinor_field(lat.field(G.EVEN))
    lat.random_seed(11)
    s = lat.gaussian_spinor_field(lat.field(G.EVEN, G.FLOAT))
    assert np.array_equal(s.download(), d.download().astype(np.complex64))  # FP32: the FP64 draw rounded


@pytest.mark.gpu
def test_gaussian_statistics():
    """Per real component: N(0, 1/2) for spinors (gaussian_spinor_field),
    N(0, 1/C(fund)) = N(0, 2) for the momenta (gaussian_momenta); means,
    variances within 5 sigma, and a Kolmogorov-Smirnov test."""
    from scipy import stats

    lat = G.Lattice(8, 8, 8, 8, 2, G.ADJ)
    lat.random_seed(2024)
    x = lat.gaussian_spinor_field(lat.field(G.FULL)).download().ravel()
    v = np.concatenate([x.real, x.imag])
    n = v.size
    assert abs(v.mean()) < 5 * np.sqrt(0.5 / n)
    assert abs(v.var() - 0.5) < 5 * 0.5 * np.sqrt(2.0 / n)
    assert stats.kstest(v / np.sqrt(0.5), "norm").pvalue > 1e-3
    lat.gaussian_momenta()
    m = lat.momenta_get().ravel()
    n = m.size
    assert abs(m.mean()) < 5 * np.sqrt(2.0 / n)
    assert abs(m.var() - 2.0) < 5 * 2.0 * np.sqrt(2.0 / n)
    assert stats.kstest(m / np.sqrt(2.0), "norm").pvalue > 1e-3


@pytest.mark.gpu
def test_hmc_with_device_draws():
    """A trajectory whose momenta and pseudofermion source are drawn on the
    device: the same seed gives the same draws, so O2MN's dH falls as dt^2
    between 16 and 32 steps, as with host draws."""
    from hirep_b200 import fields as F
    from hirep_b200.hmc import HMC

    dims, ng, beta, mass = (4, 4, 4, 4), 2, 2.25, -1.0
    u0 = F.smooth_gauge(7, 256, ng, 0.3)
    dh = {}
    for n in (16, 32):
        lat = G.Lattice(*dims, ng, G.ADJ)
        lat.set_gauge(u0)
        lat.represent_gauge_field(True)
        hmc = HMC(lat, beta, mass, tau=0.5, nsteps=n, force_err2=1e-26, force_solver="cg", draws="device")
        dh[n] = hmc.trajectory(np.random.default_rng(8), metropolis=False)["dH"]
    assert abs(dh[16]) < 1.0
    assert 3.5 < dh[16] / dh[32] < 4.5, dh
