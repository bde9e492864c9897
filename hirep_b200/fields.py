"""Seeded synthetic inputs in HiRep's host layout.

The workloads are synthetic by design (HiRep publishes no dataset for this path):
  * hot start: every link an independent Haar-random SU(N) matrix;
  * smooth links U = exp(i * eps * H), H a Gaussian traceless Hermitian NG x NG
    matrix per link;
  * Gaussian spinors with unit variance per real component.

Layouts: fundamental links complex128 [V, 4, NG, NG] indexed by HiRep's site
index ix and direction mu (Include/field_ordering.h:10); spinors complex128
[nsites, 4, NF].
"""
import numpy as np


def haar_su_n(rng, count, n):
    """`count` Haar-random SU(n) matrices (QR of a complex Gaussian, phase fixed)."""
    z = (rng.standard_normal((count, n, n)) + 1j * rng.standard_normal((count, n, n))) / np.sqrt(2.0)
    q, r = np.linalg.qr(z)
    d = np.diagonal(r, axis1=1, axis2=2)
    q = q * (d / np.abs(d))[:, None, :]
    det = np.linalg.det(q)
    return q / (det ** (1.0 / n))[:, None, None]


def exp_i_hermitian(h):
    """exp(i h) for a stack of Hermitian matrices, by eigendecomposition (2x2
    traceless: cos|a| + i sin|a| h/|a|, |a|^2 = -det h)."""
    if h.shape[-1] == 2 and np.allclose(h[..., 0, 0] + h[..., 1, 1], 0.0, atol=1e-14):
        a = np.sqrt(np.maximum(-np.linalg.det(h).real, 0.0))[..., None, None]
        sinc = np.where(a > 0, np.sin(a) / np.where(a > 0, a, 1.0), 1.0)
        return np.cos(a) * np.eye(2) + 1j * sinc * h
    w, v = np.linalg.eigh(h)
    return np.einsum("...ij,...j,...kj->...ik", v, np.exp(1j * w), v.conj())


def gaussian_traceless_hermitian(rng, count, n):
    """H = sum_A h_A T_A with h_A ~ N(0,1) and Tr T_A T_B = delta_AB/2.

    For SU(3) and eps = 0.3 this gives an average plaquette of about 0.79."""
    a = rng.standard_normal((count, n, n)) + 1j * rng.standard_normal((count, n, n))
    h = (0.5 / np.sqrt(2.0)) * (a + np.conj(np.swapaxes(a, 1, 2)))
    tr = np.trace(h, axis1=1, axis2=2).real / n
    h -= tr[:, None, None] * np.eye(n)
    return h


def hot_gauge(seed, volume, ng):
    rng = np.random.default_rng(seed)
    return haar_su_n(rng, 4 * volume, ng).reshape(volume, 4, ng, ng)


def smooth_gauge(seed, volume, ng, eps):
    rng = np.random.default_rng(seed)
    out = np.empty((volume, 4, ng, ng), np.complex128)
    flat = out.reshape(4 * volume, ng, ng)
    chunk = 1 << 18
    for s in range(0, 4 * volume, chunk):
        e = min(4 * volume, s + chunk)
        flat[s:e] = exp_i_hermitian(eps * gaussian_traceless_hermitian(rng, e - s, ng))
    return out


def gaussian_spinor(seed, nsites, nf, dtype=np.complex128):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((nsites, 4, nf)) + 1j * rng.standard_normal((nsites, 4, nf))
    return a.astype(dtype)


def nf_of(ng, repr_name):
    return {"FUND": ng, "ADJ": ng * ng - 1, "SYM": ng * (ng + 1) // 2, "ASYM": ng * (ng - 1) // 2}[repr_name]


def point_source(nsites, nf, spin, col, site=0, dtype=np.complex128):
    """One spin-colour point source: 1 at component (spin, col) of one site, in
    HiRep's site order (site 0 = the origin, an even site).  HiRep's
    create_full_point_source (LibHR/Observables/sources.c:114-140) fills source
    index spin + 4*col this way at timeslice tau."""
    a = np.zeros((nsites, 4, nf), dtype)
    a[site, spin, col] = 1.0
    return a
