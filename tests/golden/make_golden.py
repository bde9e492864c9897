"""Writes the golden fixtures of this folder from HiRep itself.

Run from the repository root after ``make -C oracle/ref`` (which builds the
reference's own library from its sources into oracle/_ref/):

    python tests/golden/make_golden.py

Each fixture hirep_<config>.npz holds HiRep's outputs for seeded inputs that
the tests regenerate with hirep_b200.fields (numpy PCG64 streams):
  links     smooth_gauge(7, V, NG, 0.3), read as read_gauge_field does
  source    gaussian_spinor(1, V/2, NF)             (even)
  X, Y      gaussian_spinor(11 / 12, V, NF)          (full lattice)
and records: the represented links of the first two sites, the even-odd
operator (Dphi_eopre, or Cphi_eopre with csw 1.0 in clover builds) at
m0 = -0.1, the multi-shift CG solution of its H^2 to err2 1e-28 with its MVM
count, in clover builds the clover term of the first two sites and the squared
norm of all of it, and the force (force_fermion_core + fermion_force_end,
dt 0.37, residue 1.3).  The geometry fixture holds ipt/iup/idn of a 4x6x2x8
lattice; config1.npz holds the average plaquette of HiRep's hot start
(random_u after rlxd_init(1, 1234), 8^4) drawn by one OpenMP thread: ranlxd
keeps one stream per thread (LibHR/Random/ranlxd.c:459-470) and random_u draws
inside a parallel site loop, so the field depends on the thread count.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import hirep_ref as H  # noqa: E402
from hirep_b200 import fields as F  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
DIMS = (4, 4, 4, 4)
MASS, CSW, DT, RES = -0.1, 1.0, 0.37, 1.3
SHIFTS = [0.1]
FIXTURES = ["su3_fund", "su3_fund_clover", "su4_asym", "su2_adj", "su3_sym_clover"]


def make(cfg):
    ng, rep, clover = H.CONFIGS[cfg]
    with H.HiRep(cfg, *DIMS, threads=1) as h:
        u = F.smooth_gauge(7, h.V, ng, 0.3)
        h.set_gauge(u)
        op = "Dphi_eopre"
        if clover:
            h.set_csw(CSW)
            op = "Cphi_eopre"
        e = F.gaussian_spinor(1, h.VH, h.nf)
        X = F.gaussian_spinor(11, h.V, h.nf)
        Y = F.gaussian_spinor(12, h.V, h.nf)
        out = {
            "gauge_f_head": h.gauge_f()[:2],
            "eopre": h.apply(op, MASS, e, H.EVEN, H.EVEN),
            "force": h.force(MASS, DT, RES, X, Y, True),
        }
        sq = "g5Cphi_eopre_sq" if clover else "g5Dphi_eopre_sq"
        x, mvm = h.cg_mshift(sq, MASS, SHIFTS, 1e-28, e, H.EVEN, max_iter=5000)
        out["cg"], out["cg_mvm"] = x, np.int64(mvm)
        if clover:
            cl = h.clover_term()
            out["cl_term_head"], out["cl_term_sqnorm"] = cl[:2], np.float64((np.abs(cl) ** 2).sum())
    np.savez_compressed(os.path.join(HERE, f"hirep_{cfg}.npz"), **out)


def main():
    for cfg in FIXTURES:
        make(cfg)
    with H.HiRep("su3_fund", 4, 6, 2, 8) as h:
        ipt, iup, idn = h.geometry()
    np.savez_compressed(os.path.join(HERE, "hirep_geometry_4x6x2x8.npz"), ipt=ipt, iup=iup, idn=idn)
    with H.HiRep("su3_fund", 8, 8, 8, 8, seed=1234, threads=1) as h:
        h.random_u()
        plaq = h.plaquette()
    np.savez_compressed(os.path.join(HERE, "hirep_config1.npz"), plaquette=np.float64(plaq))


if __name__ == "__main__":
    main()
