"""HiRep's own check programs run through the drop-in binding.

TestProgram/DiracOperator/check_diracoperator_{1,3,6}.c and
TestProgram/Inverters/check_inverters_{1,6}.c, compiled from the reference
sources and linked (oracle/ref/one.mk, target shim) against HiRep's library
with every hot-path function redirected by the linker's --wrap to
hirep_b200/shim/hrgpu_hirep.c, which forwards it to libhrgpu.so.  The programs
are unchanged: they draw their fields with HiRep's ranlux, call Dphi, the
even-odd operators, their FP32 forms and cg_mshift / cg_mshift_flt through
HiRep's API, and check gauge covariance (< 1e-14), hermiticity (< 1e-14),
FP32 against FP64 and the solvers' true residuals with HiRep's own
tolerances; their exit status is the number of failed checks.  The binaries
are built where the reference sources are; they run here without them.

Each program runs for the three builds of the binding (SU(3) fundamental,
SU(4) two-index antisymmetric, SU(2) adjoint) on its own input's lattice.
"""
import os
import subprocess
import tempfile

import pytest

import hirep_ref as H

pytestmark = pytest.mark.gpu

# program -> (lattice T, X, Y, Z, ranlux seed), as in the program's .in file (serial: NP = 1)
PROGRAMS = {
    "check_diracoperator_1": ((6, 4, 4, 4), 12345),
    "check_diracoperator_3": ((6, 4, 4, 4), 12345),
    "check_diracoperator_6": ((6, 4, 4, 4), 12345),
    "check_inverters_1": ((8, 8, 4, 4), 13813),
    "check_inverters_6": ((8, 8, 4, 4), 13813),
}
BUILDS = ["su3_fund", "su4_asym", "su2_adj"]


def run_program(cfg, prog):
    exe = os.path.join(H.REF_DIR, cfg, "shim", prog)
    if not os.access(exe, os.X_OK):
        pytest.skip(f"{exe} not built (make -C oracle/ref with the reference sources)")
    (T, X, Y, Z), seed = PROGRAMS[prog]
    with tempfile.TemporaryDirectory(prefix="hrgpu_dropin_") as d:
        with open(os.path.join(d, "input_file"), "w") as f:
            f.write(f"GLB_T = {T}\nGLB_X = {X}\nGLB_Y = {Y}\nGLB_Z = {Z}\nNP_T = 1\nNP_X = 1\nNP_Y = 1\nNP_Z = 1\n"
                    f"N_REP = 1\nlog:default = -1\nlog:inverter = -1\nrlx_level = 1\nrlx_seed = {seed}\n"
                    "rlx_start = new\nrlx_state = rand_state\n")
        env = dict(os.environ, OMP_NUM_THREADS="4")
        p = subprocess.run([exe, "-i", "input_file"], cwd=d, env=env, capture_output=True, text=True, timeout=600)
        log = ""
        for name in ("out_0", "err_0"):
            path = os.path.join(d, name)
            if os.path.exists(path):
                log += open(path).read()
    return p.returncode, log


@pytest.mark.parametrize("cfg", BUILDS)
@pytest.mark.parametrize("prog", list(PROGRAMS))
def test_hirep_check_program_through_the_dropin(cfg, prog):
    rc, log = run_program(cfg, prog)
    assert rc == 0, f"{prog} ({cfg}) exit {rc}:\n{log[-3000:]}"
    assert "FAILED" not in log
    assert "hot path on the GPU (libhrgpu)" in log  # the binding ran, not HiRep's own operators
