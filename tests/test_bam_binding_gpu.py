"""The drop-in inside BAM itself: the reference binary with the B200
binding module linked in (oracle/_ref/bam_gpu, built from the reference
sources by oracle/build_ref.py with baum_b200/bam/nrgpu_bam.c) runs the same
parfile as the plain reference binary (oracle/_ref/bam); every evolved
variable after the run agrees within 1e-12 relative.  Two modes:
"callback" replaces BAM's geometry rhs and boundary callbacks (BAM keeps its
RK4, vladd and algcon), "resident" runs the whole RK4 step + algcon on the
GPU at the EVOLVE hook."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, relerr
from oracle import dumpfile

pytestmark = pytest.mark.gpu

BAM = os.path.join(ROOT, "oracle", "_ref", "bam")
BAM_GPU = os.path.join(ROOT, "oracle", "_ref", "bam_gpu")

PAR = """physics = adm bssn punctures nrharness%s
mass1 = 1
mass2 = 0
punctures_solver = none
bssn_initial_lapse = oochi05
bssn_initial_shift = zero
bssn_lapse = 1+log withshift
bssn_shift = gamma0 withGadv withBadv withShiftadv
bssn_shiftdriver = 2.0
bssn_shiftgammacoeff = 0.75
grid = box
nxyz = 24
dxyz = 0.4
order_centered = 4
order_advection = 4
advection_lopsided = 1
order_dissipation = 6
dissipation_factor = 0.1
evolution_method = rk
evolution_method_rk = rk4
dtfac = 0.25
boundary = radiative
iterations = 6
nrharness_dir = .
nrharness_dump = 6
%s
"""


def run(binary, extra_physics, extra):
    work = tempfile.mkdtemp(prefix="bamgpu_")
    try:
        with open(os.path.join(work, "t.par"), "w") as f:
            f.write(PAR % (extra_physics, extra))
        r = subprocess.run([binary, "-nt", "4", "t.par"], cwd=work, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
        return dumpfile.read(os.path.join(work, "state_it6_l0.bin"))["data"], r.stdout
    finally:
        shutil.rmtree(work, ignore_errors=True)


@pytest.fixture(scope="module")
def cpu_state():
    if not (os.path.exists(BAM) and os.path.exists(BAM_GPU)):
        pytest.skip("the reference binaries are built by oracle/build_ref.py where the reference sources exist")
    return run(BAM, "", "")[0]


@pytest.mark.parametrize("mode,extra", [("callback", "nrgpu_mode = callback"),
                                        ("resident", "nrgpu_mode = resident\nbssn_register_algcon = no")])
def test_bam_with_the_gpu_path_matches_bam(gpu, cpu_state, mode, extra):
    u, out = run(BAM_GPU, " nrgpu", extra)
    assert "nrgpu: %s mode" % mode in out
    assert relerr(u, cpu_state).max() < 1e-12
