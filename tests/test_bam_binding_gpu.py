"""The drop-in inside BAM itself: the reference binary with the B200
binding module linked in (oracle/_ref/bam_gpu, built from the reference
sources by oracle/build_ref.py with baum_b200/bam/nrgpu_bam.c) runs the same
parfile as the plain reference binary (oracle/_ref/bam); every evolved
variable after the run agrees within 1e-12 relative.  Two modes:
"callback" replaces BAM's geometry rhs and boundary callbacks (BAM keeps its
RK4, vladd and algcon), "resident" runs the whole RK4 step + algcon on the
GPU at the EVOLVE hook."""
import os
import re
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


FMR_PAR = """physics = adm z4 nrharness%s
adm_data = Minkowski
z4_lapse = 1+log withshift
z4_shift = gamma0 withGadv withBadv withShiftadv withB
z4_shiftdriver = 2.0
z4_shiftgammacoeff = 0.75
z4_kappa1 = 0.02
z4_kappa2 = 0.0
grid = box
amr = bo newfmr
amr_fmr = nestedboxes
amr_lmax = 2
amr_nbuffer = 3
nxyz = 16
dxyz = 0.5
order_centered = 4
order_advection = 4
advection_lopsided = 1
order_dissipation = 6
dissipation_factor = 0.1
evolution_method = rk
evolution_method_rk = rk4
dtfac = 0.25
boundary = radiative
iterations = 2
mass1 = 1
mass2 = 0
nrharness_dir = .
nrharness_data = fourier
nrharness_amp = 0.05
nrharness_length = 16
nrharness_dump = 2 4 8
%s
"""


# the binary's grid: punctures at x = +-2.75 place one level-1 box and two
# separate level-2 boxes (the data are the harness's Fourier data)
BINARY = ("physics = adm z4 nrharness", "physics = adm z4 punctures nrharness"), ("nxyz = 16", "nxyz = 32"), \
    ("mass1 = 1\nmass2 = 0", "mass1 = 0.5\npx1 = 2.75\nmass2 = 0.5\npx2 = -2.75\npunctures_solver = none")
# the BSSN system on the single-puncture grid
BSSN_FMR = ("physics = adm z4 nrharness", "physics = adm bssn nrharness"), \
    ("""z4_lapse = 1+log withshift
z4_shift = gamma0 withGadv withBadv withShiftadv withB
z4_shiftdriver = 2.0
z4_shiftgammacoeff = 0.75
z4_kappa1 = 0.02
z4_kappa2 = 0.0""", """bssn_lapse = 1+log withshift
bssn_shift = gamma0 withGadv withBadv withShiftadv
bssn_shiftdriver = 2.0
bssn_shiftgammacoeff = 0.75""")


# the single-puncture grid with moving boxes: amr_move_force = 4 moves the
# puncture along x at speed amr_move_force_o (move.c:187-192), and level 2's
# box follows it by one level-1 cell at t = 0.1875 (level 2's 6th step)
MOVING = (("amr = bo newfmr", "amr = bo newfmr move\namr_move_force = 4\namr_move_force_o = 1.5\n"
                              "amr_verbose = move"),)


# the single-puncture grid with the CPBC2 background boundary on level 0
BACKGROUND = (("boundary = radiative", "boundary = background"),)


def run_fmr(binary, extra_physics, extra, grid="single", keep=None):
    """Dumps of every level after 2 coarse steps and the run's stdout; with
    keep, a list of output files (matched by name anywhere in the run
    directory) whose text is also returned."""
    work = tempfile.mkdtemp(prefix="bamgpu_")
    par = FMR_PAR
    for a, b in {"binary": BINARY, "bssn": BSSN_FMR, "moving": MOVING, "background": BACKGROUND}.get(grid, ()):
        assert a in par
        par = par.replace(a, b)
    try:
        with open(os.path.join(work, "t.par"), "w") as f:
            f.write(par % (extra_physics, extra))
        r = subprocess.run([binary, "-nt", "4", "t.par"], cwd=work, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
        dumps = [dumpfile.read(os.path.join(work, "state_it%d_l%d.bin" % (2 * 2 ** l, l))) for l in range(3)]
        if keep is None:
            return dumps, r.stdout
        texts = {}
        for root, _, files in os.walk(work):
            for fn in files:
                if fn in keep:
                    texts[fn] = open(os.path.join(root, fn)).read()
        return dumps, r.stdout, texts
    finally:
        shutil.rmtree(work, ignore_errors=True)


@pytest.mark.parametrize("grid", ["single", "binary", "bssn", "moving", "background"])
def test_bam_fmr_mode_matches_bam(gpu, cpu_state, grid):
    """nrgpu_mode = fmr: the whole Berger-Oliger step of the 3-level Z4c grid
    on the GPU at level 0's EVOLVE hook.  BAM dumps every level right after
    the level's own step (POST_EVOLVE), before its child restricts into it
    and before its parent prolongs into its buffer zone; with the GPU hook
    the host arrays already hold the end of the coarse step.  So the levels
    are compared, after 2 coarse steps, on the points that this last
    restriction and prolongation do not write, within the refinement
    tolerance of the oracle pin (2e-11).  The binary's grid has two boxes
    on level 2; "bssn" runs the BSSN system on the single-puncture grid;
    "moving" moves level 2's box once during the run (amr = bo newfmr move,
    forced motion), BAM on the host and the device hierarchy inside its
    coarse step, and the moved box is compared too; "background" runs
    level 0 with the CPBC2 box boundary."""
    from baum_b200 import abi
    from oracle import oracle
    ref, ref_out = run_fmr(BAM, "", "", grid)
    algcon = "bssn_register_algcon = no" if grid == "bssn" else "z4_register_algcon = no"
    got, out = run_fmr(BAM_GPU, " nrgpu", "nrgpu_mode = fmr\n" + algcon, grid)
    assert "nrgpu: fmr mode" in out
    if grid == "moving":
        assert "moving box(es) on level 2" in ref_out
        assert out.count("nrgpu: moved 1 level(s) from level 2 on") == ref_out.count("moving box(es) on level 2")
        for a, b in zip(got, ref):
            assert np.array_equal(np.asarray(a["boxes"]), np.asarray(b["boxes"]))
        # the box moved: its origin differs from the unmoved run's
        still, _ = run_fmr(BAM, "", "", "single")
        assert not np.array_equal(np.asarray(ref[2]["boxes"]), np.asarray(still[2]["boxes"]))
    levels = []
    for d in ref:
        levels.append(abi.Level([(int(b[0]), int(b[1]), int(b[2]), b[4], b[5], b[6]) for b in d["boxes"]],
                                float(d["dx"]), d["boundary"]))
    assert levels[2].desc.nboxes == (2 if grid == "binary" else 1)
    keep = [np.ones(lv.npoints, dtype=bool) for lv in levels]
    for l in (1, 2):
        uc = np.zeros((1, levels[l - 1].npoints))
        uf = np.ones((1, levels[l].npoints))
        oracle.fmr_restrict_prolong(levels[l - 1], levels[l], uc, uf, 4, 3)
        keep[l - 1] &= uc[0] < 0.5     # restricted parent points
        keep[l] &= uf[0] > 0.5         # prolonged buffer points (prolongation of zeros)
    for l in range(3):
        a, b = got[l]["data"][:, keep[l]], ref[l]["data"][:, keep[l]]
        err = np.abs(a - b).max(axis=1) / np.maximum(np.abs(b).max(axis=1), 1e-8)
        assert keep[l].sum() > 0.3 * levels[l].npoints
        assert err.max() < 2e-11, (l, err.max())


@pytest.mark.parametrize("method", ["int", "extint", "ext"])
def test_bam_fmr_mode_tracks_punctures(gpu, cpu_state, method):
    """nrgpu_mode = fmr with Gauge = moving_puncture on the binary's grid:
    the punctures are tracked on the device after every finest-level step
    and BAM's puncture positions are set from there, by the shift
    integrator, the extremum search of the lapse for the first puncture and
    the integrator for the second, or the search for both.  The positions
    after 2 coarse steps (8 finest steps) match the reference's own tracker
    on the CPU to the 7 digits of its output file
    (moving_punctureN_integrate, written with %14.6e by
    write_tracked_puncture_N, Gauge/moving_punctures.c:54-80)."""
    gauge = "Gauge = moving_puncture\nmoving_puncture_fixz = none\nmoving_puncture_track_method = " + method
    files = ["moving_puncture_integrate%d.lxyz2" % n for n in (1, 2)]
    _, _, texts = run_fmr(BAM, " Gauge", gauge, "binary", keep=files)
    _, out = run_fmr(BAM_GPU, " Gauge nrgpu", "nrgpu_mode = fmr\nz4_register_algcon = no\n" + gauge, "binary")
    got = {}
    for line in out.splitlines():
        if line.startswith("nrgpu: puncture "):
            w = line.split()
            got[int(w[2])] = np.array([float(x) for x in w[4:7]])
    assert sorted(got) == [1, 2]
    for n in (1, 2):
        rows = [r for r in texts[files[n - 1]].splitlines() if r.strip() and not r.startswith('"')]
        want = np.array([float(x) for x in rows[-1].split()[:3]])
        start = np.array([2.75 if n == 1 else -2.75, 0.0, 0.0])
        if method == "int" or (method == "extint" and n == 2):
            assert np.abs(want - start).max() > 1e-5  # the reference's integrated puncture moved
        assert np.abs(got[n] - want).max() <= 1e-6 * max(1.0, np.abs(want).max()), (n, got[n], want)


def run_mg(binary, extra_physics, extra):
    """The reference's puncture solve of tests/golden/mg_binary_34.par (a
    Bowen-York binary on a 34^3 grid, full-V multigrid to 1e-10); returns
    punctures_u after the solve and the run's stdout."""
    par = open(os.path.join(ROOT, "tests", "golden", "mg_binary_34.par")).read()
    par = par.replace("physics = adm punctures multigrid nrharness",
                      "physics = adm punctures multigrid nrharness" + extra_physics) + extra + "\n"
    work = tempfile.mkdtemp(prefix="bamgpu_")
    try:
        with open(os.path.join(work, "t.par"), "w") as f:
            f.write(par)
        r = subprocess.run([binary, "-nt", "4", "t.par"], cwd=work, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
        return dumpfile.read(os.path.join(work, "mg_u_l0.bin"))["data"][0], r.stdout
    finally:
        shutil.rmtree(work, ignore_errors=True)


def test_bam_multigrid_on_the_gpu_matches_bam(gpu, cpu_state):
    """nrgpu_multigrid = yes: BAM's punctures_solver = multigrid call
    (PunctureSolve.c:282) runs nrgpu_mg_solve; the same number of V cycles as
    BAM's own multigrid and the same u to 1e-10 relative (the tolerance of
    the multigrid parity tests)."""
    import re
    u_ref, out_ref = run_mg(BAM, "", "")
    u_gpu, out_gpu = run_mg(BAM_GPU, " nrgpu", "nrgpu_multigrid = yes")
    n_ref = int(re.search(r"after (\d+) V-cycles", out_ref).group(1))
    m = re.search(r"nrgpu_multigrid: (\d+) V-cycles on the GPU, residual ([0-9.e+-]+)", out_gpu)
    assert m, out_gpu[-2000:]
    assert int(m.group(1)) == n_ref
    assert float(m.group(2)) <= 1e-10
    assert np.abs(u_gpu - u_ref).max() <= 1e-10 * np.abs(u_ref).max()
    # switched off, the wrapped build runs BAM's own solver
    u_host, out_host = run_mg(BAM_GPU, " nrgpu", "nrgpu_multigrid = no")
    assert "multigrid on the host" in out_host
    assert np.abs(u_host - u_ref).max() <= 1e-12 * np.abs(u_ref).max()   # OpenMP sums may reorder


Z4_PAR = """physics = adm z4 nrharness%s
adm_data = Minkowski
z4_lapse = 1+log withshift
z4_shift = gamma0 withGadv withBadv withShiftadv withB
z4_shiftdriver = 2.0
z4_shiftgammacoeff = 0.75
z4_kappa1 = 0.02
z4_kappa2 = 0.0
grid = %s
nxyz = 20
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
iterations = 4
nrharness_dir = .
nrharness_data = fourier
nrharness_amp = 0.05
nrharness_length = 8
nrharness_dump = 4
%s
"""


def run_z4(binary, extra_physics, grid, extra, boundary="radiative"):
    work = tempfile.mkdtemp(prefix="bamgpu_")
    try:
        with open(os.path.join(work, "t.par"), "w") as f:
            f.write((Z4_PAR % (extra_physics, grid, extra)).replace("boundary = radiative", "boundary = " + boundary))
        r = subprocess.run([binary, "-nt", "4", "t.par"], cwd=work, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
        return dumpfile.read(os.path.join(work, "state_it4_l0.bin"))["data"], r.stdout
    finally:
        shutil.rmtree(work, ignore_errors=True)


@pytest.mark.parametrize("grid", ["box", "box octant"])
@pytest.mark.parametrize("mode,extra", [("callback", "nrgpu_mode = callback"),
                                        ("resident", "nrgpu_mode = resident\nz4_register_algcon = no")])
def test_bam_z4_with_the_gpu_path_matches_bam(gpu, cpu_state, grid, mode, extra):
    """The Z4c system inside BAM: the GPU rhs and boundary callbacks (BAM
    keeps its RK4 and algcon), or the whole RK4 step at the EVOLVE hook, on
    a plain box and on an octant grid (symmetry reflections), against plain
    BAM after 4 steps."""
    ref, _ = run_z4(BAM, "", grid, "")
    got, out = run_z4(BAM_GPU, " nrgpu", grid, extra)
    assert "nrgpu: %s mode" % mode in out
    assert relerr(got, ref).max() < 1e-12


@pytest.mark.parametrize("boundary", ["background", "background radcentered"])
@pytest.mark.parametrize("mode,extra", [("callback", "nrgpu_mode = callback"),
                                        ("resident", "nrgpu_mode = resident\nz4_register_algcon = no")])
def test_bam_z4_background_boundary_matches_bam(gpu, cpu_state, boundary, mode, extra):
    """The Z4c background box boundaries inside BAM (CPBC2 and the centred
    radiative condition): the state extrapolated by the rhs persists through
    BAM's RK4 in the callback mode, and the resident step writes out
    evolve_rk_rk4; against plain BAM after 4 steps."""
    ref, _ = run_z4(BAM, "", "box", "", boundary)
    got, out = run_z4(BAM_GPU, " nrgpu", "box", extra, boundary)
    assert "nrgpu: %s mode" % mode in out
    assert relerr(got, ref).max() < 1e-12


def run_moving(binary, extra_physics, extra):
    """tests/test_moving_policy.py's 4-level grid with two puncture boxes
    on the forced circular motion, 2 coarse steps: the run's stdout and,
    per level, the dump after its last step and the dump after its last
    move, if it moved after that step (nrharness_dump_moved)."""
    from test_moving_policy import MOVING_PAR
    work = tempfile.mkdtemp(prefix="bamgpu_")
    try:
        with open(os.path.join(work, "t.par"), "w") as f:
            f.write(MOVING_PAR % (extra_physics, extra))
        r = subprocess.run([binary, "-nt", "4", "t.par"], cwd=work, capture_output=True, text=True, timeout=900)
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
        state, moved = [], []
        for l in range(4):
            it = 2 * 2 ** l
            state.append(dumpfile.read(os.path.join(work, "state_it%d_l%d.bin" % (it, l))))
            fn = os.path.join(work, "moved_it%d_l%d.bin" % (it, l))
            moved.append(dumpfile.read(fn) if os.path.exists(fn) else None)
        return state, moved, r.stdout
    finally:
        shutil.rmtree(work, ignore_errors=True)


def test_bam_fmr_mode_moving_cascade_matches_bam(gpu, cpu_state):
    """Moving boxes inside the device's coarse step against BAM's own
    move_box: 4 levels, two puncture boxes on level 3 and joined boxes
    below, every level following the forced motion, 2 coarse steps with
    12 moves (cascades from level 1 at the end of each coarse step and
    moves of level 3 within it).  The module's hook decides with BAM's
    find_nested_bboxes and make_level_bboxes and moves the device data with
    nrgpu_fmr_regrid.  After the run every level has the reference's boxes
    and the reference's state: after its last move for the levels that
    moved at the end of the last coarse step, else after its last step.
    The points compared are those that no restriction or prolongation
    writes after the reference's dump (with the GPU hook BAM's host
    recursion still runs its own restriction and prolongation on the host
    arrays, from time levels it never computed); tolerance 2e-11 x 4^level
    (workloads.level_tolerance)."""
    from baum_b200 import abi, workloads
    from oracle import oracle
    ref, ref_moved, ref_out = run_moving(BAM, "", "")
    got, _, out = run_moving(BAM_GPU, " nrgpu", "nrgpu_mode = fmr\nz4_register_algcon = no")
    assert "nrgpu: fmr mode" in out
    nref = len(re.findall(r"(moving|setting) box\(es\) on level", ref_out))
    ngot = sum(int(x) for x in re.findall(r"nrgpu: moved (\d+) level", out))
    assert nref >= 10 and ngot == nref, (ngot, nref)
    final = [m if m is not None else d for m, d in zip(ref_moved, ref)]
    assert sum(m is not None for m in ref_moved) >= 2

    def level(d):
        return abi.Level([(int(b[0]), int(b[1]), int(b[2]), b[4], b[5], b[6]) for b in d["boxes"]],
                         float(d["dx"]), d["boundary"])

    lv = [level(d) for d in final]
    keep = [np.ones(x.npoints, dtype=bool) for x in lv]
    for l in range(1, 4):
        uf = np.ones((1, lv[l].npoints))
        oracle.fmr_restrict_prolong(lv[l - 1], lv[l], np.zeros((1, lv[l - 1].npoints)), uf, 4, 3)
        keep[l] &= uf[0] > 0.5  # prolonged buffer points
        # restricted points of the parent: from the child's boxes before its
        # last move (the reference's restriction) and after it (the host's)
        for child in (level(ref[l]), lv[l]):
            uc = np.zeros((1, lv[l - 1].npoints))
            oracle.fmr_restrict_prolong(lv[l - 1], child, uc, np.ones((1, child.npoints)), 4, 3)
            keep[l - 1] &= uc[0] < 0.5
    for l in range(4):
        assert np.array_equal(np.asarray(got[l]["boxes"]), np.asarray(final[l]["boxes"])), l
        a, b = got[l]["data"][:, keep[l]], final[l]["data"][:, keep[l]]
        err = np.abs(a - b).max(axis=1) / np.maximum(np.abs(b).max(axis=1), 1e-8)
        assert keep[l].sum() > 0.2 * lv[l].npoints, l
        assert err.max() < workloads.level_tolerance(l), (l, err.max())
