"""Regenerate the golden fixtures of tests/golden from the reference itself.

Runs the reference CPU code, built single-rank as oracle/_ref/bam by
oracle/build_ref.py, on small parfiles and stores its raw FP64 dumps
(oracle/harness/nrharness.c) as compressed .npz files.  Needs the reference
sources in this container; the fixtures it writes are committed so the tests
never need the reference at run time.

    python tests/golden/make_golden.py [case ...]
"""
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import dumpfile  # noqa: E402

BAM = os.path.join(ROOT, "oracle", "_ref", "bam")
OUT = os.path.dirname(os.path.abspath(__file__))

BSSN_COMMON = """
bssn_lapse = 1+log withshift
bssn_shift = gamma0 withGadv withBadv withShiftadv
bssn_shiftdriver = 2.0
bssn_shiftgammacoeff = 0.75
grid = box
evolution_method = rk
evolution_method_rk = rk4
dtfac = 0.25
boundary = radiative
dissipation_factor = 0.1
nrharness_dir = .
"""

CASES = {
    # generic smooth data: every term of the rhs is active (advection too)
    "bssn_fourier_o4": BSSN_COMMON + """
physics = adm bssn nrharness
adm_data = Minkowski
nxyz = 10
dxyz = 0.5
order_centered = 4
order_advection = 4
advection_lopsided = 1
order_dissipation = 6
iterations = 2
nrharness_dump = 0 2
nrharness_rhs = yes
nrharness_data = fourier
nrharness_amp = 0.05
nrharness_length = 4.5
nrharness_seed = 7
""",
    "bssn_fourier_o6": BSSN_COMMON + """
physics = adm bssn nrharness
adm_data = Minkowski
nxyz = 10
dxyz = 0.5
order_centered = 6
order_advection = 6
advection_lopsided6 = 2
order_dissipation = 6
iterations = 1
nrharness_dump = 0 1
nrharness_rhs = yes
nrharness_data = fourier
nrharness_amp = 0.05
nrharness_length = 4.5
nrharness_seed = 11
""",
    "bssn_fourier_o4_ko4": BSSN_COMMON + """
physics = adm bssn nrharness
adm_data = Minkowski
nxyz = 10
dxyz = 0.4
order_centered = 4
order_advection = 4
advection_lopsided = 1
order_dissipation = 4
iterations = 0
nrharness_dump = 0
nrharness_rhs = yes
nrharness_data = fourier
nrharness_amp = 0.08
nrharness_length = 3.6
nrharness_seed = 3
""",
    # single Schwarzschild puncture, precollapsed lapse, zero shift
    "bssn_punc_o4": BSSN_COMMON + """
physics = adm bssn punctures nrharness
mass1 = 1
mass2 = 0
punctures_solver = none
bssn_initial_lapse = oochi05
bssn_initial_shift = zero
nxyz = 10
dxyz = 0.5
order_centered = 4
order_advection = 4
advection_lopsided = 1
order_dissipation = 6
iterations = 4
nrharness_dump = 0 4
""",
    # symmetry reflections (set_boundary_symmetry, symmetry.c:93-140): the
    # puncture on an octant grid (two ghost planes below zero on each axis,
    # reflected with each variable's parity), and the Fourier data on a
    # bitant grid (z reflection only; the data themselves are not symmetric,
    # so the ghosts differ from the reflection until the first stage)
    "bssn_punc_octant": BSSN_COMMON.replace("grid = box", "grid = box octant") + """
physics = adm bssn punctures nrharness
mass1 = 1
mass2 = 0
punctures_solver = none
bssn_initial_lapse = oochi05
bssn_initial_shift = zero
nxyz = 24
dxyz = 0.25
order_centered = 4
order_advection = 4
advection_lopsided = 1
order_dissipation = 6
iterations = 4
nrharness_rhs = yes
nrharness_dump = 0 4
""",
    "bssn_fourier_bitant": BSSN_COMMON.replace("grid = box", "grid = box bitant") + """
physics = adm bssn nrharness
adm_data = Minkowski
nxyz = 14
dxyz = 0.5
order_centered = 4
order_advection = 4
advection_lopsided = 1
order_dissipation = 6
iterations = 2
nrharness_dump = 0 2
nrharness_rhs = yes
nrharness_data = fourier
nrharness_amp = 0.05
nrharness_length = 4.5
nrharness_seed = 3
""",
    # puncture with generic shift and KO: ADM variables and constraints
    "bssn_punc_con": BSSN_COMMON + """
physics = adm bssn punctures nrharness
mass1 = 1
mass2 = 0
punctures_solver = none
bssn_initial_lapse = oochi05
bssn_initial_shift = zero
nxyz = 12
dxyz = 0.5
order_centered = 4
order_advection = 4
advection_lopsided = 1
order_dissipation = 6
iterations = 3
nrharness_dump = 3
nrharness_constraints = yes
adm_normalizedConstraints = yes
""",
}


Z4_COMMON = """
physics = adm z4 nrharness
adm_data = Minkowski
z4_lapse = 1+log withshift
z4_shift = gamma0 withGadv withBadv withShiftadv withB
z4_shiftdriver = 2.0
z4_shiftgammacoeff = 0.75
z4_kappa1 = 0.02
z4_kappa2 = 0.0
grid = box
evolution_method = rk
evolution_method_rk = rk4
dtfac = 0.25
boundary = radiative
dissipation_factor = 0.1
nrharness_dir = .
nrharness_data = fourier
nrharness_amp = 0.05
"""

Z4_BG = Z4_COMMON.replace("boundary = radiative", "boundary = background radcentered") + """
nxyz = 12
dxyz = 0.5
order_centered = 4
order_advection = 4
advection_lopsided = 1
order_dissipation = 6
nrharness_length = 6.5
nrharness_seed = 3
"""

CASES.update({
    # the Z4c "background" box boundaries (set_boundary's background branch,
    # z4_boundary_box_rad / z4_boundary_box): one rhs with the boundary
    # callback, and 3 RK4 steps from the same data
    "z4_bg_rad_rhs": Z4_BG + "iterations = 0\nnrharness_dump = 0\nnrharness_rhs = yes\n",
    "z4_bg_rad": Z4_BG + "iterations = 3\nnrharness_dump = 0 3\n",
    "z4_bg_cpbc_rhs": Z4_BG.replace("background radcentered", "background") +
                      "iterations = 0\nnrharness_dump = 0\nnrharness_rhs = yes\n",
    "z4_bg_cpbc": Z4_BG.replace("background radcentered", "background") + "iterations = 3\nnrharness_dump = 0 3\n",
    "z4_fourier_o4": Z4_COMMON + """
nxyz = 10
dxyz = 0.5
order_centered = 4
order_advection = 4
advection_lopsided = 1
order_dissipation = 6
iterations = 2
nrharness_dump = 0 2
nrharness_rhs = yes
nrharness_length = 4.5
nrharness_seed = 5
""",
    # B-driver branch: "withB" must come before "withBadv" for the
    # reference's first-occurrence token test to see it
    "z4_fourier_o4_B": Z4_COMMON.replace("gamma0 withGadv withBadv withShiftadv withB",
                                         "gamma0 withB withGadv withBadv withShiftadv") + """
nxyz = 10
dxyz = 0.5
order_centered = 4
order_advection = 4
advection_lopsided = 1
order_dissipation = 4
iterations = 1
nrharness_dump = 0 1
nrharness_rhs = yes
nrharness_length = 4.5
nrharness_seed = 13
""",
    # ADM variables from the Z4c state and term-by-term normalised constraints
    "z4_fourier_con": Z4_COMMON + """
nxyz = 12
dxyz = 0.4
order_centered = 6
order_advection = 6
order_dissipation = 6
iterations = 2
nrharness_dump = 2
nrharness_constraints = yes
adm_normalizedConstraints = yes TermByTerm
nrharness_length = 4.8
nrharness_seed = 21
""",
    "z4_fourier_o6": Z4_COMMON + """
nxyz = 10
dxyz = 0.5
order_centered = 6
order_advection = 6
order_dissipation = 6
iterations = 1
nrharness_dump = 0 1
nrharness_rhs = yes
nrharness_length = 4.5
nrharness_seed = 9
""",
})

MG_CASES = {
    # Bowen-York binary with momenta and spins, multigrid to 1e-10 RMS
    "mg_binary_34": """
physics = adm punctures multigrid nrharness
mass1 = 0.5
px1 = 2.1
my1 = 0.1
sz1 = 0.1
mass2 = 0.6
px2 = -2.6
my2 = -0.1
sx2 = -0.05
sz2 = 0.08
punctures_solver = multigrid
punctures_persist = yes
punctures_tolerance = 1e-10
grid = box
nxyz = 32
dxyz = 0.5
mg_verbose = some
mg_vcycle_nmax = 2000
mg_relax_npre = 3
mg_relax_npost = 3
mg_size_nmin = 4
mg_exact_nmin = 10
mg_exact_nmax = 200
iterations = 0
nrharness_dir = .
nrharness_mg = yes
""",
}


# three nested levels, Berger-Oliger subcycling on every level, 4th-order
# restriction/prolongation with 3 buffer points, 3rd-order time
# interpolation; Fourier data on a flat background (the batched FMR
# workload at small size)
FMR_CASES = {
    "z4_fmr3": Z4_COMMON + """
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
iterations = 2
mass1 = 1
mass2 = 0
nrharness_length = 16
nrharness_seed = 1
nrharness_flags = yes
nrharness_dump = 0 2 4 8
""",
}
# a binary on the same kind of grid: the punctures' level-1 boxes merge
# into one 60x40x40 box, the level-2 boxes (40^3 around x = +-2.75) stay
# apart, so level 2 has two boxes (FlagRegridPunctures, FlagRegrid.c:34-160;
# the puncture data are replaced by the Fourier data, the punctures only
# place the boxes)
FMR_CASES["z4_fmr3_binary"] = FMR_CASES["z4_fmr3"].replace(
    "physics = adm z4 nrharness", "physics = adm z4 punctures nrharness").replace(
    "nxyz = 16", "nxyz = 32").replace("mass1 = 1\nmass2 = 0", """mass1 = 0.5
px1 = 2.75
mass2 = 0.5
px2 = -2.75
punctures_solver = none""")
# time interpolation of orders 4 and 6 (evolve.c:298-340) on the same grid:
# enough coarse steps that level 0 reaches the full order (iteration + 2 >
# order_timeinterpolation) and level 1 runs at it for several steps
for _o, _its in ((4, 4), (6, 6)):
    FMR_CASES["z4_fmr3_ti%d" % _o] = FMR_CASES["z4_fmr3"].replace(
        "iterations = 2", "iterations = %d\norder_timeinterpolation = %d" % (_its, _o)).replace(
        "nrharness_dump = 0 2 4 8", "nrharness_dump = 0 %d %d %d" % (_its, 2 * _its, 4 * _its))
# the dumps and fields kept: the end of the second coarse step on every
# level and the finest level after its second step; g11, chi, A12, Khat,
# Gamma1, Theta, alpha, beta1 (the initial state is regenerated by
# baum_b200/synthetic.py, bit for bit); for the binary, chi and alpha at the
# end of the second coarse step (the fixture stays near 4 MB)
FMR_KEEP = {"state_it2_l0", "state_it4_l1", "state_it8_l2", "state_it2_l2"}
FMR_VARS = [0, 6, 8, 13, 14, 17, 18, 19]
FMR_KEEP_BY_CASE = {"z4_fmr3": (FMR_KEEP, FMR_VARS),
                    "z4_fmr3_ti4": ({"state_it4_l0", "state_it8_l1", "state_it16_l2"}, FMR_VARS),
                    "z4_fmr3_ti6": ({"state_it6_l0", "state_it12_l1", "state_it24_l2"}, FMR_VARS),
                    "z4_fmr3_binary": ({"state_it2_l0", "state_it4_l1", "state_it8_l2"}, [6, 18])}

# the shift-integration puncture tracker (track_moving_puncture_integrate,
# Gauge/moving_punctures_integrate.c:29-100) run by the reference from a list
# of start positions after a state dump: a single box at order_RP 2, 4 and 6
# (positions inside, on nodes, within dequaleps of a node, and with
# interpolation cubes that leave the box), the octant (positions below the
# symmetry planes stay), and the binary's two-box finest level (positions in
# either box, between them, and with cubes that cross a box face)
TRACK_BOX_POINTS = ("0.1 -0.3 0.7  0.5 0.5 -0.5  1.23456789 -1.87654321 0.333333333  -2.2 0.0 0.4  "
                    "2.2 1.0 -1.0  1.74999999999 0.25 -0.75  -0.75 -0.75 -0.75  0.0 0.0 0.0  "
                    "-1.1 0.9 1.3")
TRACK_CASES = {
    "track_box": CASES["bssn_fourier_o4"].replace("nrharness_rhs = yes\n", "").replace(
        "nrharness_dump = 0 2", "nrharness_dump = 2\nnrharness_track = yes\nnrharness_track_points = "
        + TRACK_BOX_POINTS),
    "track_octant": CASES["bssn_punc_octant"].replace("nrharness_rhs = yes\n", "").replace(
        "nrharness_dump = 0 4", "nrharness_dump = 4\nnrharness_track = yes\nnrharness_track_points = "
        "0.3 0.4 0.2  -0.1 0.5 0.5  0.5 -0.2 0.6  0.6 0.7 -0.05  1.0 1.0 1.0  0.126 0.126 0.126  2.9 0.2 0.3"),
    "track_fmr_binary": FMR_CASES["z4_fmr3_binary"].replace("nrharness_flags = yes\n", "").replace(
        "nrharness_dump = 0 2 4 8", "nrharness_dump = 8\nnrharness_track = yes\nnrharness_track_points = "
        "2.75 0.1 -0.2  -2.6 0.3 0.1  0.0 0.0 0.0  0.4 0.0 0.0  0.6 0.2 0.1  5.0 0.0 0.0  5.1 0.0 0.0  "
        "-0.35 0.0 0.0  -2.9 -2.0 1.9  3.3 2.2 -2.2"),
}
for _o in (2, 6):
    TRACK_CASES["track_box_rp%d" % _o] = TRACK_CASES["track_box"] + "order_RP = %d\n" % _o
# with the Gauge project the harness also runs the extremum search
# (track_moving_puncture_extremum, moving_punctures_integrate.c:160-235) on
# the lapse (its defaults: minimum, minimal move 0.01 dx)
for _c in TRACK_CASES:
    _p = TRACK_CASES[_c]
    for _a in ("physics = adm bssn nrharness", "physics = adm bssn punctures nrharness",
               "physics = adm z4 punctures nrharness"):
        _p = _p.replace(_a, _a + " Gauge")
    TRACK_CASES[_c] = _p + "Gauge = moving_puncture\n"
# the reductions of the 0d output (write_level_0d, output0d.c:28-116: max,
# min, norm, normInf, integral over the flag-0 points) of the evolved list
# after a state dump, on a box and on an octant grid (SYMBOUND points
# excluded); the state and the reference's results are stored
RED0D_CASES = {
    "red0d_box": CASES["bssn_fourier_o4"].replace("nrharness_rhs = yes\n", "").replace(
        "nrharness_dump = 0 2", "nrharness_dump = 2\nnrharness_0d = yes"),
    "red0d_octant": CASES["bssn_punc_octant"].replace("nrharness_rhs = yes\n", "").replace(
        "nrharness_dump = 0 4", "nrharness_dump = 4\nnrharness_0d = yes"),
}


ADMMASS_COMMON = """
physics = adm bssn punctures ADM_mass nrharness
mass1 = 0.5
px1 = 1.0
my1 = 0.2
sz1 = 0.1
mass2 = 0.6
px2 = -1.2
my2 = -0.15
sx2 = 0.05
sz2 = -0.08
punctures_solver = none
bssn_initial_lapse = oochi05
bssn_initial_shift = zero
order_centered = 4
order_advection = 4
advection_lopsided = 1
order_dissipation = 6
iterations = 1
0doutiter = 1
ADM_mass_persist = yes
ADM_mass_ncircles = 21
ADM_mass_npoints = 40
nrharness_dump = 1
nrharness_admmass = yes
"""
ADMMASS_CASES = {
    # one box: a Bowen-York binary (momenta and spins) without the
    # Hamiltonian-constraint solve, after one RK4 step
    "admmass_box": BSSN_COMMON + ADMMASS_COMMON + """
nxyz = 24
dxyz = 0.4
ADM_mass_r = 2 3
""",
    # three nested levels: the integrands filled from parents and children
    # (set_boundary_refinement_cf) before the spheres of each level
    "admmass_fmr": BSSN_COMMON + ADMMASS_COMMON + """
nxyz = 16
dxyz = 0.8
amr = bo newfmr
amr_fmr = nestedboxes
amr_lmax = 2
amr_nbuffer = 3
ADM_mass_r = 1 2.5 3.5
""",
}


PSI4_EXTRA = """
nrharness_psi4 = yes
0doutput = rpsi4 ipsi4 Csqr
invariants_persist = yes
"""
PSI4_CASES = {
    # psi4, Csqr and the l = 2..4 modes of the same data
    "psi4_box": ADMMASS_CASES["admmass_box"].replace("physics = adm bssn punctures ADM_mass nrharness",
                                                     "physics = adm bssn punctures Invariants nrharness")
    .replace("nrharness_admmass = yes\n", PSI4_EXTRA.lstrip()).replace("ADM_mass_r = 2 3", "invariants_modes_r = 2 3"),
    "psi4_fmr": ADMMASS_CASES["admmass_fmr"].replace("physics = adm bssn punctures ADM_mass nrharness",
                                                     "physics = adm bssn punctures Invariants nrharness")
    .replace("nrharness_admmass = yes\n", PSI4_EXTRA.lstrip())
    .replace("ADM_mass_r = 1 2.5 3.5", "invariants_modes_r = 1 2.5 3.5"),
}


def run_psi4_case(name, par):
    """Per level of the final stack: geometry, the 16 inputs of the psi4
    computation (adm g, K, alpha, beta) in full, the reference's rpsi4,
    ipsi4 (restricted, prolonged, times r) and Csqr at 2048 seeded points,
    and its l = 2..4 modes at each radius from rpsi4_modes_rN.lL /
    ipsi4_modes_rN.lL (written with 17 digits, Invariants.c:580-600)."""
    work = tempfile.mkdtemp(prefix="golden_")
    try:
        with open(os.path.join(work, name + ".par"), "w") as f:
            f.write(par)
        r = subprocess.run([BAM, "-nt", "4", name + ".par"], cwd=work, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(r.stdout[-3000:] + r.stderr[-3000:])
        arrays = {}
        l = 0
        inv = os.path.join(work, name, "Invariants")
        while os.path.exists(os.path.join(work, "psi4_it%d_l%d.bin" % (2 ** l, l))):
            d = dumpfile.read(os.path.join(work, "psi4_it%d_l%d.bin" % (2 ** l, l)))
            arrays["boxes_l%d" % l] = np.array(d["boxes"], dtype=np.float64)
            arrays["dx_l%d" % l] = d["dx"]
            arrays["boundary_l%d" % l] = d["boundary"]
            arrays["inputs_l%d" % l] = d["data"][3:]
            idx = np.sort(np.random.default_rng(10 + l).choice(len(d["boundary"]), 2048, replace=False))
            arrays["sample_l%d" % l] = idx.astype(np.int32)
            arrays["psi4_l%d" % l] = d["data"][:3, idx]
            n = 1
            modes = []
            while os.path.exists(os.path.join(inv, "rpsi4_modes_r%d.l%d" % (n, l))):
                rr = np.loadtxt(os.path.join(inv, "rpsi4_modes_r%d.l%d" % (n, l)), comments='"', ndmin=2)[-1]
                ii = np.loadtxt(os.path.join(inv, "ipsi4_modes_r%d.l%d" % (n, l)), comments='"', ndmin=2)[-1]
                modes.append(np.stack([rr[1:], ii[1:]], axis=1))
                n += 1
            arrays["modes_l%d" % l] = np.array(modes)
            arrays["time_l%d" % l] = d["time"]
            l += 1
        np.savez_compressed(os.path.join(OUT, name + ".npz"), nlevels=l, **arrays)
        with open(os.path.join(OUT, name + ".par"), "w") as f:
            f.write(par.lstrip())
        print("wrote", name, l, "levels", [arrays["modes_l%d" % q].shape for q in range(l)])
    finally:
        shutil.rmtree(work)


def run_admmass_case(name, par):
    """Per level of the final time-aligned stack: geometry, the ADM mass
    inputs and the reference's integrands (admmass_itN_lL.bin), and its
    sphere integrals (admmass_itN_lL.txt: radius, 8 integrals)."""
    work = tempfile.mkdtemp(prefix="golden_")
    try:
        with open(os.path.join(work, name + ".par"), "w") as f:
            f.write(par)
        r = subprocess.run([BAM, "-nt", "4", name + ".par"], cwd=work, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(r.stdout[-3000:] + r.stderr[-3000:])
        arrays = {}
        l = 0
        while os.path.exists(os.path.join(work, "admmass_it%d_l%d.bin" % (2 ** l, l))):
            tag = "admmass_it%d_l%d" % (2 ** l, l)
            d = dumpfile.read(os.path.join(work, tag + ".bin"))
            arrays["boxes_l%d" % l] = np.array(d["boxes"], dtype=np.float64)
            arrays["dx_l%d" % l] = d["dx"]
            arrays["boundary_l%d" % l] = d["boundary"]
            # the 14 inputs in full; the reference's 8 integrands at 1024
            # seeded points (all of them on the points its spheres read
            # would make the fixture large)
            arrays["inputs_l%d" % l] = d["data"][8:]
            idx = np.sort(np.random.default_rng(l).choice(len(d["boundary"]), 1024, replace=False))
            arrays["sample_l%d" % l] = idx.astype(np.int32)
            arrays["integrands_l%d" % l] = d["data"][:8, idx]
            arrays["integrals_l%d" % l] = np.loadtxt(os.path.join(work, tag + ".txt"), ndmin=2).reshape(-1, 9)
            l += 1
        np.savez_compressed(os.path.join(OUT, name + ".npz"), nlevels=l, names=np.array(d["names"]), **arrays)
        with open(os.path.join(OUT, name + ".par"), "w") as f:
            f.write(par.lstrip())
        print("wrote", name, l, "levels", [arrays["integrals_l%d" % q].shape[0] for q in range(l)])
    finally:
        shutil.rmtree(work)


def run_red0d_case(name, par):
    work = tempfile.mkdtemp(prefix="golden_")
    try:
        with open(os.path.join(work, name + ".par"), "w") as f:
            f.write(par)
        r = subprocess.run([BAM, "-nt", "4", name + ".par"], cwd=work, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(r.stdout[-3000:] + r.stderr[-3000:])
        txt = [fn for fn in os.listdir(work) if fn.startswith("red0d_") and fn.endswith(".txt")][0]
        d = dumpfile.read(os.path.join(work, txt.replace("red0d_", "state_").replace(".txt", ".bin")))
        np.savez_compressed(os.path.join(OUT, name + ".npz"), state=d["data"], boundary=d["boundary"],
                            boxes=np.array(d["boxes"], dtype=np.float64), dx=d["dx"],
                            result=np.loadtxt(os.path.join(work, txt), ndmin=2))
        with open(os.path.join(OUT, name + ".par"), "w") as f:
            f.write(par.lstrip())
        print("wrote", name)
    finally:
        shutil.rmtree(work)


# the fields of a tracking fixture are kept within TRACK_HALO points of a
# start position (the rest is zero): the tracker reads only the cubes
# around the start positions, which the CPU pins check
TRACK_HALO = 5


def run_track_case(name, par):
    work = tempfile.mkdtemp(prefix="golden_")
    try:
        with open(os.path.join(work, name + ".par"), "w") as f:
            f.write(par)
        r = subprocess.run([BAM, "-nt", "4", name + ".par"], cwd=work, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(r.stdout[-3000:] + r.stderr[-3000:])
        arrays = {}
        for fn in sorted(os.listdir(work)):
            if not (fn.startswith("track_") and fn.endswith(".txt")):
                continue
            tag = fn[:-4]
            res = np.loadtxt(os.path.join(work, fn), ndmin=2)
            d = dumpfile.read(os.path.join(work, tag + ".bin"))
            keep = np.zeros(len(d["boundary"]), dtype=bool)
            for bx in d["boxes"]:
                m, n, o, off = (int(v) for v in bx[:4])
                x0 = np.array(bx[4:7])
                for p in res[::2, 2:5]:
                    c = np.floor((p - x0) / np.array([d["dx"], d["dy"], d["dz"]]) + 0.5).astype(int)
                    lo = np.maximum(c - TRACK_HALO, 0)
                    hi = np.minimum(c + TRACK_HALO + 1, [m, n, o])
                    if np.any(lo >= hi):
                        continue
                    k, j, i = np.meshgrid(np.arange(lo[2], hi[2]), np.arange(lo[1], hi[1]),
                                          np.arange(lo[0], hi[0]), indexing="ij")
                    keep[off + i + m * j + m * n * k] = True
            idx = np.nonzero(keep)[0].astype(np.int32)
            arrays[tag + "_idx"] = idx
            arrays[tag + "_beta"] = d["data"][:, idx]
            arrays[tag + "_boxes"] = np.array(d["boxes"], dtype=np.float64)
            arrays[tag + "_h"] = np.array([d["dx"], d["dy"], d["dz"], d["dt"]])
            arrays[tag + "_boundary"] = d["boundary"].astype(np.int8)
            arrays[tag + "_result"] = res
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **arrays)
        with open(os.path.join(OUT, name + ".par"), "w") as f:
            f.write(par.lstrip())
        print("wrote", name, sorted(arrays))
    finally:
        shutil.rmtree(work)


def run_fmr_case(name, par):
    work = tempfile.mkdtemp(prefix="golden_")
    try:
        with open(os.path.join(work, name + ".par"), "w") as f:
            f.write(par)
        r = subprocess.run([BAM, "-nt", "4", name + ".par"], cwd=work, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(r.stdout[-3000:] + r.stderr[-3000:])
        arrays = {}
        for l in range(3):
            d = dumpfile.read(os.path.join(work, "state_it0_l%d.bin" % l))
            arrays["boxes_l%d" % l] = np.array(d["boxes"], dtype=np.float64)
            arrays["dx_l%d" % l] = d["dx"]
            arrays["boundary_l%d" % l] = d["boundary"]
            fl = dumpfile.read(os.path.join(work, "flags_l%d.bin" % l))
            for nm, a in zip(fl["names"], fl["data"]):
                arrays["%s_l%d" % (nm, l)] = a.astype(np.int8)
        keep, fvars = FMR_KEEP_BY_CASE[name]
        for tag in sorted(keep):
            d = dumpfile.read(os.path.join(work, tag + ".bin"))
            arrays[tag] = d["data"][fvars]
        np.savez_compressed(os.path.join(OUT, name + ".npz"), vars=np.array(fvars), **arrays)
        with open(os.path.join(OUT, name + ".par"), "w") as f:
            f.write(par.lstrip())
        print("wrote", name, sorted(arrays))
    finally:
        shutil.rmtree(work)


def run_mg_case(name, par):
    import re
    work = tempfile.mkdtemp(prefix="golden_")
    try:
        with open(os.path.join(work, name + ".par"), "w") as f:
            f.write(par)
        r = subprocess.run([BAM, "-nt", "4", name + ".par"], cwd=work, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(r.stdout[-3000:] + r.stderr[-3000:])
        ncyc = int(re.search(r"after (\d+) V-cycles", r.stdout).group(1))
        # residual table after the cycles: the finest level is the last row
        block = r.stdout.split("V-cycles")[-1]
        res = float(re.findall(r"l\d+\s+\d+x\s*\d+x\s*\d+\s+([0-9.e+-]+)", block)[-1])
        d = dumpfile.read(os.path.join(work, "mg_u_l0.bin"))
        np.savez_compressed(os.path.join(OUT, name + ".npz"), u=d["data"][0], dx=d["dx"],
                            m=d["boxes"][0][0], vcycles=ncyc, residual=res)
        with open(os.path.join(OUT, name + ".par"), "w") as f:
            f.write(par.lstrip())
        print("wrote", name, "V-cycles", ncyc, "residual", res)
    finally:
        shutil.rmtree(work)


def run_case(name, par):
    work = tempfile.mkdtemp(prefix="golden_")
    try:
        with open(os.path.join(work, name + ".par"), "w") as f:
            f.write(par)
        r = subprocess.run([BAM, "-nt", "4", name + ".par"], cwd=work, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(r.stdout[-3000:] + r.stderr[-3000:])
        arrays = {}
        meta = None
        for fn in sorted(os.listdir(work)):
            if not fn.endswith(".bin"):
                continue
            d = dumpfile.read(os.path.join(work, fn))
            tag = fn[:-4]
            arrays[tag] = d["data"]
            if meta is None:
                meta = d
        np.savez_compressed(os.path.join(OUT, name + ".npz"), boundary=meta["boundary"],
                            boxes=np.array(meta["boxes"], dtype=np.float64),
                            dx=meta["dx"], dt=meta["dt"] if meta["dt"] else 0.25 * meta["dx"],
                            names=np.array(meta["names"]), **arrays)
        with open(os.path.join(OUT, name + ".par"), "w") as f:
            f.write(par.lstrip())
        print("wrote", name, sorted(arrays))
    finally:
        shutil.rmtree(work)


if __name__ == "__main__":
    if not os.path.exists(BAM):
        sys.exit("oracle/_ref/bam missing: run python oracle/build_ref.py first")
    only = set(sys.argv[1:])  # optional: regenerate only the named cases
    for n, p in CASES.items():
        if not only or n in only:
            run_case(n, p)
    for n, p in MG_CASES.items():
        if not only or n in only:
            run_mg_case(n, p)
    for n, p in FMR_CASES.items():
        if not only or n in only:
            run_fmr_case(n, p)
    for n, p in TRACK_CASES.items():
        if not only or n in only:
            run_track_case(n, p)
    for n, p in RED0D_CASES.items():
        if not only or n in only:
            run_red0d_case(n, p)
    for n, p in ADMMASS_CASES.items():
        if not only or n in only:
            run_admmass_case(n, p)
    for n, p in PSI4_CASES.items():
        if not only or n in only:
            run_psi4_case(n, p)
