"""The box arrangement of baum_b200/moving.py against the reference's own
moving grid: the reference binary (oracle/_ref/bam) runs a 4-level Z4c grid
whose two puncture boxes follow the forced circular motion (amr = bo newfmr
move, amr_move_force = 3, move.c:176-186) with amr_verbose = move, which
prints every move (move.c:880-895).  The same calls of move_box, replayed
in the reference's recursion order (main.c:397-446) with nested_bboxes and
box_size, give the same sequence of moves and boxes (to the printed 3
decimals), and level_of_bboxes the same points per box."""
import os
import re
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT
from baum_b200 import moving

BAM = os.path.join(ROOT, "oracle", "_ref", "bam")

# two punctures on a circle of radius 1 at angular velocity 3; levels 1-2
# sized by nxyz, level 3 by amr_move_nxyz, every level following the forced
# positions
MOVING_PAR = """physics = adm z4 punctures nrharness%s
punctures_solver = none
mass1 = 0.5
px1 = 1.0
mass2 = 0.5
px2 = -1.0
z4_lapse = 1+log withshift
z4_shift = gamma0 withGadv withBadv withShiftadv withB
z4_shiftdriver = 2.0
z4_shiftgammacoeff = 0.75
z4_kappa1 = 0.02
z4_kappa2 = 0.0
grid = box
amr = bo newfmr move
amr_fmr = nestedboxes
amr_lmax = 3
amr_nbuffer = 3
amr_move_lcube = 2
amr_move_nxyz = 12
amr_move_force = 3
amr_move_force_r = 1.0
amr_move_force_o = 3.0
amr_verbose = move
nxyz = 48
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
nrharness_dir = .
nrharness_data = fourier
nrharness_amp = 0.05
nrharness_length = 16
nrharness_dump = 2 4 8 16
nrharness_dump_moved = yes
%s
"""
NX, LCUBE, MOVE_NXYZ, NBUF, LMAX, DX0, DTFAC = 48, 2, 12, 3, 3, 0.5, 0.25

BOX = re.compile(r"l=(\d+), h=[0-9.,]+: \[\s*([-0-9.]+),\s*([-0-9.]+)\]x\[\s*([-0-9.]+),\s*([-0-9.]+)\]x"
                 r"\[\s*([-0-9.]+),\s*([-0-9.]+)\]\s+(\d+)x(\d+)x(\d+)")


def reference_moves(out):
    """[(kind, level, [bbox...], [counts...])] from the printed moves."""
    lines = out.splitlines()
    ev = []
    i = 0
    while i < len(lines):
        m = re.match(r"(moving|setting) box\(es\) on level (\d+)", lines[i])
        if not m:
            i += 1
            continue
        kind, lev = m.group(1), int(m.group(2))
        i += 1
        if kind == "moving":  # "from", the old boxes, "to"; "setting ... to" is one line
            while not lines[i].startswith("to"):
                i += 1
            i += 1
        boxes, counts = [], []
        while i < len(lines) and BOX.match(lines[i]):
            g = BOX.match(lines[i]).groups()
            boxes.append([float(x) for x in g[1:7]])
            counts.append([int(x) for x in g[7:10]])
            i += 1
        ev.append((kind, lev, boxes, counts))
    return ev


def replayed_moves(nsteps):
    """The same calls of move_box with the restated arrangement."""
    pos = moving.circle_positions(1.0, 3.0)
    dx = [DX0 / 2 ** l for l in range(LMAX + 1)]
    dt = [DTFAC * h for h in dx]
    it = [0] * (LMAX + 1)
    sizes = lambda lp: moving.box_size(lp, NX, LCUBE, MOVE_NXYZ, nbuffer=NBUF)  # noqa: E731
    sbox = {lp: moving.nested_bboxes(dx[lp], sizes(lp), pos(0.0))[0] for lp in range(LMAX)}
    ev = []

    def move_box(L):
        for lv in range(L, LMAX + 1):
            t = it[lv - 1] * dt[lv - 1]
            boxes, ibox = moving.nested_bboxes(dx[lv - 1], sizes(lv - 1), pos(t))
            old = sbox.get(lv - 1)
            if old is not None and len(old) == len(boxes) and np.allclose(old, boxes, atol=1e-10, rtol=0):
                continue
            ev.append(("setting" if old is None else "moving", lv, boxes, [[k + 1 for k in b] for b in ibox]))
            sbox[lv - 1] = boxes
            sbox[lv] = None

    def advance(l):
        it[l] += 1
        if l < LMAX:
            advance(l + 1)
            advance(l + 1)
        if l + 1 <= LMAX:
            if l == 0 or it[l] * dt[l] < it[l - 1] * dt[l - 1] - 1e-10:
                move_box(l + 1)

    for _ in range(nsteps):
        advance(0)
    return ev


def test_restated_box_arrangement_moves_as_the_reference():
    if not os.path.exists(BAM):
        pytest.skip("the reference binary is built by oracle/build_ref.py where the reference sources exist")
    work = tempfile.mkdtemp(prefix="bammove_")
    try:
        with open(os.path.join(work, "t.par"), "w") as f:
            f.write(MOVING_PAR % ("", ""))
        r = subprocess.run([BAM, "-nt", "4", "t.par"], cwd=work, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-3000:]
    finally:
        shutil.rmtree(work, ignore_errors=True)
    ref = reference_moves(r.stdout)
    got = replayed_moves(2)
    assert len(ref) >= 10  # cascades from level 1 and moves of the two level-3 boxes
    assert [(k, l) for k, l, _, _ in got] == [(k, l) for k, l, _, _ in ref]
    for (_, _, bg, cg), (_, _, br, cr) in zip(got, ref):
        assert np.abs(np.array(bg) - np.array(br)).max() < 6e-4
        assert cg == cr
        # make_level_bboxes: 2 (n + 1) fine points per side of each box
        lev = moving.level_of_bboxes(bg, [[c - 1 for c in b] for b in cg], 1.0)
        assert [(b.m, b.n, b.o) for b in lev.boxes] == [tuple(2 * c for c in b) for b in cg]
