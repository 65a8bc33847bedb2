"""Moving boxes for the host-side hierarchy (fmr.Hierarchy): the reference's
box arrangement around the punctures and the level built from it, for
grids without symmetry, driving nrgpu_fmr_regrid from the move hook.

* ``nested_bboxes``: find_nested_bboxes (main/amr/move.c:121-463) for one or
  two punctures and no symmetry: a box of the level's size around each
  puncture, centred on the puncture snapped to the parent's grid, boxes
  that overlap joined into their bounding box.
* ``level_of_bboxes``: the points of the finer level on those boxes
  (make_level_bboxes, main/amr/box.c:465-560): 2 (n + 1) points per coarse
  interval count n, first point a quarter parent cell below the box, the
  outer layer of every box the refinement boundary.
* ``MovingBoxes``: the hook of move_box (move.c:808-986): at each call for
  level l, the boxes of levels l.. from the positions at the parent's time;
  the levels whose boxes changed are regridded in one call.
"""
import numpy as np

from . import abi

EPS = 1e-10  # dequaleps (main/main/bam_main.h:19)
REFBOUND = -1  # refinement boundary flag (bam_amr.h)


def _dless(a, b):
    return a < b - EPS


def box_size(l_parent, nx, lcube=0, move_nxyz=0, nxyz_list=None, nbuffer=3, addextra=True):
    """Coarse points per side of a box of level l_parent + 1 (move.c:
    229-262): nx, amr_move_nxyz above amr_move_lcube, or the amr_nxyz
    list entry; plus the buffer; halved and rounded up to even."""
    n = nx
    if l_parent + 1 > lcube and move_nxyz:
        n = move_nxyz
    if nxyz_list:
        j = min(len(nxyz_list) - 1, l_parent + 1)
        n = int(nxyz_list[j])
        if n % 4:
            raise ValueError("box sizes in amr_nxyz have to be multiples of 4")
    if addextra:
        n += 2 * nbuffer
    return n // 2 + (n // 2) % 2


def nested_bboxes(h, n, positions, moving=True):
    """Bounding boxes [xmin, xmax, ymin, ymax, zmin, zmax] of the child
    boxes on a parent of spacing h, and their coarse interval counts: n
    coarse points per side around each position (all at the origin when
    not moving: the fixed cubes of levels up to amr_move_lcube; forced
    positions, amr_move_force >= 0, replace the origin there too,
    move.c:141-227), joined where they overlap (move.c:263-330)."""
    p = np.zeros_like(np.asarray(positions, dtype=float)) if not moving else np.asarray(positions, dtype=float)
    boxes = []
    for q in p:
        b = []
        for i in range(3):
            c = int(q[i] / h) * h  # (int) truncates toward zero, symmetric about the origin
            b += [c - (n - 1) * h / 2, c + (n - 1) * h / 2]
        boxes.append(b)

    def overlap(a, b):
        return all(not (_dless(a[2 * d + 1], b[2 * d]) or _dless(b[2 * d + 1], a[2 * d])) for d in range(3))

    i = 0
    while i < len(boxes) - 1:
        j = i + 1
        while j < len(boxes):
            if overlap(boxes[i], boxes[j]):
                a, b = boxes[i], boxes[j]
                boxes[i] = [min(a[0], b[0]), max(a[1], b[1]), min(a[2], b[2]), max(a[3], b[3]),
                            min(a[4], b[4]), max(a[5], b[5])]
                del boxes[j]
                j = i + 1  # the reference restarts the inner loop (j = i, then j++)
            else:
                j += 1
        i += 1
    ibox = [[int((b[2 * d + 1] - b[2 * d]) / h + 0.5) for d in range(3)] for b in boxes]
    return boxes, ibox


def level_of_bboxes(boxes, ibox, h):
    """abi.Level of the finer level (spacing h / 2) on these boxes: the
    boxes one after the other, REFBOUND on each box's outer layer."""
    dx = h / 2
    spec, flags = [], []
    for b, ib in zip(boxes, ibox):
        m, n, o = (2 * (k + 1) for k in ib)
        spec.append((m, n, o, b[0] - dx / 2, b[2] - dx / 2, b[4] - dx / 2))
        e = [np.zeros(k, dtype=bool) for k in (m, n, o)]
        for a in e:
            a[0] = a[-1] = True
        e3 = e[2][:, None, None] | e[1][None, :, None] | e[0][None, None, :]
        flags.append(np.where(e3, REFBOUND, 0).astype(np.int32).ravel())
    return abi.Level(spec, dx, np.concatenate(flags))


def circle_positions(r, omega):
    """The forced motion amr_move_force = 3 (move.c:176-186): two punctures
    on an ellipse of half-axes 0.9 r (x) and r (y), half a turn apart."""
    def pos(t):
        return np.array([[0.9 * r * np.sin(np.pi + omega * t), r * np.cos(np.pi + omega * t), 0.0],
                         [0.9 * r * np.sin(omega * t), r * np.cos(omega * t), 0.0]])
    return pos


class MovingBoxes:
    """move_box for a fmr.Hierarchy: levels above lcube follow positions(t)
    (n x 3 array at time t), levels 1..lcube stay cubes about the origin
    (unless forced: then every level follows the positions).
    sizes(l_parent) gives the coarse points per side of level l_parent + 1's
    boxes (box_size).  Install with hierarchy.set_move(policy.hook) after
    giving the list of states that advance steps (policy.u)."""

    def __init__(self, H, positions, sizes, lcube=0, forced=False):
        self.H = H
        self.positions = positions
        self.sizes = sizes
        self.lcube = lcube
        self.forced = forced  # amr_move_force >= 0: positions on every level
        self.u = None
        self.moves = []
        # the current boxes of every parent (level->sbox): those that built
        # the hierarchy's levels
        self.sbox = {}
        for l in range(1, len(H.levels)):
            self.sbox[l - 1] = self.boxes_of(l - 1, self.H.iteration(l - 1) * H.dt[l - 1])[0]

    def boxes_of(self, lp, t):
        h = self.H.levels[lp].dx
        return nested_bboxes(h, self.sizes(lp), self.positions(t), moving=self.forced or lp + 1 > self.lcube)

    def hook(self, l, stream):
        H = self.H
        new = []
        for lv in range(l, len(H.levels)):
            t = H.iteration(lv - 1) * H.dt[lv - 1]
            boxes, ibox = self.boxes_of(lv - 1, t)
            old = self.sbox.get(lv - 1)
            if old is not None and len(old) == len(boxes) and all(
                    all(not (_dless(a, b) or _dless(b, a)) for a, b in zip(x, y)) for x, y in zip(old, boxes)):
                new.append(None)
                continue
            self.sbox[lv - 1] = boxes
            # a new level has no boxes of its own yet (make_level_bboxes
            # leaves level->sbox empty): its child is set up again
            self.sbox[lv] = None
            new.append(level_of_bboxes(boxes, ibox, H.levels[lv - 1].dx))
        if any(x is not None for x in new):
            self.moves.append((l, [H.iteration(q) for q in range(len(H.levels))],
                               [None if x is None else [(b.m, b.n, b.o, b.x0, b.y0, b.z0) for b in x.boxes]
                                for x in new]))
            H.regrid(l, new, self.u, stream)
