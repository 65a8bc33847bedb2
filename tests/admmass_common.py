"""Shared pieces of the ADM mass tests: the fixtures of tests/golden/
admmass_*.npz (made from the reference by tests/golden/make_golden.py) and
the comparison of integrands and integrals with the reference's."""
import numpy as np

from conftest import load_golden

NTHETA, NPHI, ORDER = 21, 40, 4   # ADM_mass_ncircles / _npoints, order_centered


def levels_of(g):
    from baum_b200 import abi
    out = []
    for l in range(int(g["nlevels"])):
        boxes = [(int(b[0]), int(b[1]), int(b[2]), b[4], b[5], b[6]) for b in g["boxes_l%d" % l]]
        out.append(abi.Level(boxes, float(g["dx_l%d" % l]), g["boundary_l%d" % l]))
    return out


def load(name):
    g = load_golden(name)
    return g, levels_of(g)


def check_integrands(g, l, got, tol=1e-12):
    """got (8, npoints) against the reference's at its sampled points,
    relative to each field's largest sampled value."""
    idx = g["sample_l%d" % l]
    want = g["integrands_l%d" % l]
    a = np.asarray(got)[:, idx]
    err = np.abs(a - want).max(axis=1) / np.maximum(np.abs(want).max(axis=1), 1e-300)
    assert err.max() < tol, (l, err)


def check_integrals(g, l, got_rows, tol=1e-11):
    """got_rows: [(r, [8 integrals])] for the radii the reference used;
    relative to the mass (full) integral of the row for the momenta, whose
    own values can be near zero."""
    want = g["integrals_l%d" % l]
    assert [r for r, _ in got_rows] == list(want[:, 0]), (l, [r for r, _ in got_rows], want[:, 0])
    for (r, vals), row in zip(got_rows, want):
        vals = np.asarray(vals)
        scale = np.maximum(np.abs(row[1:]), np.abs(row[1]))
        err = np.abs(vals - row[1:]) / scale
        assert err.max() < tol, (l, r, err, vals, row[1:])
