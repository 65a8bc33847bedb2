"""CPU restatement of the Z4c "background" box boundary (test
infrastructure: the checker of the device path, never used by the product).

* extrapolate(level, u): set_boundary_extrapolate
  (utility/boundary/extrapolate.c:22-47) on the PHYBOUND points of every
  variable of u: per direction the linear extrapolation from the two inner
  neighbours where the point is on that face (else the centred mean, used
  only when no direction is on a face), the mean of the face directions;
  three passes.
* ladder(level): the flag-0 points one inside a box face
  (forinnerpoints_ijk_openmp + boundaryNaway(1),
  main/amr/bam_amr_loops_box.h:138,215).
* rad_rhs(level, u, pts): z4_boundary_box_rad (z4_boundary_box_rad.m),
  centred 2nd-order derivatives, s = x/r.
* cpbc_rhs(level, u, pts, p): z4_boundary_box (z4_boundary_box.m:14-420),
  the CPBC2 conditions, in einsum form, with the a <= b components of
  the symmetric tensors standing for both orders as in the generated code;
  the shift-driver terms are zero (z4_bc_use_eta = no).
* rhs(level, u, p, mode): the rhs with this boundary: the state
  extrapolated first (z4_rhs_movpunc_N.c:148-152), the interior rhs (the C
  oracle), the boundary rhs at the ladder points, the rhs extrapolated
  (utility/boundary/boundary.c:190-210).
* evolve(level, u, dt, nsteps, p, mode): evolve_rk_rk4 written out
  (utility/evolve/rk.c:216-255) and z4_algcon after each step.

Pinned by tests/test_z4bg_oracle.py to the reference's own rhs and states
(tests/golden/z4_bg_*.npz, made by tests/golden/make_golden.py).
"""
import ctypes as C

import numpy as np

from . import oracle

SY = [[0, 1, 2], [1, 3, 4], [2, 4, 5]]
MODES = {"rad": 1, "cpbc": 2}


def _box_of(level):
    """Per point: box index, i, j, k."""
    np_ = level.npoints
    bi = np.zeros(np_, dtype=np.int64)
    ijk = np.zeros((3, np_), dtype=np.int64)
    for n, b in enumerate(level.boxes):
        q = np.arange(b.m * b.n * b.o)
        s = slice(b.noffset, b.noffset + len(q))
        bi[s] = n
        ijk[0, s] = q % b.m
        ijk[1, s] = (q // b.m) % b.n
        ijk[2, s] = q // (b.m * b.n)
    return bi, ijk


def _geometry(level, pts):
    bi, ijk = _box_of(level)
    dims = np.array([[b.m, b.n, b.o] for b in level.boxes])[bi[pts]].T
    strides = np.array([[1, b.m, b.m * b.n] for b in level.boxes])[bi[pts]].T
    return ijk[:, pts], dims, strides


def extrapolate(level, u):
    """In place on u (nv, npoints); returns u."""
    pts = np.nonzero(level.boundary == 1)[0]
    if not len(pts):
        return u
    idx, dims, st = _geometry(level, pts)
    nb = []
    for d in range(3):
        # neighbours along d, the point itself where the box has none
        m1 = np.where(idx[d] >= 1, pts - st[d], pts)
        m2 = np.where(idx[d] >= 2, pts - 2 * st[d], pts)
        p1 = np.where(idx[d] + 1 < dims[d], pts + st[d], pts)
        p2 = np.where(idx[d] + 2 < dims[d], pts + 2 * st[d], pts)
        nb.append((idx[d] + 1 >= dims[d], idx[d] == 0, m1, m2, p1, p2))
    for _ in range(3):
        vals, use = [], []
        for at_hi, at_lo, m1, m2, p1, p2 in nb:
            hi = 2.0 * u[:, m1] - u[:, m2]
            lo = 2.0 * u[:, p1] - u[:, p2]
            mid = 0.5 * (u[:, p1] + u[:, m1])
            vals.append(np.where(at_hi, hi, np.where(at_lo, lo, mid)))
            use.append((at_hi | at_lo).astype(np.float64))
        nu = use[0] + use[1] + use[2]
        with np.errstate(invalid="ignore", divide="ignore"):
            face = (use[0] * vals[0] + use[1] * vals[1] + use[2] * vals[2]) / nu
        u[:, pts] = np.where(nu > 0, face, (vals[0] + vals[1] + vals[2]) / 3.0)
    return u


def ladder(level):
    bi, ijk = _box_of(level)
    dims = np.array([[b.m, b.n, b.o] for b in level.boxes])[bi].T
    near = np.zeros(level.npoints, dtype=bool)
    for d in range(3):
        near |= (ijk[d] == 1) | (ijk[d] == dims[d] - 2)
    return np.nonzero(near & (level.boundary == 0))[0]


class _Stencil:
    def __init__(self, level, u, pts):
        self.u, self.pts = u, pts
        self.idx, self.dims, self.st = _geometry(level, pts)
        self.h = [level.desc.dx, level.desc.dy, level.desc.dz]

    def v(self, var, off=0):
        return self.u[var, self.pts + off]

    def d1(self, var, a):
        s = self.st[a]
        return (1 / (2 * self.h[a])) * (-self.v(var, -s) + self.v(var, s))

    def d2(self, var, a, b):
        a, b = min(a, b), max(a, b)
        sa, sb = self.st[a], self.st[b]
        if a == b:
            return (1 / (self.h[a] * self.h[a])) * (-2. * self.v(var) + self.v(var, -sa) + self.v(var, sa))
        return (1 / (4 * self.h[a] * self.h[b])) * (self.v(var, -sa - sb) - self.v(var, sa - sb)
                                                    - self.v(var, -sa + sb) + self.v(var, sa + sb))


def _coords(level, pts):
    x, y, z = level.coords()
    return x[pts], y[pts], z[pts]


def rad_rhs(level, u, pts):
    """(11, npts): rhs of A (6), Khat, G (3), Theta."""
    S = _Stencil(level, u, pts)
    x, y, z = _coords(level, pts)
    r = np.sqrt(x * x + y * y + z * z)
    s = [x / r, y / r, z / r]

    def sdot(var):
        return s[0] * S.d1(var, 0) + s[1] * S.d1(var, 1) + s[2] * S.d1(var, 2)

    out = [-sdot(7 + q) - S.v(7 + q) / r for q in range(6)]
    out.append(-np.sqrt(2.0) * (sdot(13) + S.v(13) / r))
    out += [-sdot(14 + q) - S.v(14 + q) / r for q in range(3)]
    out.append(-sdot(17) - S.v(17) / r)
    return np.array(out)


def _sym(comp):
    """(P, 3, 3) from 6 components in xx, xy, xz, yy, yz, zz order."""
    return np.stack([np.stack([comp[SY[a][b]] for b in range(3)], -1) for a in range(3)], -2)


def cpbc_rhs(level, u, pts, p):
    """(11, npts): the CPBC2 rhs of A (6), Khat, G (3), Theta."""
    S = _Stencil(level, u, pts)
    P = len(pts)
    E = np.einsum
    g = _sym([S.v(q) for q in range(6)])
    A = _sym([S.v(7 + q) for q in range(6)])
    G = np.stack([S.v(14 + a) for a in range(3)], -1)
    beta = np.stack([S.v(19 + a) for a in range(3)], -1)
    chi, Khat, Theta, alpha = S.v(6), S.v(13), S.v(17), S.v(18)
    da = np.stack([S.d1(18, a) for a in range(3)], -1)
    dda = np.array([[S.d2(18, a, b) for b in range(3)] for a in range(3)]).transpose(2, 0, 1)
    db = np.array([[S.d1(19 + b, a) for b in range(3)] for a in range(3)]).transpose(2, 0, 1)
    ddb = np.array([[[S.d2(19 + c, a, b) for c in range(3)] for b in range(3)] for a in range(3)]).transpose(3, 0, 1, 2)
    dchi = np.stack([S.d1(6, a) for a in range(3)], -1)
    ddchi = np.array([[S.d2(6, a, b) for b in range(3)] for a in range(3)]).transpose(2, 0, 1)
    dg = np.array([[[S.d1(SY[a][b], c) for b in range(3)] for a in range(3)] for c in range(3)]).transpose(3, 0, 1, 2)
    ddg = np.array([[[[S.d2(SY[c][d], a, b) for d in range(3)] for c in range(3)] for b in range(3)]
                    for a in range(3)]).transpose(4, 0, 1, 2, 3)
    dKhat = np.stack([S.d1(13, a) for a in range(3)], -1)
    dA = np.array([[[S.d1(7 + SY[b][c], a) for c in range(3)] for b in range(3)] for a in range(3)]).transpose(3, 0, 1, 2)
    dG = np.array([[S.d1(14 + b, a) for b in range(3)] for a in range(3)]).transpose(2, 0, 1)
    dTheta = np.stack([S.d1(17, a) for a in range(3)], -1)
    # normal of the face (give_cube_normal, utility/boundary/normals.c:14-48)
    shat = np.zeros((P, 3))
    for a in range(3):
        shat[:, a] = np.where(S.idx[a] == S.dims[a] - 2, 1.0, np.where(S.idx[a] == 1, -1.0, 0.0))
    shat /= np.sqrt((shat * shat).sum(-1))[:, None]
    x, y, z = _coords(level, pts)
    r = np.sqrt(x * x + y * y + z * z)
    chig = np.where(chi < p.chiDivFloor, p.chiDivFloor, chi)
    g11, g12, g13, g22, g23, g33 = (S.v(q) for q in range(6))
    detginv = 1 / (2. * g12 * g13 * g23 + g11 * g22 * g33 - g33 * g12 ** 2 - g22 * g13 ** 2 - g11 * g23 ** 2)
    detginv = np.where(detginv < 0.00001, 1.0, detginv)
    ginv = detginv[:, None, None] * _sym([g22 * g33 - g23 ** 2, g13 * g23 - g12 * g33, g12 * g23 - g13 * g22,
                                          g11 * g33 - g13 ** 2, g12 * g13 - g11 * g23, g11 * g22 - g12 ** 2])
    Gi = chig[:, None, None] * ginv
    mod = E('pab,pa,pb->p', Gi, shat, shat)
    mod = np.where(mod < 0.00001, (shat * shat).sum(-1), mod)
    sd = shat / np.sqrt(mod)[:, None]
    su = E('pab,pb->pa', Gi, sd)
    dl = np.broadcast_to(np.eye(3), (P, 3, 3))
    qud = dl - E('pa,pb->pab', su, sd)
    qdd = g / chig[:, None, None] - E('pa,pb->pab', sd, sd)
    quu = Gi - E('pa,pb->pab', su, su)
    qP = 0.5 * (E('pca,pdb->pcdab', qud, qud) + E('pcb,pda->pcdab', qud, qud) - E('pcd,pab->pcdab', quu, qdd))
    muL = 2 / alpha
    muS = 1 / chig
    vbetas = 2 * np.sqrt(muS / 3)
    vbetaA = np.sqrt(muS)
    sdrv = 0.0
    K = Khat + 2 * Theta
    dK = dKhat + 2 * dTheta
    gdo = 0.5 * (E('pabc->pcab', dg) + E('pbac->pcab', dg) - dg)
    gam = E('pcd,pdab->pcab', ginv, gdo)
    Gfg = E('pbc,pabc->pa', ginv, gam)
    dGfg = (E('pbc,pde,padec->pab', ginv, ginv, ddg)
            - E('pbc,pdf,peg,pgef,pacd->pab', ginv, ginv, ginv, dg, dg)
            - E('pbe,pgc,pdf,pgef,pacd->pab', ginv, ginv, ginv, dg, dg))
    R = (E('pcd,pcdab->pab', ginv, -0.5 * ddg)
         + E('pcd,peca,pbed->pab', ginv, gam, gdo) + E('pcd,pecb,paed->pab', ginv, gam, gdo)
         + E('pcd,pead,pecb->pab', ginv, gam, gdo)
         + 0.5 * (E('pca,pbc->pab', g, dG) + E('pcb,pac->pab', g, dG) + E('pc,pabc->pab', Gfg, gdo)
                  + E('pc,pbac->pab', Gfg, gdo)))
    oocp = 1 / p.chipsipower
    f = oocp * np.log(chig)
    psim4 = np.exp(-4 * f)
    df = oocp * dchi / chig[:, None]
    ddf = oocp * ddchi / chig[:, None, None] - p.chipsipower * E('pa,pb->pab', df, df)
    cddf = ddf - E('pcab,pc->pab', gam, df)
    trcddf = E('pab,pab->p', ginv, cddf)
    dfdf = E('pcd,pc,pd->p', ginv, df, df)
    Rf = (R + 4 * E('pa,pb->pab', df, df) - 2 * cddf - 2 * g * trcddf[:, None, None]
          - 4 * g * dfdf[:, None, None])
    Rhat = psim4 * E('pab,pab->p', ginv, Rf)
    cdda = (dda - E('pcab,pc->pab', gam, da)
            - 2 * (E('pa,pb->pab', df, da) + E('pb,pa->pab', df, da)
                   - g * E('pcd,pc,pd->p', ginv, df, da)[:, None, None]))
    for a in range(3):
        for b in range(a):
            cdda[:, a, b] = cdda[:, b, a]
    trcdda = psim4 * E('pab,pab->p', ginv, cdda)
    AA = E('pcd,pac,pdb->pab', ginv, A, A)
    Ainv = E('pac,pbd,pcd->pab', ginv, ginv, A)
    cdA = dA - E('pdca,pbd->pcab', gam, A) - E('pdcb,pad->pcab', gam, A)
    divb = db[:, 0, 0] + db[:, 1, 1] + db[:, 2, 2]
    tdb = 2 / 3 * divb
    lieg = (E('pc,pcab->pab', beta, dg) - g * tdb[:, None, None] + E('pac,pbc->pab', db, g)
            + E('pbc,pac->pab', db, g))
    lieA = (E('pc,pcab->pab', beta, dA) - A * tdb[:, None, None] + E('pac,pbc->pab', db, A)
            + E('pbc,pac->pab', db, A))
    DKhat = E('pa,pa->p', su, dKhat)
    DK = E('pa,pa->p', su, dK)
    DTheta = E('pa,pa->p', su, dTheta)
    smuL = np.sqrt(muL)
    lienKhat = -smuL * DKhat - smuL * Khat / r
    lienTheta = -(DTheta + Theta / r) - p.kappa1 * (2 + p.kappa2) * Theta
    rKhat = E('pa,pa->p', beta, dKhat) + alpha * lienKhat
    rGams = (-vbetas * (dG[:, 0, 0] + dG[:, 1, 1] + dG[:, 2, 2]) + E('pb,pa,pab->p', sd, beta, dG)
             + 2 * sdrv / np.sqrt(3) / vbetaA * divb
             + E('pab,pc,pabc->p', quu, sd, ddb) / chig - E('pa,pbc,pabc->p', su, qud, ddb) / chig
             + 4 * alpha * smuL / (3 * (vbetas + smuL)) * DKhat / chig
             + 2 * alpha / (3 * (vbetas + 1)) * DTheta / chig)
    rTheta = alpha * lienTheta + E('pa,pa->p', beta, dTheta)
    dGd = dG - dGfg
    rACss = (-alpha * chig * (2 * E('pb,pca,pcab->p', su, ginv, cdA) - 4 / 3 * DK + 2 * DTheta
                              - 3 * E('pa,pbc,pc,pab->p', su, ginv, dchi, A) / chig
                              - p.kappa1 * chig * E('pa,pa->p', sd, G - Gfg)
                              + 2 / 3 * chig * E('pa,pb,pab->p', su, sd, dGd)
                              - 1 / 3 * chig * E('pab,pab->p', qud, dGd))
             + E('pa,pb,pab->p', su, su,
                 psim4[:, None, None] * (-cdda + alpha[:, None, None] * Rf)
                 - 1 / 3 * g * (-trcdda + alpha * Rhat)[:, None, None]
                 + alpha[:, None, None] * (K[:, None, None] * A - 2 * AA) + lieA))
    rACqq = chig * E('pab,pab->p', Ainv, -2 * alpha[:, None, None] * A + lieg) - rACss
    c1 = (1 / chig)[:, None]
    rGamA = (-vbetaA[:, None] * (E('pa,pkb,pab->pk', su, qud, dG) - E('pka,pb,pab->pk', quu, sd, dG) * c1)
             + E('pab,pkc,pabc->pk', quu, qud, ddb) * c1
             + 4 * E('pb,pc,pka,pabc->pk', su, sd, quu, ddb) / 3 * c1
             + E('pbc,pka,pabc->pk', qud, quu, ddb) / 3 * c1
             - 4 * alpha[:, None] * E('pka,pa->pk', quu, dKhat) / 3 * c1
             - 2 * alpha[:, None] * E('pka,pa->pk', quu, dTheta) / 3 * c1
             + (sdrv / (chig * vbetaA))[:, None] * (E('pa,pkb,pab->pk', su, qud, db)
                                                   - E('pa,pkb,pba->pk', sd, quu, db))
             + E('pkb,pa,pab->pk', qud, beta, dG))
    rACsA = (-(alpha * chig)[:, None] * (E('pbc,pda,pbcd->pa', ginv, qud, cdA) - 2 / 3 * E('pda,pd->pa', qud, dK)
                                         + E('pda,pd->pa', qud, dTheta)
                                         - 3 * E('pda,pbc,pbd,pc->pa', qud, ginv, A, dchi) / (2 * chi)[:, None]
                                         - p.kappa1 * chig[:, None] * E('pda,pd->pa', qdd, G - Gfg) / 2
                                         - E('pda,pb,pbd->pa', qud, su, Rf)
                                         + chig[:, None] * E('pb,pda,pbd->pa', su, qdd, dGd) / 2)
             - chig[:, None] * E('pda,pb,pbd->pa', qud, su, cdda)
             + alpha[:, None] * E('pb,pda,pbd->pa', su, qud, A * K[:, None, None] - 2 * AA)
             + E('pb,pda,pbd->pa', su, qud, lieA))
    inner = (E('pe,pecd->pcd', su, cdA) - 0.5 * E('pe,pcde->pcd', su, cdA) - 0.5 * E('pe,pdce->pcd', su, cdA)
             + (1 / (4 * chig))[:, None, None] * E('pe,pec,pd->pcd', su, A, dchi)
             + (1 / (4 * chig))[:, None, None] * E('pe,ped,pc->pcd', su, A, dchi)
             - (1 / (2 * chig))[:, None, None] * A * E('pe,pe->p', su, dchi)[:, None, None])
    rTF = (-alpha[:, None, None] * E('pcdab,pcd->pab', qP, inner)
           - chig[:, None, None] * E('pcdab,pcd->pab', qP, cdda)
           - alpha[:, None, None] * E('pcdab,pcd->pab', qP, AA)
           + 2 / 3 * (alpha * K)[:, None, None] * E('pcdab,pcd->pab', qP, A)
           + E('pcdab,pcd->pab', qP, lieA))
    rA = (rTF + E('pka,pb,pk->pab', qud, sd, rACsA) + E('pkb,pa,pk->pab', qud, sd, rACsA)
          + E('pa,pb->pab', sd, sd) * rACss[:, None, None] + qdd / 2 * rACqq[:, None, None])
    rG = su * rGams[:, None] + E('pak,pk->pa', qud, rGamA)
    out = [rA[:, a, b] for a in range(3) for b in range(a, 3)]
    out.append(rKhat)
    out += [rG[:, a] for a in range(3)]
    out.append(rTheta)
    return np.array(out)


def boundary(level, unew, ucur, p, mode):
    """set_boundary's background branch with c = 0 (unew is the rhs)."""
    extrapolate(level, ucur)
    pts = ladder(level)
    bc = rad_rhs(level, ucur, pts) if MODES[mode] == 1 else cpbc_rhs(level, ucur, pts, p)
    unew[7:18, pts] = bc
    extrapolate(level, unew)
    return unew


def rhs(level, u, p, mode):
    """The rhs of u (25, npoints) with the background boundary; u is
    extrapolated on the boundary in place, as the reference does."""
    extrapolate(level, u)
    out = np.zeros_like(u)
    pu, pn = oracle._ptrs(u), oracle._ptrs(out)
    if oracle.lib().oracle_z4_rhs(C.byref(level.desc), pn, pu, 0.0, pu, C.byref(p)):
        raise RuntimeError("oracle z4 rhs failed")
    return boundary(level, out, u, p, mode)


def evolve(level, u, dt, nsteps, p, mode):
    for _ in range(nsteps):
        up = u.copy()
        a, b = (0.0, dt / 2, dt / 2, dt), (dt / 6, dt / 3, dt / 3, dt / 6)
        r = None
        for s in range(4):
            v = u if s == 0 else up + a[s] * r
            r = rhs(level, v, p, mode)
            u += b[s] * r
        oracle.lib().oracle_z4_algcon(C.byref(level.desc), oracle._ptrs(u), C.byref(p))
    return u
