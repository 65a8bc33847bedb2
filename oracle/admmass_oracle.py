"""CPU restatement of the reference's ADM mass analysis (test infrastructure,
the checker of the device path; never used by the product).

* integrands(level, inputs): the eight integrands of ADM_mass
  (projects/ADM_mass/ADM_mass.c:80-87): adm_mass_integrand.c (the surface
  term g^jk (d_j g_ik - d_i g_jk) N^i R^2 sqrt(det g) / 16 pi),
  adm_mass_integrand_chi.c ((d_i chi N^i) R^2 / (8 pi chi^1.25)) and
  adm_pj_integrand.c (P_m and J_m from v_m = g^jk N_j K_km - N_m K), at the
  flag-0 points, first derivatives by the 2nd-order centred stencil.
* sphere_integral(level, f, r, ntheta, nphi, order): integral_over_sphere_
  Simpson (utility/NumericUtils/Integral_over_sphere.c:197-357) with the
  value at each sphere point by interpolate_xyz_local_minimal
  (utility/interpolate/interpolate.c:633-676): a Lagrange cube of order^3
  nodes whose first node is floor((x - xmin + 1e-10)/h) - (order-1)/2
  from the level's lower corner, in the first box that holds that node and
  the whole cube; 0 if a point has none.

Pinned by tests/test_admmass_oracle.py to the reference's own integrands and
integrals (tests/golden/admmass_*.npz, made by tests/golden/make_golden.py).
"""
import math

import numpy as np

PI = 3.1415926535897932
EPS = 1e-10
SY = [[0, 1, 2], [1, 3, 4], [2, 4, 5]]


def _coords(level):
    return level.coords()


def integrands(level, inputs, out=None):
    """inputs: (14, npoints) = g (6), K (6), trK, chi; returns (8, npoints)
    with zeros off the flag-0 points (or the given out there)."""
    np_ = level.npoints
    out = np.zeros((8, np_)) if out is None else out
    x, y, z = _coords(level)
    h = [level.desc.dx, level.desc.dy, level.desc.dz]
    for b in level.boxes:
        m, n, o, off = b.m, b.n, b.o, b.noffset
        sl = slice(off, off + m * n * o)

        def box(a):
            return a[..., sl].reshape(a.shape[:-1] + (o, n, m))

        g = box(inputs[0:6])
        K = box(inputs[6:12])
        trK = box(inputs[12])
        chi = box(inputs[13])
        X = [box(x), box(y), box(z)]
        flag = box(level.boundary)
        inner = (flag == 0)
        # centred differences (zero at the faces, which are never flag 0)
        dg = np.zeros((3,) + g.shape)
        dchi = np.zeros((3,) + chi.shape)
        for d, ax in enumerate((-1, -2, -3)):
            s_p = [slice(None)] * 3
            s_m = [slice(None)] * 3
            s_c = [slice(None)] * 3
            s_p[ax] = slice(2, None)
            s_m[ax] = slice(0, -2)
            s_c[ax] = slice(1, -1)
            o2h = 1 / (2 * h[d])
            dg[d][(slice(None),) + tuple(s_c)] = o2h * (-g[(slice(None),) + tuple(s_m)] + g[(slice(None),) + tuple(s_p)])
            dchi[d][tuple(s_c)] = o2h * (-chi[tuple(s_m)] + chi[tuple(s_p)])
        det = (2. * g[1] * g[2] * g[4] + g[0] * g[3] * g[5] - g[5] * g[1] ** 2 - g[3] * g[2] ** 2
               - g[0] * g[4] ** 2)
        with np.errstate(divide="ignore", invalid="ignore"):
            idet = 1 / det
            gi = [idet * (g[3] * g[5] - g[4] ** 2), idet * (g[2] * g[4] - g[1] * g[5]),
                  idet * (-(g[2] * g[3]) + g[1] * g[4]), idet * (g[0] * g[5] - g[2] ** 2),
                  idet * (g[1] * g[2] - g[0] * g[4]), idet * (g[0] * g[3] - g[1] ** 2)]
            R = np.sqrt(X[0] ** 2 + X[1] ** 2 + X[2] ** 2)
            N = [X[a] / R for a in range(3)]
            area = R * R * np.sqrt(det)
            s = 0.0
            for a in range(3):
                for bb in range(3):
                    t = sum((dg[a][SY[c][bb]] - dg[c][SY[a][bb]]) * N[c] for c in range(3))
                    s = s + gi[SY[a][bb]] * t
            res = [0.0625 * s * area / PI,
                   0.125 * (dchi[0] * N[0] + dchi[1] * N[1] + dchi[2] * N[2]) * (R * R) / (PI * chi ** 1.25)]
            v = []
            for mm in range(3):
                w = sum(gi[SY[a][bb]] * N[a] * K[SY[bb][mm]] for a in range(3) for bb in range(3))
                v.append(w - N[mm] * trK)
            f8 = 0.125 * area / PI
            res += [v[0] * f8, v[1] * f8, v[2] * f8, (X[1] * v[2] - X[2] * v[1]) * f8,
                    (X[2] * v[0] - X[0] * v[2]) * f8, (X[0] * v[1] - X[1] * v[0]) * f8]
        for q in range(8):
            ob = out[q, sl].reshape(o, n, m)
            ob[inner] = res[q][inner]
    return out


def _lagrange(n, x, xmin, h):
    c = []
    for i in range(n):
        d = 1.0
        for j in range(n):
            if j != i:
                d *= ((x - xmin) - j * h) / ((i - j) * h)
        c.append(d)
    return c


def interpolate(level, f, p, order):
    """(value, found) at point p (interpolate_xyz_local_minimal)."""
    h = [level.desc.dx, level.desc.dy, level.desc.dz]
    lo = [min(b.x0 for b in level.boxes), min(b.y0 for b in level.boxes), min(b.z0 for b in level.boxes)]
    nh = (order - 1) // 2
    xc = [lo[d] + h[d] * (math.floor((p[d] - lo[d] + EPS) / h[d]) - nh) for d in range(3)]
    for b in level.boxes:
        org, dims = (b.x0, b.y0, b.z0), (b.m, b.n, b.o)
        idx = []
        for d in range(3):
            i = int(math.floor((xc[d] - org[d]) / h[d] + 0.5))
            if i < 0 or i >= dims[d] or abs(xc[d] - (org[d] + i * h[d])) > EPS:
                idx = None
                break
            idx.append(i)
        if idx is None:
            continue
        if any(idx[d] + order > dims[d] for d in range(3)):
            return 0.0, False
        i, j, k = idx
        cube = f[b.noffset:b.noffset + b.m * b.n * b.o].reshape(b.o, b.n, b.m)[k:k + order, j:j + order,
                                                                               i:i + order]
        cz = _lagrange(order, p[2], xc[2], h[2])
        cy = _lagrange(order, p[1], xc[1], h[1])
        cx = _lagrange(order, p[0], xc[0], h[0])
        vz = np.tensordot(np.array(cz), cube, axes=(0, 0))      # (y, x)
        vy = np.tensordot(np.array(cy), vz, axes=(0, 0))        # (x,)
        return float(np.dot(np.array(cx), vy)), True
    return 0.0, False


def sphere_integral(level, f, r, ntheta, nphi, order, center=(0.0, 0.0, 0.0)):
    """integral_over_sphere_Simpson on a grid without symmetry."""
    dtheta, dphi = PI / (ntheta + 1), 2.0 * PI / nphi
    ct = np.zeros(ntheta + 2)
    cp = np.zeros(nphi + 2)
    for i in range(1, ntheta - 1, 2):
        ct[i], ct[i + 1] = 2, 1
    ct[ntheta], ct[ntheta + 1] = 2, 0.5
    cp[1] = 0.5
    for i in range(2, nphi + 1, 2):
        cp[i], cp[i + 1] = 2, 1
    cp[nphi + 1] = 0.5
    total = 0.0
    for i in range(1, ntheta + 2):
        th = i * dtheta
        st, cs = math.sin(th), math.cos(th)
        for j in range(1, nphi + 2):
            ph = (j - 1) * dphi
            c = 4 * dtheta * dphi / 9 * ct[i] * cp[j] * st
            p = (center[0] + r * st * math.cos(ph), center[1] + r * st * math.sin(ph), center[2] + r * cs)
            v, ok = interpolate(level, f, p, order)
            if not ok:
                return 0.0
            total += c * v
    return total
