"""Small hand-built networks for the after-minimization quantities: filaments
whose tips sit a few nanometres from the planes of a cubic boundary, some
growing towards a plane and some away from it."""
import ctypes as C

import numpy as np

from medyan_b200._abi import BoundaryParams, CylindersView, NLParams, SystemView, f64
from medyan_b200.network import cubic_planes

BOX = 1000.0
CYL_LEN = 108.0


def tip_network(seed=0, n_fil=12, n_cyl=3):
    rng = np.random.default_rng(seed)
    planes = cubic_planes(BOX)
    xs, b1, b2, fil, pos, minus, st, bd = [], [], [], [], [], [], [], []
    for f in range(n_fil):
        p = planes[rng.integers(len(planes))]
        n = p[:3]
        # the plus-end tip 3-30 nm inside the plane (n points into the box),
        # the filament running back into the box along u, so the tip grows
        # towards the plane; every third filament lies nearly parallel to
        # the plane, so its minus end grows away from it (clamped projection)
        tip_dist = rng.uniform(3.0, 30.0)
        foot = rng.uniform(400.0, 600.0, 3)
        foot -= (n @ foot + p[3]) * n  # project onto the plane
        tip = foot + tip_dist * n
        if f % 3 == 2:
            t = rng.normal(size=3)
            t -= (t @ n) * n
            u = t / np.linalg.norm(t) + 0.1 * n
        else:
            u = n + 0.3 * rng.normal(size=3)
            u -= min(0.0, u @ n - 0.3) * n  # keep the body inside
        u /= np.linalg.norm(u)
        beads = [tip + (n_cyl - k) * CYL_LEN * u for k in range(n_cyl + 1)]
        base = len(xs)
        xs += beads
        for k in range(n_cyl):
            b1.append(base + k)
            b2.append(base + k + 1)
            fil.append(f)
            pos.append(k)
            minus.append(1 if k == 0 else 0)
            st.append((3 * (base + k), 3 * (base + k + 1)))
        for k in range(n_cyl - 1):
            bd.append((3 * (base + k), 3 * (base + k + 1), 3 * (base + k + 2)))
    x = np.asarray(xs).reshape(-1)
    nb = len(xs)
    sv = SystemView(nb, stretch_beads=np.array(st), stretch_k=np.full(len(st), 100.0),
                    stretch_l0=np.full(len(st), CYL_LEN), bend_beads=np.array(bd), bend_k=np.full(len(bd), 672.0),
                    bend_theta0=np.zeros(len(bd)))
    nc = len(b1)
    cv = CylindersView(b1, b2, np.arange(nc), fil, pos, np.zeros(nc), np.full(nc, -1), minus, np.full(nc, CYL_LEN),
                       np.full(nc, 1e5))
    nlp = NLParams()
    nlp.rmax, nlp.rmin = 54.0, 0.0
    for d in range(3):
        nlp.grid_size[d] = BOX
    planes_f = f64(planes)
    bp = BoundaryParams()
    bp.n_planes = len(planes)
    bp.plane_eq = planes_f.ctypes.data_as(C.POINTER(C.c_double))
    bp.k, bp.screen_length, bp.cutoff = 41.0, 2.7, 300.0
    # tips: the plus end (last cylinder) and the minus end (first) of each filament
    tips_cyl = [f * n_cyl + n_cyl - 1 for f in range(n_fil)] + [f * n_cyl for f in range(n_fil)]
    tips_plus = [1] * n_fil + [0] * n_fil
    return sv, x, cv, nlp, bp, planes_f, np.array(tips_cyl), np.array(tips_plus)
