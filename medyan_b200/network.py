"""Seeded synthetic filament networks with the shapes of the benchmark workloads.

A network is what MEDYAN's SubSystem + ForceFieldManager::vectorizeAllForceFields
hand to the mechanics path: bead coordinates in DOF order, cylinder topology,
and the per-force-field index/parameter arrays. Excluded-volume and boundary
terms come from a neighbor-list build (on the GPU in the product, on the CPU
in the tests) and are filled in separately.

Generation rules follow the reference's random filament initializer
(src/FilamentInitializer.cpp:32-135): first point uniform in the grid,
direction uniform on the sphere (src/Rand.h:66-72), end point
p1 + (n_cyl*L_cyl - 0.01)*dir, accept only when both ends lie inside the cubic
boundary and at least BoundaryCutoff/4 from every plane. Beads are evenly
spaced between the ends, so every cylinder is slightly shorter than its
108 nm rest length. Randomness is numpy's MT19937 seeded per workload.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import ctypes as C

import numpy as np

from ._abi import BoundaryParams, CylindersView, NLParams, SystemView, f64

CYL_LEN = 108.0
BOUNDARY_OFFSET = 25.0  # BoundaryCubic planes sit 25 nm inside the grid (src/Structure/BoundaryImpl.cpp:28-34)


@dataclass
class NetworkSpec:
    """Composition of one workload (sizes in nm, constants in pN and nm)."""
    name: str
    n_fil: int
    cyl_per_fil: int
    box: float
    n_linker: int = 0
    n_motor: int = 0
    n_branch: int = 0
    seed: int = 0
    fstretch_k: float = 100.0        # FSTRETCHINGK
    fbend_k: float = 672.0           # FBENDINGK
    fbend_theta: float = 0.0         # FBENDINGTHETA
    volume_k: float = 1e5            # VOLUMEK
    volume_cutoff: float = 54.0      # VOLUMECUTOFF
    linker_k: float = 8.0
    linker_dist: tuple = (30.0, 40.0)
    motor_k: float = 2.5
    motor_dist: tuple = (175.0, 225.0)
    motor_l0: tuple = (175.0, 225.0)
    br_stretch_k: float = 100.0
    br_stretch_l0: float = 6.0
    br_bend_k: float = 10.0
    br_bend_theta: float = 1.22
    br_dihedral_k: float = 10.0
    br_position_k: float = 0.0       # BranchingPosition off unless set (k = 20 in the reference example)
    boundary_k: float = 41.0         # BOUNDARYINTERACTIONK
    boundary_slen: float = 2.7       # BOUNDARYSCREENLENGTH
    boundary_cutoff: float = 300.0   # BOUNDARYCUTOFF
    min_separation: float = 10.0     # placement: closest approach between cylinders of different filaments


# The five benchmark workloads: CPU-runnable plain FP64, medium, batched
# ensemble member composition, differentiation, large (400k cylinders).
def workload_spec(index: int, seed: int | None = None, **over) -> NetworkSpec:
    specs = {
        0: NetworkSpec("cfg0_50x10_2um", 50, 10, 2000.0, n_linker=100),
        1: NetworkSpec("cfg1_2000x20_5um", 2000, 20, 5000.0, n_linker=4000, n_motor=500, n_branch=400),
        3: NetworkSpec("cfg3_500x20_3um", 500, 20, 3000.0, n_linker=1000, n_motor=100),
        4: NetworkSpec("cfg4_20000x20_10um", 20000, 20, 10000.0, n_linker=100000, n_motor=10000, n_branch=5000),
    }
    s = specs[index]
    s.seed = index if seed is None else seed
    for k, v in over.items():
        setattr(s, k, v)
    return s


@dataclass
class Network:
    spec: NetworkSpec
    coords: np.ndarray                      # (n_beads, 3) float64, DOF order
    # cylinder topology, Cylinder::getCylinders() order
    cyl_bead1: np.ndarray
    cyl_bead2: np.ndarray
    cyl_id: np.ndarray
    cyl_fil: np.ndarray
    cyl_pos: np.ndarray
    cyl_type: np.ndarray
    cyl_branching: np.ndarray
    cyl_minus_end: np.ndarray
    cyl_eqlen: np.ndarray
    cyl_exclk: np.ndarray
    ff: dict = field(default_factory=dict)  # per-force-field arrays (SystemView keywords)

    @property
    def n_beads(self) -> int:
        return self.coords.shape[0]

    @property
    def n_cyl(self) -> int:
        return self.cyl_bead1.size

    def flat_coords(self) -> np.ndarray:
        return np.ascontiguousarray(self.coords.reshape(-1))

    def plane_eq(self) -> np.ndarray:
        return cubic_planes(self.spec.box)

    def nl_params(self) -> NLParams:
        p = NLParams()
        p.rmax = self.spec.volume_cutoff
        p.rmin = 0.0
        for d in range(3):
            p.grid_size[d] = self.spec.box
        return p

    def boundary_params(self):
        planes = f64(self.plane_eq())
        b = BoundaryParams()
        b.n_planes = planes.size // 4
        b.plane_eq = planes.ctypes.data_as(C.POINTER(C.c_double))
        b.k = self.spec.boundary_k
        b.screen_length = self.spec.boundary_slen
        b.cutoff = self.spec.boundary_cutoff
        return b, planes

    def cylinders_view(self) -> CylindersView:
        return CylindersView(self.cyl_bead1, self.cyl_bead2, self.cyl_id, self.cyl_fil, self.cyl_pos,
                             self.cyl_type, self.cyl_branching, self.cyl_minus_end, self.cyl_eqlen,
                             self.cyl_exclk)

    def system_view(self, **extra) -> SystemView:
        arrays = dict(self.ff)
        arrays.update(extra)
        return SystemView(self.n_beads, **arrays)


def cubic_planes(box: float) -> np.ndarray:
    """BoundaryCubic planes (src/Structure/BoundaryImpl.cpp:24-52) as a*x+b*y+c*z+d=0 rows."""
    lo = BOUNDARY_OFFSET
    hi = box - BOUNDARY_OFFSET
    rows = []
    for axis in range(3):
        for point, sign in ((lo, 1.0), (hi, -1.0)):
            n = [0.0, 0.0, 0.0]
            n[axis] = sign
            d = -sign * point
            rows.append(n + [d])
    return np.asarray(rows, dtype=np.float64)


def _unit_vectors(rng: np.random.Generator, n: int) -> np.ndarray:
    theta = rng.uniform(0.0, 2.0 * np.pi, n)
    z = rng.uniform(-1.0, 1.0, n)
    r = np.sqrt(1.0 - z * z)
    return np.stack([r * np.cos(theta), r * np.sin(theta), z], axis=1)


def _inside(p: np.ndarray, box: float, margin: float) -> np.ndarray:
    lo = BOUNDARY_OFFSET + margin
    hi = box - BOUNDARY_OFFSET - margin
    return np.all((p >= lo) & (p <= hi), axis=-1)


def seg_seg_distance(p1, q1, p2, q2):
    """Closest distance between segments p1-q1 and p2-q2 (row-wise, numpy)."""
    d1 = q1 - p1
    d2 = q2 - p2
    r = p1 - p2
    a = np.einsum("ij,ij->i", d1, d1)
    e = np.einsum("ij,ij->i", d2, d2)
    f = np.einsum("ij,ij->i", d2, r)
    c = np.einsum("ij,ij->i", d1, r)
    b = np.einsum("ij,ij->i", d1, d2)
    den = a * e - b * b
    s = np.where(den > 1e-12, np.clip((b * f - c * e) / np.where(den > 1e-12, den, 1.0), 0.0, 1.0), 0.0)
    t = (b * s + f) / e
    t0 = np.clip(t, 0.0, 1.0)
    s = np.where(t < 0.0, np.clip(-c / a, 0.0, 1.0), np.where(t > 1.0, np.clip((b - c) / a, 0.0, 1.0), s))
    t = t0
    c1 = p1 + d1 * s[:, None]
    c2 = p2 + d2 * t[:, None]
    return np.linalg.norm(c1 - c2, axis=1)


class _Placer:
    """Accepts straight filaments one batch at a time, rejecting any filament
    that comes closer than ``sep`` to a cylinder of another accepted filament
    (``ignore`` exempts one filament, e.g. a branch child's parent)."""

    def __init__(self, ncyl: int, sep: float):
        self.ncyl = ncyl
        self.sep = sep
        self.p = np.zeros((0, 3))   # cylinder start points
        self.q = np.zeros((0, 3))   # cylinder end points
        self.fil = np.zeros(0, np.int64)
        self.n_fil = 0
        self.tree = None
        self.frac = np.arange(ncyl + 1) / ncyl

    def _segments(self, start, direction, length):
        pts = start[:, None, :] + (length * self.frac)[None, :, None] * direction[:, None, :]
        return pts[:, :-1, :].reshape(-1, 3), pts[:, 1:, :].reshape(-1, 3), pts

    def _rebuild(self):
        from scipy.spatial import cKDTree
        self.tree = cKDTree(0.5 * (self.p + self.q)) if self.p.shape[0] else None

    def offer(self, starts, dirs, length, ignore=None):
        """Try candidates in order; returns the indices accepted."""
        from scipy.spatial import cKDTree
        if self.sep <= 0:
            acc = np.arange(starts.shape[0])
            self._add(starts, dirs, length)
            return acc
        m = starts.shape[0]
        P, Q, _ = self._segments(starts, dirs, length)
        mid = 0.5 * (P + Q)
        reach = CYL_LEN + self.sep
        owner = np.repeat(np.arange(m), self.ncyl)
        bad = np.zeros(m, bool)
        ign = np.full(m, -1) if ignore is None else np.asarray(ignore)
        if self.tree is not None:
            hits = self.tree.query_ball_point(mid, reach)
            rows = np.repeat(np.arange(mid.shape[0]), [len(h) for h in hits])
            cols = np.fromiter((c for h in hits for c in h), np.int64, rows.size)
            if rows.size:
                keep = self.fil[cols] != ign[owner[rows]]
                rows, cols = rows[keep], cols[keep]
                d = seg_seg_distance(P[rows], Q[rows], self.p[cols], self.q[cols])
                bad[np.unique(owner[rows[d < self.sep]])] = True
        # conflicts inside the batch: keep the earlier candidate
        pairs = cKDTree(mid).query_pairs(reach, output_type="ndarray")
        if pairs.size:
            a, b = pairs[:, 0], pairs[:, 1]
            diff = owner[a] != owner[b]
            a, b = a[diff], b[diff]
            d = seg_seg_distance(P[a], Q[a], P[b], Q[b])
            close = d < self.sep
            fa, fb = owner[a][close], owner[b][close]
            lo, hi = np.minimum(fa, fb), np.maximum(fa, fb)
            order = np.argsort(lo, kind="stable")
            for u, v in zip(lo[order], hi[order]):
                if not bad[u]:
                    bad[v] = True
        acc = np.nonzero(~bad)[0]
        self._add(starts[acc], dirs[acc], length)
        return acc

    def _add(self, starts, dirs, length):
        P, Q, _ = self._segments(starts, dirs, length)
        self.p = np.concatenate([self.p, P])
        self.q = np.concatenate([self.q, Q])
        self.fil = np.concatenate([self.fil, np.repeat(np.arange(self.n_fil, self.n_fil + starts.shape[0]), self.ncyl)])
        self.n_fil += starts.shape[0]
        self._rebuild()


def _sample_filaments(rng, placer: _Placer, n: int, ncyl: int, box: float, margin: float):
    starts = np.empty((0, 3))
    dirs = np.empty((0, 3))
    length = ncyl * CYL_LEN - 0.01
    while starts.shape[0] < n:
        m = min(max(2 * (n - starts.shape[0]), 64), 4096)
        p1 = rng.uniform(0.0, box, (m, 3))
        u = _unit_vectors(rng, m)
        p2 = p1 + length * u
        ok = _inside(p1, box, margin) & _inside(p2, box, margin)
        p1, u = p1[ok][: n - starts.shape[0]], u[ok][: n - starts.shape[0]]
        acc = placer.offer(p1, u, length)
        starts = np.concatenate([starts, p1[acc]])
        dirs = np.concatenate([dirs, u[acc]])
    return starts[:n], dirs[:n]


def _random_points_on_cylinders(rng, net_coords, b1, b2, n):
    cyl = rng.integers(0, b1.size, n)
    t = rng.uniform(0.0, 1.0, n)
    pts = net_coords[b1[cyl]] * (1.0 - t)[:, None] + net_coords[b2[cyl]] * t[:, None]
    return cyl, t, pts


def _pair_attachments(rng, coords, b1, b2, fil, n_want, dmin, dmax):
    """Random (cylinder, position) pairs on different filaments whose attachment
    points are dmin..dmax apart. A cylinder pair may carry several linkers at
    different positions, as binding sites allow in the reference."""
    from scipy.spatial import cKDTree

    if n_want <= 0:
        return np.zeros((0, 2), np.int64), np.zeros((0, 2)), np.zeros(0)
    box_vol = np.prod(coords.max(0) - coords.min(0) + 1.0)
    shell = 4.0 / 3.0 * np.pi * (dmax ** 3 - dmin ** 3)
    # expected pairs among N uniform points: N^2/2 * shell/vol; aim for ~3x n_want
    n_pts = int(np.sqrt(6.0 * n_want * box_vol / shell)) + 256
    for _ in range(12):
        cyl, t, pts = _random_points_on_cylinders(rng, coords, b1, b2, n_pts)
        pairs = cKDTree(pts).query_pairs(dmax, output_type="ndarray")
        if pairs.size:
            d = np.linalg.norm(pts[pairs[:, 0]] - pts[pairs[:, 1]], axis=1)
            ok = (d >= dmin) & (fil[cyl[pairs[:, 0]]] != fil[cyl[pairs[:, 1]]])
            pairs, d = pairs[ok], d[ok]
            if pairs.shape[0] >= n_want:
                pick = np.sort(rng.permutation(pairs.shape[0])[:n_want])
                pairs, d = pairs[pick], d[pick]
                c = np.stack([cyl[pairs[:, 0]], cyl[pairs[:, 1]]], axis=1)
                tt = np.stack([t[pairs[:, 0]], t[pairs[:, 1]]], axis=1)
                return c.astype(np.int64), tt, d
        n_pts = int(n_pts * 1.6)
    raise RuntimeError(f"could not place {n_want} attachments {dmin}-{dmax} nm apart")


def make_network(spec: NetworkSpec) -> Network:
    rng = np.random.Generator(np.random.MT19937(spec.seed))
    ncyl = spec.cyl_per_fil
    nbpf = ncyl + 1
    margin = spec.boundary_cutoff / 4.0
    n_parent = spec.n_fil - spec.n_branch
    placer = _Placer(ncyl, spec.min_separation)
    starts, dirs = _sample_filaments(rng, placer, n_parent, ncyl, spec.box, margin)
    length = ncyl * CYL_LEN - 0.01
    frac = np.arange(nbpf) / ncyl
    fil_coords = [starts[:, None, :] + (length * frac)[None, :, None] * dirs[:, None, :]]

    # Branch children: a new filament whose minus-end bead sits br_stretch_l0
    # from a point on a random parent cylinder, growing at br_bend_theta from
    # the parent's direction.
    branch_parent_cyl = np.zeros(0, np.int64)
    branch_pos = np.zeros(0)
    if spec.n_branch > 0:
        pcyl_list, ppos_list, child_list = [], [], []
        while len(child_list) < spec.n_branch:
            m = 4 * (spec.n_branch - len(child_list))
            pf = rng.integers(0, n_parent, m)
            pc = rng.integers(0, ncyl, m)
            pp = rng.uniform(0.1, 0.9, m)
            par_dir = dirs[pf]
            base = starts[pf] + (pc + pp)[:, None] * (length / ncyl) * par_dir
            # a perpendicular frame around the parent direction
            helper = np.where(np.abs(par_dir[:, :1]) < 0.9, np.array([[1.0, 0, 0]]), np.array([[0, 1.0, 0]]))
            e1 = np.cross(par_dir, helper)
            e1 /= np.linalg.norm(e1, axis=1, keepdims=True)
            e2 = np.cross(par_dir, e1)
            phi = rng.uniform(0, 2 * np.pi, m)
            perp = np.cos(phi)[:, None] * e1 + np.sin(phi)[:, None] * e2
            th = spec.br_bend_theta
            cdir = np.cos(th) * par_dir + np.sin(th) * perp
            offset = np.cos(phi + 1.0)[:, None] * e1 + np.sin(phi + 1.0)[:, None] * e2
            c0 = base + spec.br_stretch_l0 * offset
            cend = c0 + length * cdir
            ok = np.nonzero(_inside(c0, spec.box, margin) & _inside(cend, spec.box, margin))[0]
            ok = ok[: spec.n_branch - len(child_list)]
            acc = placer.offer(c0[ok], cdir[ok], length, ignore=pf[ok])
            for q in ok[acc]:
                pcyl_list.append(pf[q] * ncyl + pc[q])
                ppos_list.append(pp[q])
                child_list.append(c0[q][None, :] + (length * frac)[:, None] * cdir[q][None, :])
        fil_coords.append(np.stack(child_list))
        branch_parent_cyl = np.asarray(pcyl_list, np.int64)
        branch_pos = np.asarray(ppos_list)

    coords = np.concatenate(fil_coords).reshape(-1, 3)
    nfil = spec.n_fil
    fil_of_cyl = np.repeat(np.arange(nfil), ncyl)
    pos_of_cyl = np.tile(np.arange(ncyl), nfil)
    b1 = (fil_of_cyl * nbpf + pos_of_cyl).astype(np.int64)
    b2 = b1 + 1
    n_cyl_total = b1.size
    branching = np.full(n_cyl_total, -1, np.int64)
    child_first_cyl = (n_parent + np.arange(spec.n_branch)) * ncyl
    branching[branch_parent_cyl] = child_first_cyl

    # FilamentStretching / FilamentBending vectorization (per cylinder / per
    # consecutive cylinder pair), MCylinder constants (src/Structure/MCylinder.cpp:35-45).
    eqlen = np.full(n_cyl_total, CYL_LEN)
    kstr = spec.fstretch_k * CYL_LEN / eqlen
    kbend = spec.fbend_k * CYL_LEN / eqlen
    stretch_beads = np.stack([3 * b1, 3 * b2], axis=1)
    inner = np.nonzero(pos_of_cyl > 0)[0]
    bend_beads = np.stack([3 * b1[inner - 1], 3 * b1[inner], 3 * b2[inner]], axis=1)

    ff = dict(stretch_beads=stretch_beads, stretch_k=kstr, stretch_l0=eqlen,
              bend_beads=bend_beads, bend_k=kbend[inner], bend_theta0=np.full(inner.size, spec.fbend_theta))

    # Linkers and motors: attachment points on two cylinders of different
    # filaments (LinkerStretching::vectorize, Linker/LinkerStretching.cpp:41-54).
    cpair, tpair, dist = _pair_attachments(rng, coords, b1, b2, fil_of_cyl, spec.n_linker, *spec.linker_dist)
    if cpair.shape[0]:
        ff.update(linker_beads=np.stack([3 * b1[cpair[:, 0]], 3 * b2[cpair[:, 0]], 3 * b1[cpair[:, 1]],
                                         3 * b2[cpair[:, 1]]], axis=1),
                  linker_k=np.full(cpair.shape[0], spec.linker_k), linker_l0=dist,
                  linker_pos1=tpair[:, 0], linker_pos2=tpair[:, 1])
    mpair, mt, _ = _pair_attachments(rng, coords, b1, b2, fil_of_cyl, spec.n_motor, *spec.motor_dist)
    if mpair.shape[0]:
        ff.update(motor_beads=np.stack([3 * b1[mpair[:, 0]], 3 * b2[mpair[:, 0]], 3 * b1[mpair[:, 1]],
                                        3 * b2[mpair[:, 1]]], axis=1),
                  motor_k=np.full(mpair.shape[0], spec.motor_k),
                  motor_l0=rng.uniform(spec.motor_l0[0], spec.motor_l0[1], mpair.shape[0]),
                  motor_pos1=mt[:, 0], motor_pos2=mt[:, 1])

    if spec.n_branch > 0:
        nb = spec.n_branch
        mask = 0b0111 | (0b1000 if spec.br_position_k > 0 else 0)
        ff.update(branch_beads=np.stack([3 * b1[branch_parent_cyl], 3 * b2[branch_parent_cyl],
                                         3 * b1[child_first_cyl], 3 * b2[child_first_cyl]], axis=1),
                  branch_pos=branch_pos,
                  branch_stretch_k=np.full(nb, spec.br_stretch_k), branch_stretch_l0=np.full(nb, spec.br_stretch_l0),
                  branch_bend_k=np.full(nb, spec.br_bend_k), branch_bend_theta0=np.full(nb, spec.br_bend_theta),
                  branch_dihedral_k=np.full(nb, spec.br_dihedral_k),
                  branch_position_k=np.full(nb, spec.br_position_k), branch_ff_mask=mask)

    return Network(
        spec=spec, coords=coords,
        cyl_bead1=b1.astype(np.int32), cyl_bead2=b2.astype(np.int32), cyl_id=np.arange(n_cyl_total, dtype=np.int32),
        cyl_fil=fil_of_cyl.astype(np.int32), cyl_pos=pos_of_cyl.astype(np.int32),
        cyl_type=np.zeros(n_cyl_total, np.int32), cyl_branching=branching.astype(np.int32),
        cyl_minus_end=(pos_of_cyl == 0).astype(np.int32), cyl_eqlen=eqlen,
        cyl_exclk=np.full(n_cyl_total, spec.volume_k), ff=ff,
    )


def make_workload(index: int, seed: int | None = None, **over) -> Network:
    return make_network(workload_spec(index, seed, **over))


def batch_specs(n_replicas: int = 256, seed: int = 2, cyl_range=(200, 4000)) -> list[NetworkSpec]:
    """The batched ensemble: replicas of the medium network's composition
    (linkers 10 %, motors 1 %, branch points 1 % of the cylinders) whose
    cylinder counts are log-uniform in cyl_range, rounded to whole filaments.
    Filaments have 10 cylinders (1.08 um) so that the smallest replicas fit
    their box; the box keeps the medium network's cylinder density
    (40,000 cylinders in a 5 um cube) but is at least 1.5 um wide."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(cyl_range[0]), np.log(cyl_range[1])
    out = []
    for r in range(n_replicas):
        ncyl = int(round(float(np.exp(rng.uniform(lo, hi))) / 10.0)) * 10
        ncyl = max(ncyl, 10)
        box = max(5000.0 * (ncyl / 40000.0) ** (1.0 / 3.0), 1500.0)
        out.append(NetworkSpec(f"cfg2_replica{r}_{ncyl}cyl", ncyl // 10, 10, box, n_linker=ncyl // 10,
                               n_motor=ncyl // 100, n_branch=ncyl // 100, seed=seed * 100000 + r))
    return out


def make_batch(n_replicas: int = 256, seed: int = 2, cyl_range=(200, 4000)) -> list[Network]:
    return [make_network(s) for s in batch_specs(n_replicas, seed, cyl_range)]
