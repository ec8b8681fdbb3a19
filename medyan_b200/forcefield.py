"""Host-side mirror of the reference's ForceFieldManager and CGMethod
interfaces over the CUDA library.

``ForceFieldManager`` follows src/Mechanics/ForceField/ForceFieldManager.h:48-216:
``vectorize_all_force_fields`` hands the per-force-field arrays to the device,
``compute_energy`` returns the total (``inf`` when a force field fails, as
ForceFieldManager.cpp:150-161 does), ``compute_individual_energies`` returns
the per-force-field report, ``compute_forces`` returns -dE/dx.
``minimize`` is CGMethod::minimize (src/Mechanics/Minimizer/CGMethod.hpp:826)
run entirely on the device.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import lib as L
from ._abi import (FF_COUNT, FF_NAMES, PREC_FP64, PREC_MIXED, CGParams, MinResult, SystemView, f64)

_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int32)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_pd)


@dataclass
class EnergyReport:
    """EnergyReport (src/Mechanics/ForceField/Types.hpp:24-33)."""
    total: float
    individual: list  # [(name, energy)]

    def as_array(self) -> np.ndarray:
        return np.array([e for _, e in self.individual])


def conjugate_gradient_params(method: int = 2, max_dist: float = 1.0, lambda_max: float = 0.01,
                              grad_tol: float = 1.0, energy_rel_tol: float = 1e-9, energy_call_limit: int = 0,
                              force_call_limit: int = 10000, try_to_recover: bool = True,
                              line_search: str = "BACKTRACKING") -> CGParams:
    """ConjugateGradientParams (CGMethod.hpp:44-63); defaults are the
    reference example's MAXDISTANCE/LAMBDAMAX and MechParams' tolerances.
    line_search: "BACKTRACKING" or "QUADRATIC" (quadraticLineSearchV2)."""
    p = CGParams()
    p.method = method
    p.max_dist = max_dist
    p.lambda_max = lambda_max
    p.grad_tol = grad_tol
    p.energy_rel_tol = energy_rel_tol
    p.energy_call_limit = energy_call_limit
    p.force_call_limit = force_call_limit
    p.try_to_recover = 1 if try_to_recover else 0
    p.line_search = {"BACKTRACKING": 0, "QUADRATIC": 1}[line_search]
    return p


class ForceFieldManager:
    def __init__(self, precision: str = "fp64"):
        self.lib = L.load()
        self.precision = {"fp64": PREC_FP64, "mixed": PREC_MIXED}[precision]
        self.handle = C.c_void_p()
        self.n_beads = 0
        self._system = None
        self._cyl = None

    # -- vectorization -----------------------------------------------------
    def vectorize_all_force_fields(self, system: SystemView) -> None:
        self._system = system
        if not self.handle:
            h = C.c_void_p()
            L.check(self.lib.medyan_mech_create(system.ref(), self.precision, C.byref(h)), "medyan_mech_create")
            self.handle = h
            self.n_beads = system.n_beads
        else:
            L.check(self.lib.medyan_mech_update(self.handle, system.ref()), "medyan_mech_update")

    # -- energy / forces ---------------------------------------------------
    def set_coords(self, coord) -> None:
        x = f64(coord)
        assert x.size == 3 * self.n_beads
        L.check(self.lib.medyan_mech_set_coords(self.handle, _dp(x)), "medyan_mech_set_coords")

    def get_coords(self) -> np.ndarray:
        x = np.zeros(3 * self.n_beads)
        L.check(self.lib.medyan_mech_get_coords(self.handle, _dp(x)), "medyan_mech_get_coords")
        return x

    def _energy(self):
        tot = C.c_double(0.0)
        per = np.zeros(FF_COUNT)
        st = self.lib.medyan_mech_energy(self.handle, C.byref(tot), _dp(per))
        if st not in (0, 3):
            L.check(st, "medyan_mech_energy")
        return tot.value, per

    def compute_energy(self, coord=None) -> float:
        if coord is not None:
            self.set_coords(coord)
        return self._energy()[0]

    def compute_individual_energies(self, coord=None) -> EnergyReport:
        if coord is not None:
            self.set_coords(coord)
        _, per = self._energy()
        return EnergyReport(total=float(np.sum(per)), individual=list(zip(FF_NAMES, per.tolist())))

    def compute_forces(self, coord=None) -> np.ndarray:
        if coord is not None:
            self.set_coords(coord)
        f = np.zeros(3 * self.n_beads)
        L.check(self.lib.medyan_mech_forces(self.handle, _dp(f)), "medyan_mech_forces")
        return f

    def evaluate(self, coord):
        """Energy, per-force-field energies and forces at coord in one call."""
        x = f64(coord)
        f = np.zeros_like(x)
        tot = C.c_double(0.0)
        per = np.zeros(FF_COUNT)
        st = self.lib.medyan_mech_evaluate(self.handle, _dp(x), C.byref(tot), _dp(per), _dp(f))
        if st not in (0, 3):
            L.check(st, "medyan_mech_evaluate")
        return tot.value, per, f

    def set_deterministic(self, on: bool = True) -> None:
        """Fixed-point force sums: bitwise reproducible forces and minimizations."""
        L.check(self.lib.medyan_mech_set_deterministic(self.handle, 1 if on else 0), "medyan_mech_set_deterministic")

    def evaluate_many(self, coords):
        """Energies and forces at each coordinate set of coords (a list of
        arrays) through the asynchronous double-buffered entry point; returns
        (energies [n, FF_COUNT + 1], forces list). The host buffers are
        page-locked so that the copies overlap."""
        import torch
        n3 = 3 * self.n_beads
        xs = [torch.from_numpy(f64(c).copy()).pin_memory() for c in coords]
        fs = [torch.empty(n3, dtype=torch.float64).pin_memory() for _ in coords]
        es = torch.empty((len(coords), FF_COUNT + 1), dtype=torch.float64).pin_memory()
        pd = C.POINTER(C.c_double)
        for i in range(len(coords)):
            L.check(self.lib.medyan_mech_evaluate_async(
                self.handle, C.cast(xs[i].data_ptr(), pd), C.cast(fs[i].data_ptr(), pd),
                C.cast(es[i].data_ptr(), pd)), "medyan_mech_evaluate_async")
        st = self.lib.medyan_mech_wait(self.handle)
        if st not in (0, 3):
            L.check(st, "medyan_mech_wait")
        return es.numpy().copy(), [f.numpy().copy() for f in fs]

    # -- minimizer ---------------------------------------------------------
    def minimize(self, coord, params: CGParams):
        """CGMethod::minimize on the device. Returns (status, coord, force, MinResult)."""
        x = f64(coord).copy()
        f = np.zeros_like(x)
        r = MinResult()
        st = self.lib.medyan_cg_minimize(self.handle, C.byref(params), _dp(x), _dp(f), C.byref(r))
        if st not in (0, 7):
            L.check(st, "medyan_cg_minimize")
        return st, x, f, r

    # -- derivatives -------------------------------------------------------
    def param_grad(self, ff_slot: int, n: int, v=None):
        """(dE/dk, dE/dp) per interaction of force field ff_slot at the
        current coordinates; with v, their derivative along v."""
        dk = np.zeros(max(n, 1))
        dp = np.zeros(max(n, 1))
        vv = f64(v) if v is not None else None
        L.check(self.lib.medyan_mech_param_grad(self.handle, ff_slot, _dp(vv) if vv is not None else None, _dp(dk),
                                                _dp(dp), n), "medyan_mech_param_grad")
        return dk[:n], dp[:n]

    def hvp(self, v) -> np.ndarray:
        """Hessian of the total energy at the current coordinates times v."""
        vv = f64(v)
        hv = np.zeros_like(vv)
        st = self.lib.medyan_mech_hvp(self.handle, _dp(vv), _dp(hv))
        if st not in (0, 3):
            L.check(st, "medyan_mech_hvp")
        return hv

    def hessian(self, delta: float = 1e-4) -> np.ndarray:
        """ForceFieldManager::computeHessian (ForceFieldManager.cpp:354-398):
        the dense finite-difference Hessian at the current coordinates,
        H[i, j] = float(-(F_j(x + delta e_i) - F_j(x - delta e_i)) / (2 delta))."""
        n = 3 * self.n_beads
        H = np.zeros((n, n))
        st = self.lib.medyan_mech_hessian(self.handle, C.c_float(delta), _dp(H))
        if st not in (0, 3):
            L.check(st, "medyan_mech_hessian")
        return H

    # -- launch shapes ----------------------------------------------------
    def get_shapes(self) -> dict:
        from ._abi import LaunchShapes
        sh = LaunchShapes()
        L.check(self.lib.medyan_mech_get_shapes(self.handle, C.byref(sh)), "medyan_mech_get_shapes")
        return sh.as_dict()

    def set_shapes(self, **shapes) -> None:
        """Block/tile shapes per potential (medyan_launch_shapes); fields not
        given keep their current values."""
        from ._abi import LaunchShapes
        cur = self.get_shapes()
        cur.update(shapes)
        sh = LaunchShapes(**cur)
        L.check(self.lib.medyan_mech_set_shapes(self.handle, C.byref(sh)), "medyan_mech_set_shapes")

    def autotune(self, reps: int = 10) -> dict:
        """Times the evaluate pass per candidate shape and keeps the fastest."""
        from ._abi import LaunchShapes
        sh = LaunchShapes()
        L.check(self.lib.medyan_mech_autotune(self.handle, reps, C.byref(sh)), "medyan_mech_autotune")
        return sh.as_dict()

    # -- after a minimization --------------------------------------------
    def force_magnitudes(self):
        """ForceFieldManager::assignallforcemags inputs at the current
        coordinates: (linker tensions k(L - l0), motor tensions, branch-point
        forces [n_branch, 3])."""
        sv = self._system
        n = (sv.count("linker_beads", 4), sv.count("motor_beads", 4), sv.count("branch_beads", 4))
        lin, mot, br = np.zeros(max(n[0], 1)), np.zeros(max(n[1], 1)), np.zeros(max(3 * n[2], 1))
        L.check(self.lib.medyan_mech_force_magnitudes(self.handle, _dp(lin), _dp(mot), _dp(br)),
                "medyan_mech_force_magnitudes")
        return lin[: n[0]], mot[: n[1]], br[: 3 * n[2]].reshape(-1, 3)

    def boundary_load_forces(self, cylinder, plus_end, n_mon, mon_size):
        """BoundaryCylinderRepulsion::computeLoadForces on filament tips:
        one array of n_mon[t] loads per tip (cylinder indices into the list
        given to set_cylinders)."""
        from ._abi import LoadTips
        cyl = np.ascontiguousarray(cylinder, np.int32)
        plus = np.ascontiguousarray(plus_end, np.int32)
        nm = np.ascontiguousarray(n_mon, np.int32)
        ms = f64(mon_size)
        total = int(nm.sum())
        out = np.zeros(max(total, 1))
        tips = LoadTips(len(cyl), cyl.ctypes.data_as(_pi), plus.ctypes.data_as(_pi), nm.ctypes.data_as(_pi),
                        ms.ctypes.data_as(_pd))
        L.check(self.lib.medyan_mech_boundary_load_forces(self.handle, C.byref(tips), _dp(out), total),
                "medyan_mech_boundary_load_forces")
        return np.split(out[:total], np.cumsum(nm)[:-1])

    # -- neighbor lists ----------------------------------------------------
    def set_cylinders(self, cylinders, nl_params, boundary_params) -> None:
        self._cyl = (cylinders, nl_params, boundary_params)
        L.check(self.lib.medyan_mech_set_cylinders(self.handle, cylinders.ref(), C.byref(nl_params),
                                                   C.byref(boundary_params) if boundary_params is not None else None),
                "medyan_mech_set_cylinders")

    def rebuild_neighbor_lists(self) -> tuple[int, int]:
        ne = C.c_int64(0)
        nb = C.c_int64(0)
        L.check(self.lib.medyan_mech_rebuild_neighbors(self.handle, C.byref(ne), C.byref(nb)),
                "medyan_mech_rebuild_neighbors")
        return ne.value, nb.value

    def excluded_volume_interactions(self):
        n = C.c_int64(0)
        L.check(self.lib.medyan_mech_get_excl_volume(self.handle, None, None, None, 0, C.byref(n)),
                "medyan_mech_get_excl_volume")
        m = n.value
        beads = np.zeros(4 * max(m, 1), np.int32)
        k = np.zeros(max(m, 1))
        eq = np.zeros(2 * max(m, 1))
        L.check(self.lib.medyan_mech_get_excl_volume(self.handle, beads.ctypes.data_as(_pi), _dp(k), _dp(eq), m,
                                                     C.byref(n)), "medyan_mech_get_excl_volume")
        return beads[: 4 * m].reshape(-1, 4), k[:m], eq[: 2 * m].reshape(-1, 2)

    # -- lifetime ----------------------------------------------------------
    def close(self) -> None:
        if self.handle:
            self.lib.medyan_mech_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class BatchMinimizer:
    """Independent networks minimized together (medyan_batch_*): every
    replica's minimization is enqueued before any is awaited, so they run
    concurrently on the device, each to its own convergence."""

    def __init__(self, systems: list, precision: str = "fp64"):
        self.lib = L.load()
        self.precision = {"fp64": PREC_FP64, "mixed": PREC_MIXED}[precision]
        self._systems = list(systems)
        arr = (type(self._systems[0].struct) * len(self._systems))(*[sv.struct for sv in self._systems]) \
            if self._systems else None
        self.handle = C.c_void_p()
        L.check(self.lib.medyan_batch_create(arr, len(self._systems), self.precision, C.byref(self.handle)),
                "medyan_batch_create")
        self.n = len(self._systems)

    def get_shapes(self) -> dict:
        from ._abi import BatchShapes
        sh = BatchShapes()
        L.check(self.lib.medyan_batch_get_shapes(self.handle, C.byref(sh)), "medyan_batch_get_shapes")
        return sh.as_dict()

    def set_shapes(self, **shapes) -> None:
        """Packed-layout shapes (medyan_batch_shapes); fields not given keep their values."""
        from ._abi import BatchShapes
        cur = self.get_shapes()
        cur.update(shapes)
        L.check(self.lib.medyan_batch_set_shapes(self.handle, C.byref(BatchShapes(**cur))), "medyan_batch_set_shapes")

    def autotune(self, reps: int = 5) -> dict:
        """Times packed evaluate passes at the replicas' current coordinates per candidate
        shape and keeps the fastest (set each replica's coordinates first)."""
        from ._abi import BatchShapes
        sh = BatchShapes()
        L.check(self.lib.medyan_batch_autotune(self.handle, reps, C.byref(sh)), "medyan_batch_autotune")
        return sh.as_dict()

    def set_deterministic(self, on: bool = True) -> None:
        """Fixed-point force sums for the packed minimizer and every replica
        (medyan_batch_set_deterministic): bitwise reproducible batches."""
        L.check(self.lib.medyan_batch_set_deterministic(self.handle, 1 if on else 0),
                "medyan_batch_set_deterministic")

    def replica(self, r: int) -> C.c_void_p:
        """The handle of replica r (for set_cylinders / rebuild_neighbors)."""
        return C.c_void_p(self.lib.medyan_batch_replica(self.handle, r))

    def rebuild_neighbor_lists(self, r: int, coord, cylinders, nl_params, boundary_params) -> tuple[int, int]:
        h = self.replica(r)
        x = f64(coord)
        L.check(self.lib.medyan_mech_set_coords(h, _dp(x)), "medyan_mech_set_coords")
        L.check(self.lib.medyan_mech_set_cylinders(h, cylinders.ref(), C.byref(nl_params),
                                                   C.byref(boundary_params) if boundary_params is not None else None),
                "medyan_mech_set_cylinders")
        ne, nb = C.c_int64(0), C.c_int64(0)
        L.check(self.lib.medyan_mech_rebuild_neighbors(h, C.byref(ne), C.byref(nb)), "medyan_mech_rebuild_neighbors")
        return ne.value, nb.value

    def minimize(self, coords: list, params: CGParams):
        """Returns (statuses, coords, forces, results) per replica."""
        xs = [f64(x).copy() for x in coords]
        fs = [np.zeros_like(x) for x in xs]
        xp = (_pd * self.n)(*[_dp(x) for x in xs])
        fp = (_pd * self.n)(*[_dp(f) for f in fs])
        res = (MinResult * self.n)()
        st = (C.c_int32 * self.n)()
        top = self.lib.medyan_batch_minimize(self.handle, C.byref(params), xp, fp, res, st)
        if top != 0:
            L.check(top, "medyan_batch_minimize")
        return list(st), xs, fs, list(res)

    def evaluate(self, coords: list):
        """Total energies and forces of every replica."""
        xs = [f64(x) for x in coords]
        fs = [np.zeros_like(x) for x in xs]
        xp = (_pd * self.n)(*[_dp(x) for x in xs])
        fp = (_pd * self.n)(*[_dp(f) for f in fs])
        e = np.zeros(self.n)
        st = self.lib.medyan_batch_evaluate(self.handle, xp, _dp(e), fp)
        if st not in (0, 3):
            L.check(st, "medyan_batch_evaluate")
        return e, fs

    def close(self) -> None:
        if self.handle:
            self.lib.medyan_batch_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def neighbor_pairs(cylinders, coord, n_beads: int, nl_params) -> np.ndarray:
    """medyan_nl_build: canonical (key, neighbor) cylinder-index pairs."""
    lib = L.load()
    x = f64(coord)
    n = C.c_int64(0)
    L.check(lib.medyan_nl_build(cylinders.ref(), _dp(x), n_beads, C.byref(nl_params), None, 0, C.byref(n)),
            "medyan_nl_build")
    pairs = np.zeros(2 * max(n.value, 1), np.int32)
    L.check(lib.medyan_nl_build(cylinders.ref(), _dp(x), n_beads, C.byref(nl_params), pairs.ctypes.data_as(_pi),
                                n.value, C.byref(n)), "medyan_nl_build")
    return pairs[: 2 * n.value].reshape(-1, 2)


@dataclass
class HessianModes:
    """The eigenmode analysis of ForceFieldManager::computeHessian
    (ForceFieldManager.cpp:400-480): eigenvalues in ascending order, the
    eigenvectors as columns, and the two participation ratios per mode,
    IPRI = sum_i v_i^4 and IPRII = sum_beads (sum_k v_{3b+k}^2)^2."""
    evalues: np.ndarray
    evectors: np.ndarray
    IPRI: np.ndarray
    IPRII: np.ndarray


def hessian_modes(H: np.ndarray) -> HessianModes:
    """Symmetrize 0.5 (H^T + H) and take its full eigendecomposition (the
    reference's dense branch, SelfAdjointEigenSolver; its sparse branch asks
    Spectra for the ndof - 1 smallest, the first ndof - 1 of these), then the
    participation ratios. The eigensolve runs on the GPU through torch when
    one is present."""
    Hs = 0.5 * (H.T + H)
    try:
        import torch
        if torch.cuda.is_available():
            w, v = torch.linalg.eigh(torch.from_numpy(Hs).cuda())
            w, v = w.cpu().numpy(), v.cpu().numpy()
        else:
            w, v = np.linalg.eigh(Hs)
    except ImportError:
        w, v = np.linalg.eigh(Hs)
    sq = v * v
    ipri = np.sum(sq * sq, axis=0)
    per_bead = sq.reshape(-1, 3, sq.shape[1]).sum(axis=1)
    iprii = np.sum(per_bead * per_bead, axis=0)
    return HessianModes(w, v, ipri, iprii)
