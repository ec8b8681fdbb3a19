"""ctypes mirrors of the structs in include/medyan_b200.h.

The same structs describe a force-field vectorization for the CUDA library,
for the CPU oracle and for the reference build, so one set of host arrays can
be handed to all three.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

FF_COUNT = 10
FF_NAMES = (
    "FilamentStretching",
    "FilamentBending",
    "LinkerStretching",
    "MotorGhostStretching",
    "BranchingStretching",
    "BranchingBending",
    "BranchingDihedral",
    "BranchingPosition",
    "CylinderExcludedVolume",
    "BoundaryRepulsion",
)

STATUS_NAMES = {
    0: "ok",
    1: "invalid argument",
    2: "bead index out of range",
    3: "non-finite energy or force",
    4: "iteration cap reached",
    5: "CUDA error",
    6: "cylinder outside the neighbor-list grid",
    7: "line search failed",
    8: "no CUDA device",
    9: "output buffer too small",
    10: "unsupported option",
}

PREC_FP64 = 0
PREC_MIXED = 1

CG_STEEPEST = 0
CG_FLETCHER_RIEVES = 1
CG_POLAK_RIBIERE = 2

_pi = C.POINTER(C.c_int32)
_pd = C.POINTER(C.c_double)


class MedyanSystem(C.Structure):
    _fields_ = [
        ("n_beads", C.c_int32),
        ("n_stretch", C.c_int32), ("stretch_beads", _pi), ("stretch_k", _pd), ("stretch_l0", _pd),
        ("n_bend", C.c_int32), ("bend_beads", _pi), ("bend_k", _pd), ("bend_theta0", _pd),
        ("n_linker", C.c_int32), ("linker_beads", _pi), ("linker_k", _pd), ("linker_l0", _pd),
        ("linker_pos1", _pd), ("linker_pos2", _pd),
        ("n_motor", C.c_int32), ("motor_beads", _pi), ("motor_k", _pd), ("motor_l0", _pd),
        ("motor_pos1", _pd), ("motor_pos2", _pd),
        ("n_branch", C.c_int32), ("branch_beads", _pi), ("branch_pos", _pd),
        ("branch_stretch_k", _pd), ("branch_stretch_l0", _pd), ("branch_bend_k", _pd),
        ("branch_bend_theta0", _pd), ("branch_dihedral_k", _pd), ("branch_position_k", _pd),
        ("branch_ff_mask", C.c_int32),
        ("n_excl", C.c_int32), ("excl_beads", _pi), ("excl_k", _pd), ("excl_eqlen", _pd),
        ("n_boundary", C.c_int32), ("boundary_beads", _pi), ("boundary_k", _pd), ("boundary_slen", _pd),
        ("n_planes", C.c_int32), ("plane_eq", _pd), ("plane_nneighbors", _pi),
    ]


class CGParams(C.Structure):
    _fields_ = [
        ("method", C.c_int32),
        ("max_dist", C.c_double),
        ("lambda_max", C.c_double),
        ("grad_tol", C.c_double),
        ("energy_rel_tol", C.c_double),
        ("energy_call_limit", C.c_int32),
        ("force_call_limit", C.c_int32),
        ("try_to_recover", C.c_int32),
        ("line_search", C.c_int32),
    ]


class MinResult(C.Structure):
    _fields_ = [
        ("energy_before", C.c_double * FF_COUNT),
        ("energy_before_total", C.c_double),
        ("energy_after", C.c_double * FF_COUNT),
        ("energy_after_total", C.c_double),
        ("error_flags", C.c_uint32),
        ("num_energy_call", C.c_int32),
        ("energy_call_limit", C.c_int32),
        ("num_force_call", C.c_int32),
        ("force_call_limit", C.c_int32),
        ("num_iter", C.c_int32),
        ("grad_inf_norm", C.c_double),
        ("grad_tol", C.c_double),
        ("energy_rel_change", C.c_double),
        ("energy_rel_tol", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {
            "energy_before": list(self.energy_before),
            "energy_before_total": self.energy_before_total,
            "energy_after": list(self.energy_after),
            "energy_after_total": self.energy_after_total,
            "error_flags": self.error_flags,
            "num_energy_call": self.num_energy_call,
            "num_force_call": self.num_force_call,
            "force_call_limit": self.force_call_limit,
            "num_iter": self.num_iter,
            "grad_inf_norm": self.grad_inf_norm,
            "energy_rel_change": self.energy_rel_change,
        }


class MedyanCylinders(C.Structure):
    _fields_ = [
        ("n_cyl", C.c_int32),
        ("bead1", _pi), ("bead2", _pi), ("id", _pi), ("filament_id", _pi),
        ("position_on_filament", _pi), ("type", _pi), ("branching_cylinder", _pi),
        ("is_minus_end", _pi), ("eq_length", _pd), ("excl_k", _pd),
    ]


class LaunchShapes(C.Structure):
    _fields_ = [("bonded_threads", C.c_int32), ("excl_threads", C.c_int32), ("chain_threads", C.c_int32),
                ("chain_energy_blocks_per_sm", C.c_int32), ("pass_layout", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchShapes(C.Structure):
    _fields_ = [("bonded_threads", C.c_int32), ("excl_threads", C.c_int32), ("chain_threads", C.c_int32),
                ("chain_chunk", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class LoadTips(C.Structure):
    _fields_ = [("n_tips", C.c_int32), ("cylinder", _pi), ("plus_end", _pi), ("n_mon", _pi), ("mon_size", _pd)]


class NLParams(C.Structure):
    _fields_ = [("rmax", C.c_float), ("rmin", C.c_float), ("grid_size", C.c_double * 3)]


class BoundaryParams(C.Structure):
    _fields_ = [
        ("n_planes", C.c_int32),
        ("plane_eq", _pd),
        ("k", C.c_double),
        ("screen_length", C.c_double),
        ("cutoff", C.c_float),
    ]


def _ptr(a: np.ndarray | None, ctype):
    if a is None or a.size == 0:
        return C.cast(None, C.POINTER(ctype))
    return a.ctypes.data_as(C.POINTER(ctype))


def i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(-1))


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))


class SystemView:
    """Owns contiguous copies of a force-field vectorization and exposes it as
    a MedyanSystem struct. Keep the view alive while the struct is in use."""

    _INT_FIELDS = ("stretch_beads", "bend_beads", "linker_beads", "motor_beads", "branch_beads",
                   "excl_beads", "boundary_beads", "plane_nneighbors")

    def __init__(self, n_beads: int, **arrays):
        self.n_beads = int(n_beads)
        self.arrays = {}
        for k, v in arrays.items():
            if v is None or k == "branch_ff_mask":
                continue
            self.arrays[k] = i32(v) if k in self._INT_FIELDS else f64(v)
        self.branch_ff_mask = int(arrays.get("branch_ff_mask", 0) or 0)
        self.struct = self._make()

    def count(self, name: str, per: int) -> int:
        a = self.arrays.get(name)
        return 0 if a is None else a.size // per

    def _make(self) -> MedyanSystem:
        s = MedyanSystem()
        s.n_beads = self.n_beads
        a = self.arrays
        for name, arr in a.items():
            setattr(s, name, _ptr(arr, C.c_int32 if name in self._INT_FIELDS else C.c_double))
        s.n_stretch = self.count("stretch_beads", 2)
        s.n_bend = self.count("bend_beads", 3)
        s.n_linker = self.count("linker_beads", 4)
        s.n_motor = self.count("motor_beads", 4)
        s.n_branch = self.count("branch_beads", 4)
        s.branch_ff_mask = self.branch_ff_mask
        s.n_excl = self.count("excl_beads", 4)
        s.n_boundary = self.count("boundary_beads", 1)
        s.n_planes = self.count("plane_eq", 4)
        return s

    def ref(self):
        return C.byref(self.struct)


class CylindersView:
    """Contiguous cylinder topology exposed as MedyanCylinders."""

    def __init__(self, bead1, bead2, cid, filament_id, position, ctype, branching, minus_end, eq_length, excl_k):
        self.arrays = dict(
            bead1=i32(bead1), bead2=i32(bead2), id=i32(cid), filament_id=i32(filament_id),
            position_on_filament=i32(position), type=i32(ctype), branching_cylinder=i32(branching),
            is_minus_end=i32(minus_end), eq_length=f64(eq_length), excl_k=f64(excl_k),
        )
        s = MedyanCylinders()
        s.n_cyl = self.arrays["bead1"].size
        for k, v in self.arrays.items():
            setattr(s, k, _ptr(v, C.c_double if v.dtype == np.float64 else C.c_int32))
        self.struct = s

    def ref(self):
        return C.byref(self.struct)
