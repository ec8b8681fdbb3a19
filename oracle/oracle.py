"""ctypes access to the CPU checkers. TEST INFRASTRUCTURE ONLY.

- ``Oracle``: the plain-C restatement (oracle/libmedyan_oracle.so).
- ``Reference``: the reference's own potential and CG sources compiled by
  ``make -C oracle ref`` (oracle/_ref/libmedyan_ref.so), when present.

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py use
this module; the product path never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from medyan_b200._abi import (FF_COUNT, CGParams, MinResult, SystemView, f64, i32)

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libmedyan_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmedyan_ref.so")
REF_STRICT_SO = os.path.join(HERE, "_ref", "libmedyan_ref_strict.so")

_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int32)


def build_oracle() -> str:
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return ORACLE_SO


def _dp(a):
    return a.ctypes.data_as(_pd)


def _ip(a):
    return a.ctypes.data_as(_pi)


class Oracle:
    def __init__(self):
        self.lib = C.CDLL(build_oracle())
        L = self.lib
        L.oracle_energy.restype = C.c_double
        L.oracle_energy.argtypes = [C.c_void_p, _pd, _pd]
        L.oracle_forces.restype = None
        L.oracle_forces.argtypes = [C.c_void_p, _pd, _pd]
        L.oracle_cg_minimize.restype = C.c_int32
        L.oracle_cg_minimize.argtypes = [C.c_void_p, C.c_void_p, _pd, _pd, C.c_void_p]
        L.oracle_nl_build.restype = C.c_int32
        L.oracle_nl_build.argtypes = [C.c_void_p, _pd, C.c_int32, C.c_void_p, _pi, C.c_int64,
                                      C.POINTER(C.c_int64)]
        L.oracle_excl_vectorize.restype = C.c_int64
        L.oracle_excl_vectorize.argtypes = [C.c_void_p, _pi, C.c_int64, _pi, _pd, _pd]
        L.oracle_boundary_vectorize.restype = C.c_int64
        L.oracle_boundary_vectorize.argtypes = [C.c_void_p, _pd, C.c_void_p, _pi, _pd, _pd, _pi]
        L.oracle_force_magnitudes.restype = None
        L.oracle_force_magnitudes.argtypes = [C.c_void_p, _pd, _pd, _pd, _pd]
        L.oracle_boundary_load_forces.restype = None
        L.oracle_boundary_load_forces.argtypes = [C.c_void_p, _pd, C.c_void_p, C.c_int32, _pi, _pi, _pi, _pd, _pd]
        L.oracle_hessian.restype = None
        L.oracle_hessian.argtypes = [C.c_void_p, _pd, C.c_float, _pd]
        L.oracle_excl_pair_energy.restype = C.c_double
        L.oracle_excl_pair_energy.argtypes = [_pd, _pd, _pd, _pd, C.c_double]

    # ForceFieldManager semantics
    def energy(self, sv: SystemView, x: np.ndarray):
        x = f64(x)
        e = np.zeros(FF_COUNT)
        tot = self.lib.oracle_energy(sv.ref(), _dp(x), _dp(e))
        return tot, e

    def forces(self, sv: SystemView, x: np.ndarray) -> np.ndarray:
        x = f64(x)
        f = np.zeros_like(x)
        self.lib.oracle_forces(sv.ref(), _dp(x), _dp(f))
        return f

    def minimize(self, sv: SystemView, x: np.ndarray, params: CGParams):
        x = f64(x).copy()
        f = np.zeros_like(x)
        r = MinResult()
        st = self.lib.oracle_cg_minimize(sv.ref(), C.byref(params), _dp(x), _dp(f), C.byref(r))
        return st, x, f, r

    def force_magnitudes(self, sv: SystemView, x: np.ndarray):
        x = f64(x)
        nl, nm, nb = sv.count("linker_beads", 4), sv.count("motor_beads", 4), sv.count("branch_beads", 4)
        lin, mot, br = np.zeros(max(nl, 1)), np.zeros(max(nm, 1)), np.zeros(max(3 * nb, 1))
        self.lib.oracle_force_magnitudes(sv.ref(), _dp(x), _dp(lin), _dp(mot), _dp(br))
        return lin[:nl], mot[:nm], br[: 3 * nb].reshape(-1, 3)

    def boundary_load_forces(self, cyl_view, x, bparams, cylinder, plus_end, n_mon, mon_size):
        x = f64(x)
        cyl = i32(cylinder)
        plus = i32(plus_end)
        nm = i32(n_mon)
        ms = f64(mon_size)
        out = np.zeros(max(int(nm.sum()), 1))
        self.lib.oracle_boundary_load_forces(cyl_view.ref(), _dp(x), C.byref(bparams), len(cyl), _ip(cyl), _ip(plus),
                                             _ip(nm), _dp(ms), _dp(out))
        return np.split(out[: int(nm.sum())], np.cumsum(nm)[:-1])

    def hessian(self, sv: SystemView, x: np.ndarray, delta: float) -> np.ndarray:
        x = f64(x)
        n = x.size
        H = np.zeros((n, n))
        self.lib.oracle_hessian(sv.ref(), _dp(x), C.c_float(delta), _dp(H))
        return H

    def neighbor_pairs(self, cyl_view, x: np.ndarray, n_beads: int, nl_params) -> tuple[int, np.ndarray]:
        x = f64(x)
        n = C.c_int64(0)
        st = self.lib.oracle_nl_build(cyl_view.ref(), _dp(x), n_beads, C.byref(nl_params), None, 0, C.byref(n))
        if st != 0:
            return st, np.zeros((0, 2), np.int32)
        pairs = np.zeros(2 * max(n.value, 1), np.int32)
        st = self.lib.oracle_nl_build(cyl_view.ref(), _dp(x), n_beads, C.byref(nl_params), _ip(pairs),
                                      pairs.size // 2, C.byref(n))
        return st, pairs[: 2 * n.value].reshape(-1, 2)

    def excl_vectorize(self, cyl_view, pairs: np.ndarray):
        p = i32(pairs)
        m = self.lib.oracle_excl_vectorize(cyl_view.ref(), _ip(p), p.size // 2, None, None, None)
        beads = np.zeros(4 * max(m, 1), np.int32)
        k = np.zeros(max(m, 1))
        eq = np.zeros(2 * max(m, 1))
        self.lib.oracle_excl_vectorize(cyl_view.ref(), _ip(p), p.size // 2, _ip(beads), _dp(k), _dp(eq))
        return beads[: 4 * m].reshape(-1, 4), k[:m], eq[: 2 * m].reshape(-1, 2)

    def boundary_vectorize(self, cyl_view, x: np.ndarray, bparams):
        x = f64(x)
        m = self.lib.oracle_boundary_vectorize(cyl_view.ref(), _dp(x), C.byref(bparams), None, None, None, None)
        beads = np.zeros(max(m, 1), np.int32)
        k = np.zeros(max(m, 1))
        sl = np.zeros(max(m, 1))
        nn = np.zeros(max(bparams.n_planes, 1), np.int32)
        self.lib.oracle_boundary_vectorize(cyl_view.ref(), _dp(x), C.byref(bparams), _ip(beads), _dp(k), _dp(sl),
                                           _ip(nn))
        return beads[:m], k[:m], sl[:m], nn[: bparams.n_planes]

    def complete(self, net) -> tuple[int, dict]:
        """Fill a network's excluded-volume and boundary arrays with the oracle's
        neighbor lists. Returns (status, extra arrays for SystemView)."""
        cv = net.cylinders_view()
        st, pairs = self.neighbor_pairs(cv, net.flat_coords(), net.n_beads, net.nl_params())
        if st != 0:
            return st, {}
        eb, ek, el = self.excl_vectorize(cv, pairs)
        bp, planes = net.boundary_params()
        bb, bk, bs, nn = self.boundary_vectorize(cv, net.flat_coords(), bp)
        return 0, dict(excl_beads=eb, excl_k=ek, excl_eqlen=el, boundary_beads=bb, boundary_k=bk,
                       boundary_slen=bs, plane_eq=planes, plane_nneighbors=nn)


class Reference:
    """The reference's compiled kernels (oracle/_ref/libmedyan_ref.so)."""

    @staticmethod
    def available(strict: bool = False) -> bool:
        return os.path.exists(REF_STRICT_SO if strict else REF_SO)

    def __init__(self, strict: bool = False):
        """strict=False: reference flags (-O2 -ffast-math); strict=True: the
        same sources rounded as written, which the oracle matches bit for bit."""
        self.lib = C.CDLL(REF_STRICT_SO if strict else REF_SO)
        L = self.lib
        L.medyan_ref_energy.restype = C.c_double
        L.medyan_ref_energy.argtypes = [C.c_void_p, _pd, _pd]
        L.medyan_ref_forces.restype = None
        L.medyan_ref_forces.argtypes = [C.c_void_p, _pd, _pd]
        L.medyan_ref_prepare.restype = C.c_void_p
        L.medyan_ref_prepare.argtypes = [C.c_void_p]
        L.medyan_ref_release.argtypes = [C.c_void_p]
        L.medyan_ref_prepared_energy.restype = C.c_double
        L.medyan_ref_prepared_energy.argtypes = [C.c_void_p, _pd, _pd]
        L.medyan_ref_prepared_forces.restype = None
        L.medyan_ref_prepared_forces.argtypes = [C.c_void_p, _pd, _pd]
        L.medyan_ref_cg_minimize.restype = C.c_int
        L.medyan_ref_cg_minimize.argtypes = [C.c_void_p, C.c_void_p, _pd, _pd, C.c_void_p]

    def energy(self, sv: SystemView, x):
        x = f64(x)
        e = np.zeros(FF_COUNT)
        tot = self.lib.medyan_ref_energy(sv.ref(), _dp(x), _dp(e))
        return tot, e

    def forces(self, sv: SystemView, x):
        x = f64(x)
        f = np.zeros_like(x)
        self.lib.medyan_ref_forces(sv.ref(), _dp(x), _dp(f))
        return f

    def minimize(self, sv: SystemView, x, params: CGParams):
        x = f64(x).copy()
        f = np.zeros_like(x)
        r = MinResult()
        st = self.lib.medyan_ref_cg_minimize(sv.ref(), C.byref(params), _dp(x), _dp(f), C.byref(r))
        return st, x, f, r


def cg_params(method=2, max_dist=1.0, lambda_max=0.01, grad_tol=1.0, energy_rel_tol=1e-9, energy_call_limit=0,
              force_call_limit=10000, try_to_recover=1, line_search=0) -> CGParams:
    p = CGParams()
    p.line_search = line_search
    p.method = method
    p.max_dist = max_dist
    p.lambda_max = lambda_max
    p.grad_tol = grad_tol
    p.energy_rel_tol = energy_rel_tol
    p.energy_call_limit = energy_call_limit
    p.force_call_limit = force_call_limit
    p.try_to_recover = try_to_recover
    return p
