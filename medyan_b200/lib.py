"""Loader for the CUDA library (medyan_b200/libmedyan_b200.so) with ctypes
prototypes for every entry point of include/medyan_b200.h.

There is no fallback: if the shared library is missing or no CUDA device is
visible, calls raise. Build it with ``python -m medyan_b200.build``.
"""
from __future__ import annotations

import ctypes as C
import os

from ._abi import STATUS_NAMES

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmedyan_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "medyan_b200.h")

_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int32)
_pi64 = C.POINTER(C.c_int64)
_vp = C.c_void_p

# name -> (restype, argtypes)
PROTOTYPES = {
    "medyan_abi_version": (C.c_int32, []),
    "medyan_status_string": (C.c_char_p, [C.c_int32]),
    "medyan_last_cuda_error": (C.c_char_p, []),
    "medyan_mech_create": (C.c_int32, [_vp, C.c_int32, C.POINTER(_vp)]),
    "medyan_mech_update": (C.c_int32, [_vp, _vp]),
    "medyan_mech_destroy": (C.c_int32, [_vp]),
    "medyan_mech_set_coords": (C.c_int32, [_vp, _pd]),
    "medyan_mech_get_coords": (C.c_int32, [_vp, _pd]),
    "medyan_mech_energy": (C.c_int32, [_vp, _pd, _pd]),
    "medyan_mech_forces": (C.c_int32, [_vp, _pd]),
    "medyan_mech_evaluate": (C.c_int32, [_vp, _pd, _pd, _pd, _pd]),
    "medyan_mech_enqueue_energy": (C.c_int32, [_vp]),
    "medyan_mech_enqueue_forces": (C.c_int32, [_vp]),
    "medyan_mech_enqueue_evaluate": (C.c_int32, [_vp]),
    "medyan_mech_synchronize": (C.c_int32, [_vp]),
    "medyan_mech_evaluate_async": (C.c_int32, [_vp, _pd, _pd, _pd]),
    "medyan_mech_set_deterministic": (C.c_int32, [_vp, C.c_int32]),
    "medyan_batch_set_deterministic": (C.c_int32, [_vp, C.c_int32]),
    "medyan_mech_set_host_packing": (C.c_int32, [_vp, C.c_int32]),
    "medyan_mech_wait": (C.c_int32, [_vp]),
    "medyan_mech_stream": (_vp, [_vp]),
    "medyan_mech_pass_kernel_count": (C.c_int32, [_vp, C.c_int32]),
    "medyan_mech_device_buffers": (C.c_int32, [_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp)]),
    "medyan_cg_minimize": (C.c_int32, [_vp, _vp, _pd, _pd, _vp]),
    "medyan_nl_build": (C.c_int32, [_vp, _pd, C.c_int32, _vp, _pi, C.c_int64, _pi64]),
    "medyan_mech_set_cylinders": (C.c_int32, [_vp, _vp, _vp, _vp]),
    "medyan_mech_rebuild_neighbors": (C.c_int32, [_vp, _pi64, _pi64]),
    "medyan_mech_get_excl_volume": (C.c_int32, [_vp, _pi, _pd, _pd, C.c_int64, _pi64]),
    "medyan_excl_energy_noalloc": (C.c_int32, [_vp, C.c_int32, _vp, _vp, C.c_int32, _pd, _vp]),
    "medyan_mech_param_grad": (C.c_int32, [_vp, C.c_int32, _pd, _pd, _pd, C.c_int64]),
    "medyan_mech_hessian": (C.c_int32, [_vp, C.c_float, _pd]),
    "medyan_mech_force_magnitudes": (C.c_int32, [_vp, _pd, _pd, _pd]),
    "medyan_mech_set_shapes": (C.c_int32, [_vp, _vp]),
    "medyan_mech_get_shapes": (C.c_int32, [_vp, _vp]),
    "medyan_mech_autotune": (C.c_int32, [_vp, C.c_int32, _vp]),
    "medyan_batch_set_shapes": (C.c_int32, [_vp, _vp]),
    "medyan_batch_get_shapes": (C.c_int32, [_vp, _vp]),
    "medyan_batch_autotune": (C.c_int32, [_vp, C.c_int32, _vp]),
    "medyan_mech_boundary_load_forces": (C.c_int32, [_vp, _vp, _pd, C.c_int64]),
    "medyan_mech_hvp": (C.c_int32, [_vp, _pd, _pd]),
    "medyan_batch_create": (C.c_int32, [_vp, C.c_int32, C.c_int32, C.POINTER(_vp)]),
    "medyan_batch_destroy": (C.c_int32, [_vp]),
    "medyan_batch_size": (C.c_int32, [_vp]),
    "medyan_batch_replica": (_vp, [_vp, C.c_int32]),
    "medyan_batch_minimize": (C.c_int32, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "medyan_batch_evaluate": (C.c_int32, [_vp, _vp, _pd, _vp]),
}

_lib = None


class MedyanError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        msg = f"{what}: {STATUS_NAMES.get(status, 'unknown')} (status {status})"
        if status in (5, 8) and _lib is not None:  # the CUDA error behind it
            msg += f" [{(_lib.medyan_last_cuda_error() or b'').decode()}]"
        super().__init__(msg)


def load() -> C.CDLL:
    """Load the library (once). Raises FileNotFoundError when it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is not built; run `python -m medyan_b200.build`")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(status: int, what: str) -> None:
    if status != 0:
        raise MedyanError(status, what)


def header_symbols() -> list[str]:
    """Function names declared in include/medyan_b200.h."""
    import re

    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(medyan_[a-z0-9_]+)\s*\(", text)))
