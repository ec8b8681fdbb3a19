"""The C ABI boundary without a GPU: the library loads, exports every entry
point include/medyan_b200.h declares, and the ctypes mirrors have the C
structs' layout (checked against offsetof/sizeof from a C compiler)."""
import ctypes as C
import os
import subprocess
import tempfile

import pytest

from medyan_b200 import _abi, lib

STRUCTS = {
    "medyan_system": _abi.MedyanSystem,
    "medyan_cg_params": _abi.CGParams,
    "medyan_min_result": _abi.MinResult,
    "medyan_cylinders": _abi.MedyanCylinders,
    "medyan_nl_params": _abi.NLParams,
    "medyan_boundary_params": _abi.BoundaryParams,
}


def test_library_exports_every_header_symbol():
    L = lib.load()
    declared = lib.header_symbols()
    assert len(declared) >= 15
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    assert L.medyan_abi_version() == 2
    assert L.medyan_status_string(6) == b"cylinder outside the neighbor-list grid"


def test_prototypes_cover_header():
    assert set(lib.header_symbols()) == set(lib.PROTOTYPES)


def test_struct_layout_matches_c():
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "medyan_b200.h"', "int main(void) {"]
    for cname, cls in STRUCTS.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-I", os.path.dirname(lib.HEADER), src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(line.split() for line in out if line)
    for cname, cls in STRUCTS.items():
        assert int(got[cname]) == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(cls, fname).offset, f"{cname}.{fname}"


def test_errors_without_device_are_reported_not_faked():
    # On a machine without a GPU the library must fail loudly instead of
    # computing anything on the CPU.
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except ImportError:
        pass
    from medyan_b200.forcefield import ForceFieldManager
    sv = _abi.SystemView(2, stretch_beads=[0, 3], stretch_k=[1.0], stretch_l0=[1.0])
    ff = ForceFieldManager()
    with pytest.raises(lib.MedyanError) as e:
        ff.vectorize_all_force_fields(sv)
    assert e.value.status in (5, 8)
    # the CUDA error behind the status is named, in the message too
    name = lib.load().medyan_last_cuda_error().decode()
    assert name.startswith("cudaError") and name in str(e.value)


def test_deterministic_switches_check_their_arguments():
    # argument checks come before any CUDA call, so they hold without a GPU
    L = lib.load()
    invalid = 1  # MEDYAN_ERR_INVALID_ARG
    assert L.medyan_mech_set_deterministic(None, 1) == invalid
    assert L.medyan_batch_set_deterministic(None, 1) == invalid
    assert L.medyan_batch_set_deterministic(None, 2) == invalid
