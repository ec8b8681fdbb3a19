"""The C++ drop-in layer (include/medyan_b200.hpp): tests/cpp/test_adaptor.cpp
is compiled against the library and the oracle and run. Without a GPU the
manager must refuse to work (no host fallback); on a GPU it must match the
oracle (energies and forces 1e-12, neighbor-list pair count, CG call
counts)."""
import os
import subprocess

import pytest

from medyan_b200 import lib
from oracle.oracle import ORACLE_SO

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_adaptor.cpp")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    lib.load()  # the library must be built
    if not os.path.exists(ORACLE_SO):
        pytest.skip("oracle library not built")
    out = str(tmp_path_factory.mktemp("cpp") / "test_adaptor")
    libdir, odir = os.path.dirname(lib.LIB_PATH), os.path.dirname(ORACLE_SO)
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-I", odir,
                    SRC, "-L", libdir, "-lmedyan_b200", "-L", odir, "-lmedyan_oracle",
                    f"-Wl,-rpath,{libdir}:{odir}", "-o", out], check=True)
    return out


def test_adaptor_refuses_without_device(exe):
    if _cuda_available():
        pytest.skip("a GPU is visible")
    r = subprocess.run([exe, "nodevice"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_adaptor_matches_oracle(gpu_lib, exe):
    r = subprocess.run([exe, "gpu"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "adaptor ok" in r.stdout
