"""medyan_excl_energy_noalloc (static device scratch, no device allocation)
against the handle path's excluded-volume slot (medyan_mech_energy), called
through the C ABI on caller-owned device arrays. Two calls in a row must both
agree, so the scratch flags are cleared between calls."""
import ctypes as C

import numpy as np
import pytest

from medyan_b200 import lib
from medyan_b200.forcefield import ForceFieldManager
from medyan_b200.network import make_workload

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12  # same kernels and summation order as the handle path


def _device_inputs(cfg, seed, oracle):
    import torch

    net = make_workload(cfg, seed=seed)
    st, extra = oracle.complete(net)
    assert st == 0
    x = net.flat_coords()
    krs = extra["excl_k"] * extra["excl_eqlen"][:, 0] * extra["excl_eqlen"][:, 1]
    dev = dict(x=torch.tensor(x, dtype=torch.float64, device="cuda"),
               beads=torch.tensor(np.ascontiguousarray(extra["excl_beads"], np.int32).reshape(-1), device="cuda"),
               krs=torch.tensor(krs, dtype=torch.float64, device="cuda"))
    return net, extra, x, dev


def _noalloc(dev, n_beads, n_pairs):
    import torch

    L = lib.load()
    e = C.c_double(0.0)
    st = L.medyan_excl_energy_noalloc(C.c_void_p(dev["x"].data_ptr()), n_beads, C.c_void_p(dev["beads"].data_ptr()),
                                      C.c_void_p(dev["krs"].data_ptr()), n_pairs, C.byref(e),
                                      C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st, e.value


@pytest.mark.parametrize("cfg,seed", [(1, 0), (0, 5)])
def test_matches_handle_path_twice(gpu_lib, oracle, cfg, seed):
    net, extra, x, dev = _device_inputs(cfg, seed, oracle)
    n_pairs = extra["excl_beads"].shape[0]
    assert n_pairs > 0
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(net.system_view(**extra))
        want = dict(ff.compute_individual_energies(x).individual)["CylinderExcludedVolume"]
    for _ in range(2):
        st, got = _noalloc(dev, net.n_beads, n_pairs)
        assert st == 0
        assert abs(got - want) <= REL_TOL * abs(want), (got, want)


def test_calls_allocate_no_device_memory(gpu_lib, oracle):
    """The property the entry point exists for: after one warm-up call (which
    loads the library's kernels on the device), further calls leave the
    device's free memory and torch's allocator untouched."""
    import torch

    net, extra, x, dev = _device_inputs(1, 0, oracle)
    n_pairs = extra["excl_beads"].shape[0]
    st, e0 = _noalloc(dev, net.n_beads, n_pairs)
    assert st == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    for _ in range(5):
        st, e = _noalloc(dev, net.n_beads, n_pairs)
        assert st == 0 and e == e0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert torch.cuda.memory_allocated() == alloc0


def test_limits_and_bad_offsets(gpu_lib, oracle):
    net, extra, x, dev = _device_inputs(0, 0, oracle)
    n_pairs = extra["excl_beads"].shape[0]
    assert _noalloc(dev, net.n_beads, 0) == (0, 0.0)
    st, _ = _noalloc(dev, net.n_beads, 262144 + 1)
    assert st == 9  # MEDYAN_ERR_CAPACITY, before any device work
    st, e0 = _noalloc(dev, net.n_beads, n_pairs)
    assert st == 0 and np.isfinite(e0)
    orig = int(dev["beads"][1])
    dev["beads"][1] = 3 * net.n_beads  # one past the last bead
    st, _ = _noalloc(dev, net.n_beads, n_pairs)
    assert st == 2  # MEDYAN_ERR_INDEX_RANGE
    dev["beads"][1] = orig
    assert _noalloc(dev, net.n_beads, n_pairs) == (0, e0)
