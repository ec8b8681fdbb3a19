"""medyan_mech_hessian: ForceFieldManager::computeHessian
(ForceFieldManager.cpp:354-398) on the device against the oracle's
restatement, on a network with every force field the small generator makes
(filaments, linkers, excluded volume), in the caller's bead order and with
shuffled bead labels.

Tolerance: entries are floats (rounded as the reference stores them); the
device and oracle forces agree to ~1e-13 relative, which the difference
quotient divides by 2*delta = 2e-4, so entries agree to 1e-6 of max|H|."""
import numpy as np
import pytest

from medyan_b200.forcefield import ForceFieldManager, hessian_modes
from medyan_b200.network import make_workload
from tests.test_gpu_bead_order import relabel

pytestmark = pytest.mark.gpu
DELTA = 1e-4  # the reference's default hessDelta


def small_net(oracle):
    net = make_workload(0, n_fil=12, cyl_per_fil=6, box=700.0, n_linker=16, seed=3)
    st, extra = oracle.complete(net)
    assert st == 0
    return net, extra


def gpu_hessian(sv, x):
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(sv)
        ff.set_coords(x)
        H = ff.hessian(DELTA)
        x_after = ff.get_coords()
        hv = ff.hvp(np.ones(x.size))
    return H, x_after, hv


def check(Hg, Ho):
    assert np.array_equal(Hg, Hg.astype(np.float32).astype(np.float64))
    assert np.abs(Hg - Ho).max() <= 1e-6 * np.abs(Ho).max()


def test_hessian_matches_oracle(gpu_lib, oracle):
    net, extra = small_net(oracle)
    sv, x = net.system_view(**extra), net.flat_coords()
    assert len(extra["excl_beads"]) > 0
    Hg, x_after, hv = gpu_hessian(sv, x)
    check(Hg, oracle.hessian(sv, x, DELTA))
    # the coordinates are restored exactly
    assert np.array_equal(x_after, x)
    # a uniform translation costs no energy: H 1 = 0 up to the difference error
    assert np.abs(Hg @ np.ones(x.size)).max() <= 1e-5 * np.abs(Hg).max()
    # the symmetric part agrees with the Hessian-vector product
    Hs = 0.5 * (Hg + Hg.T)
    v = np.random.default_rng(0).normal(size=x.size)
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(sv)
        ff.set_coords(x)
        hv = ff.hvp(v)
    assert np.abs(Hs @ v - hv).max() <= 1e-4 * np.abs(hv).max()
    m = hessian_modes(Hg)
    assert np.all(m.IPRI <= 1 + 1e-9) and np.all(m.IPRII <= 1 + 1e-9)


def test_hessian_shuffled_beads(gpu_lib, oracle):
    net, extra = small_net(oracle)
    sv, x, perm = relabel(net, extra, 7)
    Hg, x_after, _ = gpu_hessian(sv, x)
    check(Hg, oracle.hessian(sv, x, DELTA))
    assert np.array_equal(x_after, x)


def test_hessian_rejects_bad_delta(gpu_lib, oracle):
    from medyan_b200.lib import MedyanError
    net, extra = small_net(oracle)
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(net.system_view(**extra))
        ff.set_coords(net.flat_coords())
        with pytest.raises(MedyanError):
            ff.hessian(0.0)
