"""After-minimization quantities on the device against the oracle:
medyan_mech_boundary_load_forces (BoundaryCylinderRepulsion::computeLoadForces,
BoundaryCylinderRepulsion.cpp:125-196) on filament tips near the planes of a
cubic boundary, and medyan_mech_force_magnitudes (the inputs of
ForceFieldManager::assignallforcemags, ForceFieldManager.cpp:346-351) on the
golden networks with linkers, motors and branch points. FP64 on both sides:
1e-12 relative (load forces: of the largest load of the tip; force
magnitudes: of the largest, with a 1e-9 pN floor for springs at rest length)."""
import json
import os

import numpy as np
import pytest

from medyan_b200.forcefield import ForceFieldManager
from tests.aux_nets import tip_network
from tests.test_oracle_pins import network_system

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("seed", [0, 3])
def test_boundary_load_forces(gpu_lib, oracle, seed):
    sv, x, cv, nlp, bp, planes, tips, plus = tip_network(seed=seed)
    n_mon = np.full(len(tips), 40)
    n_mon[::5] = 13  # tips of another filament type
    mon = np.where(n_mon == 40, 2.7, 5.4)
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(sv)
        ff.set_coords(x)
        ff.set_cylinders(cv, nlp, bp)
        ff.rebuild_neighbor_lists()
        got = ff.boundary_load_forces(tips, plus, n_mon, mon)
        # twice in a row: the same loads (they are recomputed, not accumulated)
        again = ff.boundary_load_forces(tips, plus, n_mon, mon)
    want = oracle.boundary_load_forces(cv, x, bp, tips, plus, n_mon, mon)
    assert sum(1 for w in want if w.max() > 1e-3) >= 3  # tips that feel the boundary
    for g, a, w in zip(got, again, want):
        assert g.shape == w.shape
        assert np.abs(g - w).max() <= 1e-12 * max(np.abs(w).max(), 1e-300)
        assert np.array_equal(g, a)


def test_boundary_load_forces_errors(gpu_lib, oracle):
    from medyan_b200.lib import MedyanError
    sv, x, cv, nlp, bp, planes, tips, plus = tip_network(seed=0)
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(sv)
        ff.set_coords(x)
        with pytest.raises(MedyanError):  # no cylinder list yet
            ff.boundary_load_forces(tips, plus, np.full(len(tips), 40), np.full(len(tips), 2.7))
        ff.set_cylinders(cv, nlp, bp)
        with pytest.raises(MedyanError):  # no neighbor list built yet
            ff.boundary_load_forces(tips, plus, np.full(len(tips), 40), np.full(len(tips), 2.7))
        ff.rebuild_neighbor_lists()
        with pytest.raises(MedyanError):  # cylinder index out of range
            ff.boundary_load_forces([10 ** 6], [1], [40], [2.7])


@pytest.mark.parametrize("tag", ["cfg0", "branched"])
def test_force_magnitudes(gpu_lib, oracle, tag):
    nets = dict(np.load(os.path.join(GOLDEN, "synthetic_networks.npz")))
    sv, x = network_system(nets, tag)
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(sv)
        ff.set_coords(x)
        lin, mot, br = ff.force_magnitudes()
    lo, mo, bo = oracle.force_magnitudes(sv, x)
    for g, w in ((lin, lo), (mot, mo), (br, bo)):
        assert g.shape == w.shape
        if w.size:
            # 1e-12 relative, with a 1e-9 pN floor for springs at rest length
            assert np.abs(g - w).max() <= 1e-12 * np.abs(w).max() + 1e-9
    assert lin.size > 0 and (tag != "branched" or br.shape[0] > 0)
