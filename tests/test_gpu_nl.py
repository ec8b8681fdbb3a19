"""GPU neighbor list vs the oracle's HybridCylinderCylinderNL restatement:
pair sets must be identical (bit-exact distance test), and the on-device
re-vectorization must reproduce CylinderExclVolume / BoundaryCylinderRepulsion
vectorize on the oracle's lists."""
import numpy as np
import pytest

from medyan_b200._abi import CylindersView, NLParams
from medyan_b200.forcefield import ForceFieldManager, neighbor_pairs
from medyan_b200.lib import MedyanError
from medyan_b200.network import make_workload

pytestmark = pytest.mark.gpu


def as_set(p):
    return set(map(tuple, np.asarray(p).reshape(-1, 2).tolist()))


@pytest.mark.parametrize("cfg,seed", [(0, 0), (0, 5), (3, 3), (1, 1), (4, 4)])
def test_pairs_match_oracle(gpu_lib, oracle, cfg, seed):
    net = make_workload(cfg, seed=seed)
    cv = net.cylinders_view()
    x = net.flat_coords()
    st, po = oracle.neighbor_pairs(cv, x, net.n_beads, net.nl_params())
    assert st == 0
    pg = neighbor_pairs(cv, x, net.n_beads, net.nl_params())
    assert pg.shape == po.shape
    assert np.array_equal(pg, po)  # same canonical order, bit-exact set


def small_cylinders(mids, half, fil=None, pos=None):
    """Cylinders along x centered at mids (n,3), length 2*half."""
    mids = np.asarray(mids, float)
    n = mids.shape[0]
    coords = np.empty((2 * n, 3))
    coords[0::2] = mids - [half, 0, 0]
    coords[1::2] = mids + [half, 0, 0]
    fil = np.arange(n) if fil is None else np.asarray(fil)
    pos = np.zeros(n, int) if pos is None else np.asarray(pos)
    cv = CylindersView(np.arange(n) * 2, np.arange(n) * 2 + 1, np.arange(n), fil, pos, np.zeros(n), np.full(n, -1),
                       np.ones(n), np.full(n, 2 * half), np.full(n, 1e5))
    return cv, coords.reshape(-1), 2 * n


def nlp(rmax=54.0, size=1000.0):
    p = NLParams()
    p.rmax = rmax
    p.rmin = 0.0
    for d in range(3):
        p.grid_size[d] = size
    return p


def test_cutoff_is_inclusive(gpu_lib, oracle):
    # midpoints exactly rmax apart are neighbors; slightly farther are not
    cv, x, nb = small_cylinders([[100, 100, 100], [154, 100, 100], [100, 100 + 54.000001, 100]], 5.0)
    pg = neighbor_pairs(cv, x, nb, nlp())
    st, po = oracle.neighbor_pairs(cv, x, nb, nlp())
    assert as_set(pg) == as_set(po) == {(1, 0)}


def test_same_filament_exclusion(gpu_lib, oracle):
    # four cylinders of one filament, 15 nm apart: all within the cutoff, but
    # only the pair with |dposition| = 3 > 2 is kept
    mids = [[100 + 15 * i, 100, 100] for i in range(4)]
    cv, x, nb = small_cylinders(mids, 5.0, fil=[0, 0, 0, 0], pos=[0, 1, 2, 3])
    pg = neighbor_pairs(cv, x, nb, nlp())
    st, po = oracle.neighbor_pairs(cv, x, nb, nlp())
    assert as_set(pg) == as_set(po) == {(3, 0)}


def test_empty_and_out_of_grid(gpu_lib):
    cv, x, nb = small_cylinders(np.zeros((0, 3)), 5.0)
    assert neighbor_pairs(cv, np.zeros(3), 1, nlp()).shape == (0, 2)
    cv, x, nb = small_cylinders([[100, 100, 100], [2000, 100, 100]], 5.0)
    with pytest.raises(MedyanError) as e:
        neighbor_pairs(cv, x, nb, nlp())
    assert e.value.status == 6


@pytest.mark.parametrize("cfg", [0, 1])
def test_device_vectorization_matches_oracle(gpu_lib, oracle, cfg):
    net = make_workload(cfg)
    st, extra = oracle.complete(net)
    assert st == 0
    x = net.flat_coords()
    sv_full = net.system_view(**extra)
    eo, pero = oracle.energy(sv_full, x)
    fo = oracle.forces(sv_full, x)
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(net.system_view())  # no excluded volume / boundary yet
        ff.set_coords(x)
        bp, planes = net.boundary_params()
        ff.set_cylinders(net.cylinders_view(), net.nl_params(), bp)
        ne, nbd = ff.rebuild_neighbor_lists()
        assert ne == extra["excl_beads"].shape[0]
        assert nbd == extra["boundary_beads"].shape[0]
        beads, krs, _ = ff.excluded_volume_interactions()
        krs_o = extra["excl_k"] * extra["excl_eqlen"][:, 0] * extra["excl_eqlen"][:, 1]
        got = sorted(zip(map(tuple, beads.tolist()), krs.tolist()))
        want = sorted(zip(map(tuple, extra["excl_beads"].tolist()), krs_o.tolist()))
        assert got == want
        e, per, f = ff.evaluate(x)
    assert abs(e - eo) <= 1e-12 * abs(eo)
    assert np.abs(f - fo).max() <= 1e-12 * np.abs(fo).max()
