"""Device packing of the force-field records (vectorize.cu, used by
medyan_mech_create and medyan_mech_update) against the host loops it
replaced (medyan_mech_set_host_packing): the same records, so with
deterministic force sums the energies, forces and parameter-gradient maps
are bit for bit the same, on the benchmark network, a branched network, a
network in shuffled bead order and networks with leftover links and bends."""
import numpy as np
import pytest

from medyan_b200._abi import SystemView
from medyan_b200.forcefield import ForceFieldManager
from medyan_b200.network import make_workload

pytestmark = pytest.mark.gpu


def both_packings(sv, x, precision="fp64"):
    out = []
    with ForceFieldManager(precision) as ff:
        ff.vectorize_all_force_fields(sv)  # create: device packing
        ff.set_deterministic(True)
        for host in (0, 1):
            if host:
                assert ff.lib.medyan_mech_set_host_packing(ff.handle, 1) == 0
                ff.vectorize_all_force_fields(sv)  # update: host loops
            e, per, f = ff.evaluate(x)
            gs = [ff.param_grad(slot, n) for slot, n in ((0, sv.count("stretch_k", 1)), (1, sv.count("bend_k", 1))) if n]
            out.append((e, per, f, gs))
        # and back to the device for an update
        assert ff.lib.medyan_mech_set_host_packing(ff.handle, 0) == 0
        ff.vectorize_all_force_fields(sv)
        out.append(ff.evaluate(x) + ([],))
    (e0, per0, f0, g0), (e1, per1, f1, g1), (e2, per2, f2, _) = out
    assert e0 == e1 == e2 and np.array_equal(per0, per1) and np.array_equal(per0, per2)
    assert np.array_equal(f0, f1) and np.array_equal(f0, f2)
    for a, b in zip(g0, g1):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    return e0, f0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_benchmark_network(gpu_lib, oracle, precision):
    net = make_workload(4)
    st, extra = oracle.complete(net)
    assert st == 0
    sv = net.system_view(**extra)
    e, f = both_packings(sv, net.flat_coords(), precision)
    eo, _ = oracle.energy(sv, net.flat_coords())
    assert abs(e - eo) <= 1e-12 * abs(eo)


def test_branched_and_shuffled(gpu_lib, oracle):
    from tests.test_gpu_bead_order import shuffled
    net = make_workload(1, n_fil=80, cyl_per_fil=8, box=1600.0, n_linker=60, n_motor=12, n_branch=16,
                        br_position_k=20.0)
    st, extra = oracle.complete(net)
    sv = net.system_view(**extra)
    x = net.flat_coords()
    e, f = both_packings(sv, x)
    assert np.abs(f - oracle.forces(sv, x)).max() <= 1e-8
    net2, extra2, sv2, x2, perm = shuffled(oracle, cfg=1, seed=2)
    e2, f2 = both_packings(sv2, x2)
    assert np.abs(f2 - oracle.forces(sv2, x2)).max() <= 1e-8


def test_leftover_links_and_bends(gpu_lib, oracle):
    """Links and bends that do not fit a chain: a second link out of a bead,
    a link closing a cycle, a bend across chain ends; and a link listed twice
    (the lower index takes the chain, the other stays a leftover)."""
    rng = np.random.default_rng(3)
    nb = 12
    x = rng.uniform(0, 40, 3 * nb)
    sb = [(0, 3), (3, 6), (6, 9), (3, 12), (9, 0), (15, 18), (18, 21), (21, 24), (15, 18), (27, 30), (30, 33)]
    bb = [(0, 3, 6), (3, 6, 9), (6, 9, 0), (15, 18, 21), (18, 21, 24), (24, 27, 30), (27, 30, 33)]
    sv = SystemView(nb, stretch_beads=np.array(sb), stretch_k=rng.uniform(1, 10, len(sb)),
                    stretch_l0=rng.uniform(5, 15, len(sb)), bend_beads=np.array(bb),
                    bend_k=rng.uniform(1, 10, len(bb)), bend_theta0=rng.uniform(0, 0.5, len(bb)))
    e, f = both_packings(sv, x)
    eo, _ = oracle.energy(sv, x)
    assert abs(e - eo) <= 1e-12 * abs(eo)
    assert np.abs(f - oracle.forces(sv, x)).max() <= 1e-8
