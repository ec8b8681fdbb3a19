"""Asynchronous double-buffered evaluation (medyan_mech_evaluate_async /
medyan_mech_wait) against the synchronous medyan_mech_evaluate and the
oracle: a stream of coordinate sets, more than the two staging slots, each
result landing in its own host buffers."""
import numpy as np
import pytest

from medyan_b200.forcefield import ForceFieldManager
from medyan_b200.network import make_workload

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("layout", [0, 1, 2])
def test_async_stream_matches_sync(gpu_lib, oracle, precision, layout):
    net = make_workload(1)
    st, extra = oracle.complete(net)
    assert st == 0
    sv = net.system_view(**extra)
    x0 = net.flat_coords()
    rng = np.random.default_rng(4)
    coords = [x0 + rng.normal(0.0, 0.05, x0.shape) for _ in range(5)]
    with ForceFieldManager(precision) as ff:
        ff.vectorize_all_force_fields(sv)
        ff.set_shapes(pass_layout=layout)
        es, fs = ff.evaluate_many(coords)
        for i, x in enumerate(coords):
            e, per, f = ff.evaluate(x)
            # the same pass on the same coordinates: energies bitwise (fixed
            # reduction order), forces to the atomics' summation order
            assert es[i, -1] == e and np.array_equal(es[i, :-1], per), i
            assert np.abs(fs[i] - f).max() <= 1e-12 * np.abs(f).max(), i
    for i in (0, 4):
        eo, _ = oracle.energy(sv, coords[i])
        fo = oracle.forces(sv, coords[i])
        tol = 1e-12 if precision == "fp64" else 1e-6
        assert abs(es[i, -1] - eo) <= 1e-12 * abs(eo)
        assert np.abs(fs[i] - fo).max() <= tol * np.abs(fo).max()


def test_async_reordered_beads(gpu_lib, oracle):
    """A caller whose bead order is not filament order (the internal layout
    reorders in and out of the staging slots)."""
    from tests.test_gpu_bead_order import shuffled
    net, extra, svp, xp, perm = shuffled(oracle, cfg=0)
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(svp)
        es, fs = ff.evaluate_many([xp, xp, xp])
        e, per, f = ff.evaluate(xp)
    fo = oracle.forces(svp, xp)
    for i in range(3):
        assert es[i, -1] == e
        assert np.abs(fs[i] - f).max() <= 1e-12 * np.abs(f).max()
        assert np.abs(fs[i] - fo).max() <= 1e-12 * np.abs(fo).max()
