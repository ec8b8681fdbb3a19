"""Batched minimization of independent networks (medyan_batch_*): every
replica must behave exactly as it does alone (same call counts and
coordinates as the oracle's CGMethod on that replica), with replicas of
uneven size and different outcomes in one batch."""
import numpy as np
import pytest

from medyan_b200._abi import SystemView
from medyan_b200.forcefield import BatchMinimizer, ForceFieldManager, conjugate_gradient_params as cgp
from medyan_b200.network import make_batch

pytestmark = pytest.mark.gpu


def replicas(oracle, n=6, seed=5, cyl_range=(200, 800)):
    nets = make_batch(n, seed, cyl_range)
    out = []
    for net in nets:
        st, extra = oracle.complete(net)
        assert st == 0
        out.append((net.system_view(**extra), net.flat_coords()))
    return out


@pytest.mark.parametrize("line_search", ["BACKTRACKING", "QUADRATIC"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_single(gpu_lib, oracle, precision, line_search):
    reps = replicas(oracle)
    p = cgp(grad_tol=1e-4, energy_rel_tol=1e-14, energy_call_limit=40, line_search=line_search)
    # the quadratic model's vertex divides energy differences: rounding grows there
    tol = 1e-7 if line_search == "BACKTRACKING" else 1e-6
    with BatchMinimizer([sv for sv, _ in reps], precision) as b:
        st, xs, fs, rs = b.minimize([x for _, x in reps], p)
    for r, (sv, x) in enumerate(reps):
        with ForceFieldManager(precision) as ff:
            ff.vectorize_all_force_fields(sv)
            s1, x1, f1, r1 = ff.minimize(x, p)
        assert st[r] == s1 == 0
        # a replica in a batch is the same computation as alone (forces
        # accumulate with atomics, so equal to rounding, not bit for bit)
        assert (rs[r].num_energy_call, rs[r].num_force_call, rs[r].num_iter) == \
            (r1.num_energy_call, r1.num_force_call, r1.num_iter)
        assert np.abs(xs[r] - x1).max() <= tol
        assert np.abs(fs[r] - f1).max() <= tol * np.abs(f1).max()
        if precision == "fp64":
            so, xo, fo, ro = oracle.minimize(sv, x, p)
            assert (rs[r].num_energy_call, rs[r].num_iter) == (ro.num_energy_call, ro.num_iter)
            assert np.abs(xs[r] - xo).max() <= tol


def test_batch_converges_each_replica(gpu_lib, oracle):
    reps = replicas(oracle, n=5, seed=7)
    p = cgp(grad_tol=1.0)
    with BatchMinimizer([sv for sv, _ in reps], "fp64") as b:
        st, xs, fs, rs = b.minimize([x for _, x in reps], p)
    iters = [r.num_iter for r in rs]
    for r in range(len(reps)):
        assert st[r] == 0
        # converged, or stopped by the force-call limit (MinimizationResult::callLimitExceeded)
        assert (rs[r].grad_inf_norm < 1.0 or rs[r].energy_rel_change < 1e-9
                or rs[r].num_force_call >= rs[r].force_call_limit), (rs[r].grad_inf_norm, rs[r].num_force_call)
        assert np.abs(fs[r]).max() == pytest.approx(rs[r].grad_inf_norm)
    assert len(set(iters)) > 1  # replicas stop at their own iteration counts


def test_batch_line_search_failure_is_per_replica(gpu_lib, oracle):
    # a degenerate replica (NaN bend energy, recovery off) next to a healthy one
    bad_x = np.array([0, 0, 0, 0, 0, 0, 10, 0, 0, 30, 5, 0, 60, 5, 0], float)
    bad = SystemView(5, bend_beads=[0, 3, 6], bend_k=[10.0], bend_theta0=[0.0], stretch_beads=[9, 12],
                     stretch_k=[5.0], stretch_l0=[20.0])
    (good, good_x), = replicas(oracle, n=1, seed=9)
    p = cgp(grad_tol=1e-3, try_to_recover=False, energy_call_limit=40)
    with BatchMinimizer([bad, good], "fp64") as b:
        st, xs, fs, rs = b.minimize([bad_x, good_x], p)
    so, xo, fo, ro = oracle.minimize(bad, bad_x, p)
    assert st[0] == so == 7 and rs[0].error_flags == ro.error_flags == 1
    assert st[1] == 0


def test_batch_evaluate(gpu_lib, oracle):
    reps = replicas(oracle, n=4, seed=11)
    with BatchMinimizer([sv for sv, _ in reps], "fp64") as b:
        e, fs = b.evaluate([x for _, x in reps])
    for r, (sv, x) in enumerate(reps):
        eo, _ = oracle.energy(sv, x)
        fo = oracle.forces(sv, x)
        assert abs(e[r] - eo) <= 1e-12 * abs(eo)
        assert np.abs(fs[r] - fo).max() <= 1e-12 * np.abs(fo).max()


def test_batch_shapes_keep_results(gpu_lib, oracle):
    # a packed layout of other block shapes is the same computation
    import ctypes as C
    reps = replicas(oracle, n=5, seed=13)
    p = cgp(grad_tol=1e-4, energy_rel_tol=1e-14, energy_call_limit=30)
    with BatchMinimizer([sv for sv, _ in reps], "fp64") as b:
        st0, xs0, _, rs0 = b.minimize([x for _, x in reps], p)
        b.set_shapes(bonded_threads=128, excl_threads=32, chain_threads=512, chain_chunk=1024)
        assert b.get_shapes() == dict(bonded_threads=128, excl_threads=32, chain_threads=512, chain_chunk=1024)
        st1, xs1, _, rs1 = b.minimize([x for _, x in reps], p)
        # the autotuner times packed passes at the replicas' coordinates
        for r, (_, x) in enumerate(reps):
            xx = np.ascontiguousarray(x, np.float64)
            b.lib.medyan_mech_set_coords(b.replica(r), xx.ctypes.data_as(C.POINTER(C.c_double)))
        chosen = b.autotune(reps=3)
        assert chosen == b.get_shapes()
        st2, xs2, _, rs2 = b.minimize([x for _, x in reps], p)
    for r in range(len(reps)):
        assert st0[r] == st1[r] == st2[r] == 0
        assert (rs0[r].num_energy_call, rs0[r].num_force_call) == (rs1[r].num_energy_call, rs1[r].num_force_call) \
            == (rs2[r].num_energy_call, rs2[r].num_force_call)
        assert np.abs(xs1[r] - xs0[r]).max() <= 1e-7 and np.abs(xs2[r] - xs0[r]).max() <= 1e-7


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_full_ensemble_start_state_matches_oracle(gpu_lib, oracle, precision):
    """The whole 256-replica ensemble of the medium network's composition
    (200-4,000 cylinders each), neighbor lists built on the device per
    replica, as the benchmark runs it. A minimization whose gradient
    tolerance holds at the start coordinates runs one packed energy pass and
    one packed force pass and moves nothing: its energy_before_total and
    returned forces are the packed kernels' values at the start coordinates,
    checked against the oracle on 16 replicas spread over the size range."""
    from medyan_b200.network import make_batch
    nets = make_batch(256, 2)
    xs = [net.flat_coords() for net in nets]
    with BatchMinimizer([net.system_view() for net in nets], precision) as b:
        for r, net in enumerate(nets):
            bp, _ = net.boundary_params()
            b.rebuild_neighbor_lists(r, xs[r], net.cylinders_view(), net.nl_params(), bp)
        st, xo, fo, rs = b.minimize(xs, cgp(grad_tol=1e30))
    tol = 1e-12 if precision == "fp64" else 1e-6
    order = np.argsort([net.n_beads for net in nets])
    sample = sorted(set(int(order[i]) for i in np.linspace(0, len(nets) - 1, 16).round().astype(int)))
    assert len(sample) >= 8
    for r in sample:
        assert st[r] == 0 and rs[r].num_iter == 0
        assert np.array_equal(xo[r], xs[r])
        stc, extra = oracle.complete(nets[r])
        assert stc == 0
        sv = nets[r].system_view(**extra)
        eo, _ = oracle.energy(sv, xs[r])
        fref = oracle.forces(sv, xs[r])
        # energies are FP64 in both precisions
        assert abs(rs[r].energy_before_total - eo) <= 1e-12 * abs(eo), (r, rs[r].energy_before_total, eo)
        assert np.abs(fo[r] - fref).max() <= tol * np.abs(fref).max(), r


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_deterministic_reproducible(gpu_lib, oracle, precision):
    """medyan_batch_set_deterministic: fixed-point force sums make a batched
    minimization bitwise reproducible, and each replica still takes the
    calls and steps it takes alone (single network, deterministic sums)."""
    reps = replicas(oracle, n=6, seed=11)
    p = cgp(grad_tol=1e-4, energy_rel_tol=1e-14, energy_call_limit=40)
    runs = []
    with BatchMinimizer([sv for sv, _ in reps], precision) as b:
        b.set_deterministic(True)
        for _ in range(2):
            runs.append(b.minimize([x for _, x in reps], p))
    (st1, xs1, fs1, rs1), (st2, xs2, fs2, rs2) = runs
    for r, (sv, x) in enumerate(reps):
        assert st1[r] == st2[r] == 0
        assert np.array_equal(xs1[r], xs2[r]) and np.array_equal(fs1[r], fs2[r])
        assert rs1[r].energy_after_total == rs2[r].energy_after_total
        assert (rs1[r].num_energy_call, rs1[r].num_iter) == (rs2[r].num_energy_call, rs2[r].num_iter)
        with ForceFieldManager(precision) as ff:
            ff.vectorize_all_force_fields(sv)
            ff.set_deterministic(True)
            s1, x1, f1, r1 = ff.minimize(x, p)
        assert s1 == 0
        assert (rs1[r].num_energy_call, rs1[r].num_force_call, rs1[r].num_iter) == \
            (r1.num_energy_call, r1.num_force_call, r1.num_iter)
        assert np.abs(xs1[r] - x1).max() <= 1e-7
        assert np.abs(fs1[r] - f1).max() <= 1e-7 * np.abs(f1).max()
