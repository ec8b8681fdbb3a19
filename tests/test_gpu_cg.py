"""Device conjugate-gradient minimizer vs the oracle's CGMethod restatement
(itself bit-for-bit with the reference's CGMethod).

Short runs (an energy-call limit) must take the same iterations, line-search
decisions and call counts as the oracle, with coordinates equal to rounding
(1e-7 nm: beta amplifies last-bit differences over the run) and energies
within 1e-12 relative. Full runs must converge as the
oracle does. Line-search failure, safe mode and the recovery step are driven
by a degenerate (zero-length) bend whose energy is NaN, exactly as in the
reference.
"""
import numpy as np
import pytest

from medyan_b200._abi import SystemView
from medyan_b200.forcefield import ForceFieldManager, conjugate_gradient_params as cgp
from medyan_b200.network import make_workload

pytestmark = pytest.mark.gpu


def small_net(oracle, **kw):
    base = dict(n_fil=12, cyl_per_fil=6, box=700.0, n_linker=16, seed=3)
    base.update(kw)
    net = make_workload(0, **base)
    st, extra = oracle.complete(net)
    assert st == 0
    return net.system_view(**extra), net.flat_coords()


def gpu_min(sv, x, p, precision="fp64"):
    with ForceFieldManager(precision) as ff:
        ff.vectorize_all_force_fields(sv)
        return ff.minimize(x, p)


@pytest.mark.parametrize("method", [0, 1, 2])
def test_short_run_matches_oracle(gpu_lib, oracle, method):
    sv, x = small_net(oracle)
    p = cgp(method=method, grad_tol=1e-4, energy_rel_tol=1e-14, energy_call_limit=40)
    so, xo, fo, ro = oracle.minimize(sv, x, p)
    sg, xg, fg, rg = gpu_min(sv, x, p)
    assert sg == so == 0
    assert (rg.num_energy_call, rg.num_force_call, rg.num_iter) == (ro.num_energy_call, ro.num_force_call, ro.num_iter)
    errs = (np.abs(xg - xo).max(), abs(rg.energy_after_total - ro.energy_after_total) / abs(ro.energy_after_total),
            abs(rg.energy_before_total - ro.energy_before_total) / abs(ro.energy_before_total),
            np.abs(fg - fo).max() / np.abs(fo).max())
    # energy-before is at identical coordinates (1e-12); energy-after is at
    # coordinates that differ by rounding carried through the run (1e-10)
    assert errs[0] <= 1e-7 and errs[1] <= 1e-10 and errs[2] <= 1e-12 and errs[3] <= 1e-7, errs


@pytest.mark.parametrize("deterministic", [False, True])
def test_both_precisions_converge_on_the_gradient(gpu_lib, oracle, deterministic):
    """The 50 x 10 network (the CPU-runnable workload): FP64 and mixed both
    reach max|F| < gradTol; their minima differ by no more than two runs of
    the oracle whose starts differ by one ulp do (3.6e-3 relative there,
    tests/test_minimization_sensitivity.py), with margin."""
    net = make_workload(0)
    st, extra = oracle.complete(net)
    assert st == 0
    sv, x = net.system_view(**extra), net.flat_coords()
    p = cgp(grad_tol=1.0, energy_rel_tol=0.0)
    out = {}
    for prec in ("fp64", "mixed"):
        with ForceFieldManager(prec) as ff:
            ff.vectorize_all_force_fields(sv)
            ff.set_deterministic(deterministic)
            out[prec] = ff.minimize(x, p)
    for prec, (sg, xg, fg, rg) in out.items():
        assert sg == 0 and rg.grad_inf_norm < 1.0, (prec, rg.grad_inf_norm)
    e64, em = out["fp64"][3].energy_after_total, out["mixed"][3].energy_after_total
    assert abs(em - e64) <= 2e-2 * abs(e64), (e64, em)


@pytest.mark.parametrize("layout", [0, 2])
def test_fused_force_pass_short_run(gpu_lib, oracle, layout):
    """The minimizer with a fused pass layout (its force pass: zero fill,
    then the chain/bonded, branching and excluded-volume kernels side by side;
    layout 2 with the chain segments staged through shared memory) takes the
    oracle's iterations and calls."""
    sv, x = small_net(oracle)
    p = cgp(grad_tol=1e-4, energy_rel_tol=1e-14, energy_call_limit=40)
    so, xo, fo, ro = oracle.minimize(sv, x, p)
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(sv)
        ff.set_shapes(pass_layout=layout)
        sg, xg, fg, rg = ff.minimize(x, p)
    assert sg == so == 0
    assert (rg.num_energy_call, rg.num_force_call, rg.num_iter) == (ro.num_energy_call, ro.num_force_call, ro.num_iter)
    assert np.abs(xg - xo).max() <= 1e-7


def test_converges_like_oracle(gpu_lib, oracle):
    sv, x = small_net(oracle)
    p = cgp(grad_tol=1.0)
    so, xo, fo, ro = oracle.minimize(sv, x, p)
    sg, xg, fg, rg = gpu_min(sv, x, p)
    assert sg == so == 0
    assert rg.grad_inf_norm < 1.0 or rg.energy_rel_change < 1e-9
    assert np.abs(fg).max() == pytest.approx(rg.grad_inf_norm)
    # trajectories separate at rounding level over hundreds of iterations:
    # the oracle itself, started one ulp away, ends 1.7e-4 relative apart on
    # this network (tests/test_minimization_sensitivity.py), so 1e-2 is that
    # spread with margin, not a looser parity
    assert abs(rg.energy_after_total - ro.energy_after_total) <= 1e-2 * abs(ro.energy_after_total)
    assert 0.5 * ro.num_iter <= rg.num_iter <= 2 * ro.num_iter


@pytest.mark.parametrize("method", [0, 2])
def test_quadratic_short_run_matches_oracle(gpu_lib, oracle, method):
    """lineSearchAlgorithm QUADRATIC: quadraticLineSearchV2's backtracking
    phase, its trial history and the quadratic-optimization passes."""
    sv, x = small_net(oracle)
    kw = dict(method=method, grad_tol=1e-4, energy_rel_tol=1e-14, energy_call_limit=40)
    p = cgp(line_search="QUADRATIC", **kw)
    so, xo, fo, ro = oracle.minimize(sv, x, p)
    # this run takes quadratic steps: it leaves the backtracking trajectory
    _, xb, _, _ = oracle.minimize(sv, x, cgp(**kw))
    assert np.abs(xb - xo).max() > 1e-3
    sg, xg, fg, rg = gpu_min(sv, x, p)
    assert sg == so == 0
    assert (rg.num_energy_call, rg.num_force_call, rg.num_iter) == (ro.num_energy_call, ro.num_force_call, ro.num_iter)
    # the model's vertex -b/2a divides differences of energies that agree to
    # 1e-12 relative: coordinates agree to 1e-6 nm rather than 1e-7
    errs = (np.abs(xg - xo).max(), abs(rg.energy_after_total - ro.energy_after_total) / abs(ro.energy_after_total),
            np.abs(fg - fo).max() / np.abs(fo).max())
    assert errs[0] <= 1e-6 and errs[1] <= 1e-9 and errs[2] <= 1e-6, errs


def test_quadratic_converges_like_oracle(gpu_lib, oracle):
    sv, x = small_net(oracle)
    p = cgp(grad_tol=1.0, line_search="QUADRATIC")
    so, xo, fo, ro = oracle.minimize(sv, x, p)
    sg, xg, fg, rg = gpu_min(sv, x, p)
    assert sg == so == 0
    assert rg.grad_inf_norm < 1.0 or rg.energy_rel_change < 1e-9
    assert abs(rg.energy_after_total - ro.energy_after_total) <= 1e-2 * abs(ro.energy_after_total)
    assert 0.5 * ro.num_iter <= rg.num_iter <= 2 * ro.num_iter


def frustrated_triangles(n=200, seed=0):
    # spring triangles with incompatible rest lengths (10, 10, 25): a unique
    # minimum (up to rigid motion) with nonzero energy
    rng = np.random.default_rng(seed)
    base = np.array([[0, 0, 0], [10, 0, 0], [5, 8, 0]], float)
    x = (base[None] + rng.normal(0, 1.0, (n, 3, 3)) + np.arange(n)[:, None, None] * np.array([50.0, 0, 0])).reshape(-1)
    b = np.arange(n) * 3
    beads = np.stack([np.stack([3 * b, 3 * (b + 1)], 1), np.stack([3 * (b + 1), 3 * (b + 2)], 1),
                      np.stack([3 * (b + 2), 3 * b], 1)], 1).reshape(-1, 2)
    sv = SystemView(3 * n, stretch_beads=beads, stretch_k=np.tile([100.0, 50.0, 20.0], n),
                    stretch_l0=np.tile([10.0, 10.0, 25.0], n))
    return sv, x


def test_mixed_precision_matches_fp64_at_convergence(gpu_lib, oracle):
    # gradTol 1e-3 pN: above the float resolution of these ~100 pN forces,
    # and close enough to the minimum that its energy is fixed to ~1e-10
    sv, x = frustrated_triangles()
    p = cgp(grad_tol=1e-3, energy_rel_tol=1e-16)
    so, xo, fo, ro = oracle.minimize(sv, x, p)
    sd, xd, fd, rd = gpu_min(sv, x, p, "fp64")
    sm, xm, fm, rm = gpu_min(sv, x, p, "mixed")
    assert so == sd == sm == 0
    # the final configurations' FP64 energies, within the stated mixed-mode
    # bound (1e-8 relative); the mixed path computes forces in float and
    # energies in double, so its line search sees the same energies
    for r, xr in ((rd, xd), (rm, xm)):
        e_fp64, _ = oracle.energy(sv, xr)
        assert abs(e_fp64 - ro.energy_after_total) <= 1e-8 * abs(ro.energy_after_total), e_fp64
        assert abs(r.energy_after_total - e_fp64) <= 1e-12 * abs(e_fp64)
        assert r.grad_inf_norm < 1e-3 or r.energy_rel_change < 1e-16


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_returned_forces_are_those_at_the_returned_coordinates(gpu_lib, oracle, precision):
    # The first line-search pass of an iteration can also compute the forces
    # at its first trial step; when the line search takes that step, the
    # iteration's force pass is skipped. Whichever path each iteration took,
    # the forces a converged minimization returns are a fresh evaluation's at
    # its final coordinates, up to the atomics' summation order. At a minimum
    # a bead's net force is a small difference of terms hundreds of times
    # larger (excluded-volume repulsion against filament tension), so the
    # order of the atomic sums shows at ~1e-12 of the net max|F|.
    sv, x = small_net(oracle, n_fil=30, cyl_per_fil=8, box=1000.0, n_linker=60, seed=11)
    p = cgp(grad_tol=0.5)
    with ForceFieldManager(precision) as ff:
        ff.vectorize_all_force_fields(sv)
        sg, xg, fg, rg = ff.minimize(x, p)
        f_fresh = ff.compute_forces(xg)
    assert sg == 0 and rg.num_iter > 20
    assert np.abs(fg - f_fresh).max() <= 1e-10 * np.abs(f_fresh).max()
    assert rg.grad_inf_norm == pytest.approx(np.abs(f_fresh).max(), rel=1e-10)


def test_already_converged(gpu_lib, oracle):
    sv, x = small_net(oracle)
    p = cgp(grad_tol=1e12)
    sg, xg, fg, rg = gpu_min(sv, x, p)
    so, xo, fo, ro = oracle.minimize(sv, x, p)
    assert sg == 0 and rg.num_iter == 0
    assert (rg.num_energy_call, rg.num_force_call) == (ro.num_energy_call, ro.num_force_call) == (2, 1)
    assert np.array_equal(xg, x)


def degenerate_system():
    # a bend whose first two beads coincide (NaN energy and forces) next to a
    # stretched spring that gives a finite max force
    x = np.array([0, 0, 0, 0, 0, 0, 10, 0, 0, 30, 5, 0, 60, 5, 0], float)
    sv = SystemView(5, bend_beads=[0, 3, 6], bend_k=[10.0], bend_theta0=[0.0],
                    stretch_beads=[9, 12], stretch_k=[5.0], stretch_l0=[20.0])
    return sv, x


@pytest.mark.parametrize("line_search", ["BACKTRACKING", "QUADRATIC"])
@pytest.mark.parametrize("recover", [0, 1])
def test_line_search_failure_paths(gpu_lib, oracle, recover, line_search):
    sv, x = degenerate_system()
    p = cgp(grad_tol=1e-3, try_to_recover=bool(recover), line_search=line_search)
    so, xo, fo, ro = oracle.minimize(sv, x, p)
    sg, xg, fg, rg = gpu_min(sv, x, p)
    assert sg == so
    assert rg.error_flags == ro.error_flags
    assert (rg.num_energy_call, rg.num_force_call, rg.num_iter) == (ro.num_energy_call, ro.num_force_call, ro.num_iter)
    if not recover:
        assert sg == 7 and rg.error_flags == 1


def test_rejects_bad_params(gpu_lib, oracle):
    from medyan_b200.lib import MedyanError
    sv, x = small_net(oracle)
    with pytest.raises(MedyanError):
        gpu_min(sv, x, cgp(method=5))
    p = cgp()
    p.line_search = 2
    with pytest.raises(MedyanError):
        gpu_min(sv, x, p)
