"""Deterministic force sums (medyan_mech_set_deterministic): forces summed as
64-bit fixed-point integers (2^-32 pN) are bitwise reproducible from run to
run, and so are whole minimizations; they agree with the oracle to the
format's resolution. Contributions beyond the format's range are reported."""
import numpy as np
import pytest

from medyan_b200._abi import SystemView
from medyan_b200.forcefield import ForceFieldManager, conjugate_gradient_params as cgp
from medyan_b200.network import make_workload

pytestmark = pytest.mark.gpu

# each contribution rounds to 2^-32 pN; a bead sums a few tens of them
ABS_TOL = 1e-8  # pN


def net_of(oracle, cfg):
    net = make_workload(cfg)
    st, extra = oracle.complete(net)
    assert st == 0
    return net.system_view(**extra), net.flat_coords()


@pytest.mark.parametrize("layout", [0, 1, 2])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_forces_reproducible_and_match_oracle(gpu_lib, oracle, precision, layout):
    sv, x = net_of(oracle, 1)
    fo = oracle.forces(sv, x)
    eo, _ = oracle.energy(sv, x)
    with ForceFieldManager(precision) as ff:
        ff.vectorize_all_force_fields(sv)
        ff.set_shapes(pass_layout=layout)
        ff.set_deterministic(True)
        runs = [ff.evaluate(x) for _ in range(3)]
        f_sep = ff.compute_forces(x)
    e0, per0, f0 = runs[0]
    for e, per, f in runs[1:]:
        assert e == e0 and np.array_equal(per, per0) and np.array_equal(f, f0)
    assert np.array_equal(f_sep, f0)
    assert abs(e0 - eo) <= 1e-12 * abs(eo)
    tol = ABS_TOL + (0.0 if precision == "fp64" else 1e-6 * np.abs(fo).max())
    assert np.abs(f0 - fo).max() <= tol


def test_minimization_reproducible(gpu_lib, oracle):
    """Two minimizations of the medium network (42k beads) from the same start
    take the same iterations and end on the same bits."""
    sv, x = net_of(oracle, 1)
    p = cgp(grad_tol=1.0, energy_rel_tol=1e-9, energy_call_limit=3000)
    out = []
    for _ in range(2):
        with ForceFieldManager("fp64") as ff:
            ff.vectorize_all_force_fields(sv)
            ff.set_deterministic(True)
            out.append(ff.minimize(x, p))
    (s0, x0, f0, r0), (s1, x1, f1, r1) = out
    assert s0 == s1 == 0
    assert (r0.num_iter, r0.num_energy_call, r0.num_force_call) == (r1.num_iter, r1.num_energy_call, r1.num_force_call)
    assert r0.num_iter > 50
    assert np.array_equal(x0, x1) and np.array_equal(f0, f1)
    assert r0.energy_after_total == r1.energy_after_total


def test_short_run_matches_oracle(gpu_lib, oracle):
    base = dict(n_fil=12, cyl_per_fil=6, box=700.0, n_linker=16, seed=3)
    net = make_workload(0, **base)
    st, extra = oracle.complete(net)
    sv, x = net.system_view(**extra), net.flat_coords()
    p = cgp(grad_tol=1e-4, energy_rel_tol=1e-14, energy_call_limit=40)
    so, xo, fo, ro = oracle.minimize(sv, x, p)
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(sv)
        ff.set_deterministic(True)
        sg, xg, fg, rg = ff.minimize(x, p)
    assert sg == so == 0
    assert (rg.num_energy_call, rg.num_force_call, rg.num_iter) == (ro.num_energy_call, ro.num_force_call, ro.num_iter)
    assert np.abs(xg - xo).max() <= 1e-7


def test_out_of_range_contribution_is_reported(gpu_lib):
    # a spring stretched far from rest with a huge constant: 1e12 pN/nm * 10 nm
    sv = SystemView(2, stretch_beads=[0, 3], stretch_k=[1e12], stretch_l0=[10.0])
    x = np.array([0.0, 0.0, 0.0, 20.0, 0.0, 0.0])
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(sv)
        e, per, f = ff.evaluate(x)  # floating-point sums: fine
        assert np.isfinite(f).all() and np.abs(f).max() == pytest.approx(1e13)
        ff.set_deterministic(True)
        st = ff.lib.medyan_mech_evaluate(ff.handle, *_args(x))
        assert st == 3  # MEDYAN_ERR_NONFINITE
        ff.set_deterministic(False)
        e2, per2, f2 = ff.evaluate(x)
        assert np.array_equal(f2, f)


def _args(x):
    import ctypes as C
    pd = C.POINTER(C.c_double)
    xx = np.ascontiguousarray(x, np.float64)
    f = np.zeros_like(xx)
    per = np.zeros(10)
    tot = C.c_double()
    _args.keep = (xx, f, per, tot)
    return xx.ctypes.data_as(pd), C.byref(tot), per.ctypes.data_as(pd), f.ctypes.data_as(pd)
