"""Pins the CPU oracle to the reference.

- bit-for-bit against the reference's own sources built with strict rounding
  (tests/golden fixtures, and the live build when present);
- within 1e-12 relative of the reference's production build (-ffast-math);
- the properties the reference's own unit tests assert (excluded-volume
  scaling, energy/force consistency, CG convergence on the harmonic problem).
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

from medyan_b200._abi import SystemView, f64
from oracle.oracle import Oracle, Reference, cg_params

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def unit():
    with open(os.path.join(GOLDEN, "reference_unit_inputs.json")) as fh:
        return json.load(fh)


@pytest.fixture(scope="module")
def nets():
    return dict(np.load(os.path.join(GOLDEN, "synthetic_networks.npz")))


def unit_systems(unit):
    """(name, SystemView, coord) for every unit-test input."""
    ex = unit["excl"]
    out = []
    for name, c in ex["consistency"].items():
        out.append(("excl_" + name, SystemView(len(c["coord"]) // 3, excl_beads=c["beads"], excl_k=c["k"],
                                               excl_eqlen=c["eqlen"]), c["coord"]))
    st = ex["stress_20210901"]
    out.append(("excl_stress", SystemView(len(st["coord"]) // 3, excl_beads=st["beads"], excl_k=st["k"],
                                          excl_eqlen=st["eqlen"]), st["coord"]))
    dh = unit["dihedral"]
    nb = len(dh["pos"])
    out.append(("dihedral", SystemView(len(dh["coord"]) // 3, branch_beads=[3 * i for i in range(4 * nb)],
                                       branch_pos=dh["pos"], branch_dihedral_k=dh["k"], branch_ff_mask=4),
                dh["coord"]))
    ps = unit["position"]
    beads = []
    for i in range(len(ps["pos"])):
        beads += [9 * i, 9 * i + 3, 9 * i + 6, 9 * i + 6]
    out.append(("position", SystemView(len(ps["coord"]) // 3, branch_beads=beads, branch_pos=ps["pos"],
                                       branch_position_k=ps["k"], branch_ff_mask=8), ps["coord"]))
    bd = unit["boundary"]
    out.append(("boundary", SystemView(len(bd["coord"]) // 3, boundary_beads=bd["beads"], boundary_k=bd["k"],
                                       boundary_slen=bd["slen"], plane_eq=bd["plane"],
                                       plane_nneighbors=bd["nneighbors"]), bd["coord"]))
    return out


def network_system(nets, tag):
    keys = [k.split("/", 1)[1] for k in nets if k.startswith(tag + "/") and k.count("/") == 1]
    arrays = {k: nets[f"{tag}/{k}"] for k in keys if k not in ("n_beads", "coord", "branch_ff_mask")}
    arrays["branch_ff_mask"] = int(nets[f"{tag}/branch_ff_mask"][0])
    return SystemView(int(nets[f"{tag}/n_beads"][0]), **arrays), nets[f"{tag}/coord"]


def test_unit_inputs_bitwise_vs_strict_reference(oracle, unit):
    for name, sv, x in unit_systems(unit):
        ref = unit["results"]["strict"][name]
        e, per = oracle.energy(sv, x)
        f = oracle.forces(sv, x)
        assert e == ref["energy"], name
        assert np.array_equal(f, np.asarray(ref["force"])), name


def test_unit_inputs_vs_reference_build(oracle, unit):
    for name, sv, x in unit_systems(unit):
        ref = unit["results"]["reference"][name]
        e, _ = oracle.energy(sv, x)
        f = oracle.forces(sv, x)
        fr = np.asarray(ref["force"])
        # the 2021-09-01 near-coplanar fixture is ill-conditioned: the reference's
        # own fast-math and strict builds differ by ~1e-5 there
        tol = 1e-4 if name == "excl_stress" else 1e-12
        assert abs(e - ref["energy"]) <= tol * abs(ref["energy"]), name
        assert np.abs(f - fr).max() <= tol * np.abs(fr).max(), name


@pytest.mark.parametrize("tag", ["cfg0", "branched"])
def test_synthetic_networks(oracle, nets, tag):
    sv, x = network_system(nets, tag)
    e, per = oracle.energy(sv, x)
    f = oracle.forces(sv, x)
    assert e == nets[f"{tag}/strict/energy"][0]
    assert np.array_equal(per, nets[f"{tag}/strict/per_ff"])
    assert np.array_equal(f, nets[f"{tag}/strict/force"])
    fr = nets[f"{tag}/reference/force"]
    assert abs(e - nets[f"{tag}/reference/energy"][0]) <= 1e-12 * abs(e)
    assert np.abs(f - fr).max() <= 1e-12 * np.abs(fr).max()


def test_excl_scaling(oracle, unit):
    # TestCylinderExclVolume.cpp:13-47: one pair equals the sum over sub-segment pairs
    sc = unit["excl"]["scaling"]
    n = len(sc["coord"]) // 3
    e0, _ = oracle.energy(SystemView(n, excl_beads=sc["beads0"], excl_k=sc["k0"], excl_eqlen=sc["eqlen0"]),
                          sc["coord"])
    e1, _ = oracle.energy(SystemView(n, excl_beads=sc["beads1"], excl_k=sc["k1"], excl_eqlen=sc["eqlen1"]),
                          sc["coord"])
    assert e0 == pytest.approx(e1, rel=1e-12)
    assert e0 == unit["results"]["strict"]["excl_scaling"]["energy0"]


def consistency_passes(energy, forces, x, rng, move_mag=1e-5, rel_eps=5e-4, reps=10):
    """testEnergyForceConsistency (TestFFCommon.hpp:101-170): E(c+dc) - E(c-dc) ~ -2 dc.F(c)."""
    x = f64(x)
    passed = 0
    for _ in range(reps):
        dc = rng.normal(0.0, move_mag, x.size)
        de = energy(x + dc) - energy(x - dc)
        de_exp = -2.0 * np.dot(dc, forces(x))
        if abs(de - de_exp) <= min(abs(de), abs(de_exp)) * rel_eps:
            passed += 1
    return passed


def test_energy_force_consistency(oracle, unit):
    # same moveMag / relEps / 9-of-10 rule as the reference's tests; the
    # near-coplanar stress fixture is excluded, as the reference disables it
    rng = np.random.default_rng(1)
    for name, sv, x in unit_systems(unit):
        if name == "excl_stress":
            continue
        n = consistency_passes(lambda c: oracle.energy(sv, c)[0], lambda c: oracle.forces(sv, c), x, rng)
        assert n >= 9, name


# --------------------------------------------------------------- CG pins
_EFN = C.CFUNCTYPE(C.c_double, C.c_void_p, C.POINTER(C.c_double))
_FFN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double))
_IFN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double))


def harmonic_callbacks(opt, w):
    """TestCGMethod.cpp:17-40: E = sum 0.5 w_i (x_i - opt_i)^2, F = -w (x - opt)."""
    n = len(opt)

    def energy(_, x):
        en = 0.0
        for i in range(n):
            en += 0.5 * w[i] * (x[i] - opt[i]) * (x[i] - opt[i])
        return en

    def forces(_, x, f):
        for i in range(n):
            f[i] = -w[i] * (x[i] - opt[i])

    def individual(_, x, per):
        per[0] = energy(None, x)

    return _EFN(energy), _FFN(forces), _IFN(individual)


def run_cb(lib, fname, n, params, x0, cbs):
    from medyan_b200._abi import MinResult
    x = f64(x0).copy()
    f = np.zeros(n)
    r = MinResult()
    fn = getattr(lib, fname)
    fn.restype = C.c_int32
    st = fn(C.c_int32(n), C.c_int32(0), C.byref(params), x.ctypes.data_as(C.POINTER(C.c_double)),
            f.ctypes.data_as(C.POINTER(C.c_double)), C.byref(r), *cbs, None)
    return st, x, f, r


@pytest.mark.parametrize("line_search", [0, 1])
@pytest.mark.parametrize("method", [0, 1, 2])
def test_cg_harmonic(oracle, unit, method, line_search):
    cg = unit["cg_harmonic"]
    p = cg_params(method=method, grad_tol=cg["params"]["gradTol"], max_dist=cg["params"]["maxDist"],
                  lambda_max=cg["params"]["lambdaMax"], try_to_recover=0, line_search=line_search)
    cbs = harmonic_callbacks(cg["opt"], cg["weight"])
    strict = Reference(strict=True) if Reference.available(strict=True) else None
    for init in cg["inits"]:
        st, x, f, r = run_cb(oracle.lib, "oracle_cg_minimize_cb", cg["n"], p, init, cbs)
        assert st == 0 and r.error_flags == 0
        assert np.all(np.abs(f) <= cg["params"]["gradTol"])
        # QUADRATIC: the reference's quadraticLineSearchV2 evaluates each trial
        # at a stale coordLineSearch (test_quadratic_reference_defect); the
        # oracle restates the algorithm as written and is checked alone
        if strict is not None and line_search == 0:
            st2, x2, f2, r2 = run_cb(strict.lib, "medyan_ref_cg_minimize_cb", cg["n"], p, init, cbs)
            assert st2 == st and np.array_equal(x, x2) and np.array_equal(f, f2)
            assert (r.num_energy_call, r.num_force_call) == (r2.num_energy_call, r2.num_force_call)


@pytest.mark.skipif(not Reference.available(strict=True), reason="reference build not present")
def test_cg_trajectory_bitwise_vs_strict_reference(oracle, nets):
    sv, x = network_system(nets, "cfg0")
    p = cg_params(grad_tol=1.0)
    st, xo, fo, ro = oracle.minimize(sv, x, p)
    st2, xr, fr, rr = Reference(strict=True).minimize(sv, x, p)
    assert st == st2 == 0
    assert np.array_equal(xo, xr) and np.array_equal(fo, fr)
    assert (ro.num_energy_call, ro.num_force_call) == (rr.num_energy_call, rr.num_force_call)
    assert ro.energy_after_total == rr.energy_after_total


def test_quadratic_line_search_converges(oracle, nets):
    """QUADRATIC (quadraticLineSearchV2 + quadraticoptimization, CGMethod.hpp:521-765)
    as written: every accepted step lowers the energy and the run converges."""
    sv, x = network_system(nets, "cfg0")
    e0, _ = oracle.energy(sv, x)
    st, xo, fo, ro = oracle.minimize(sv, x, cg_params(grad_tol=1.0, line_search=1))
    assert st == 0 and ro.error_flags == 0
    assert np.abs(fo).max() < 1.0
    # the soft network stops at gradTol = 1 pN on a plateau: the backtracking
    # run from the same start ends within a few percent of the same energy
    st_b, xb, _, rb = oracle.minimize(sv, x, cg_params(grad_tol=1.0))
    assert st_b == 0 and ro.energy_after_total < 0.6 * e0
    assert abs(ro.energy_after_total - rb.energy_after_total) <= 0.05 * abs(rb.energy_after_total)


@pytest.mark.skipif(not Reference.available(strict=True), reason="reference build not present")
def test_quadratic_reference_defect(oracle, unit):
    """The reference's quadraticLineSearchV2 calls moveAlongSearchDir(coord, lambda)
    (coord += lambda*d, in place) and then energyFunc(coordLineSearch), a buffer
    it never fills: every trial sees the same stale energy, the Armijo test
    cannot pass, and the first line search returns lambda = 0 after moving
    coord by the sum of the trial steps. Pinned here on the harmonic problem
    of TestCGMethod.cpp so the difference from the oracle stays documented."""
    cg = unit["cg_harmonic"]
    p = cg_params(method=2, grad_tol=cg["params"]["gradTol"], max_dist=cg["params"]["maxDist"],
                  lambda_max=cg["params"]["lambdaMax"], try_to_recover=0, line_search=1)
    cbs = harmonic_callbacks(cg["opt"], cg["weight"])
    init = cg["inits"][0]
    st, x, f, r = run_cb(oracle.lib, "oracle_cg_minimize_cb", cg["n"], p, init, cbs)
    st2, x2, f2, r2 = run_cb(Reference(strict=True).lib, "medyan_ref_cg_minimize_cb", cg["n"], p, init, cbs)
    assert st == 0 and r.error_flags == 0
    assert r2.error_flags & 1  # errorLineSearch


@pytest.mark.skipif(not Reference.available(strict=True), reason="reference build not present")
def test_lambda_running_average_is_a_no_op(oracle):
    """ConjugateGradientParams::lambdaRunningAverageProbability. CGMethod::minimize
    creates a new LambdaRunningAverageManager in every iteration
    (Mechanics/Minimizer/CGMethod.hpp:1316-1317) and the line search records
    into it once (CGMethod.hpp:363-366); the manager's status, which alone
    lets it cap lambda, changes only when its tenth record arrives
    (LineSearch.hpp:33-42), so it never does, and no random number is drawn.
    Any probability gives the trajectory of 0: checked here on the
    reference's own compiled CGMethod with probability 1."""
    import ctypes as C
    from medyan_b200.forcefield import conjugate_gradient_params as cgp
    from medyan_b200.network import make_workload
    ref = Reference(strict=True)
    ref.lib.medyan_ref_set_lambda_running_average.argtypes = [C.c_double]
    ref.lib.medyan_ref_set_lambda_running_average.restype = None
    net = make_workload(0, n_fil=12, cyl_per_fil=6, box=700.0, n_linker=16, seed=3)
    st, extra = oracle.complete(net)
    sv, x = net.system_view(**extra), net.flat_coords()
    p = cgp(grad_tol=1.0)
    runs = []
    for prob in (0.0, 1.0):
        ref.lib.medyan_ref_set_lambda_running_average(prob)
        runs.append(ref.minimize(sv, x, p))
    ref.lib.medyan_ref_set_lambda_running_average(0.0)
    (s0, x0, f0, r0), (s1, x1, f1, r1) = runs
    assert s0 == s1
    assert (r0.num_iter, r0.num_energy_call, r0.num_force_call) == (r1.num_iter, r1.num_energy_call, r1.num_force_call)
    # the reference reports no iteration count; one force call per iteration
    assert r0.num_force_call > 10  # enough line searches that a persistent manager would have acted
    assert np.array_equal(x0, x1) and r0.energy_after_total == r1.energy_after_total
