"""Beads in any order. The library keeps its own internal bead order
(filament chains contiguous, fixed at create) and converts at the C ABI. A
network whose bead labels are shuffled must give the oracle's energies,
forces, minimization and neighbor-list interactions on that labelling, and
the same physics as the unshuffled network."""
import numpy as np
import pytest

from medyan_b200._abi import CylindersView, SystemView
from medyan_b200.forcefield import ForceFieldManager, conjugate_gradient_params as cgp
from medyan_b200.network import make_workload

pytestmark = pytest.mark.gpu

BEAD_FIELDS = ("stretch_beads", "bend_beads", "linker_beads", "motor_beads", "branch_beads", "excl_beads",
               "boundary_beads")


def relabel(net, extra, seed):
    """The network with bead b renamed perm[b]."""
    perm = np.random.default_rng(seed).permutation(net.n_beads)
    arrays = dict(net.ff)
    arrays.update(extra)
    out = {k: (3 * perm[np.asarray(v, np.int64) // 3] if k in BEAD_FIELDS and v is not None else v)
           for k, v in arrays.items()}
    x = net.flat_coords().reshape(-1, 3)
    xn = np.empty_like(x)
    xn[perm] = x
    return SystemView(net.n_beads, **out), xn.reshape(-1), perm


def shuffled(oracle, cfg=1, seed=1):
    net = make_workload(cfg, seed=seed)
    st, extra = oracle.complete(net)
    assert st == 0
    sv, x, perm = relabel(net, extra, seed + 100)
    return net, extra, sv, x, perm


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_energy_and_forces(gpu_lib, oracle, precision):
    net, extra, sv, x, perm = shuffled(oracle)
    eo, pero = oracle.energy(sv, x)
    fo = oracle.forces(sv, x)
    with ForceFieldManager(precision) as ff:
        ff.vectorize_all_force_fields(sv)
        e, per, f = ff.evaluate(x)
        xg = ff.get_coords()
    tol = 1e-12 if precision == "fp64" else 1e-6
    assert abs(e - eo) <= 1e-12 * abs(eo)
    assert np.abs(f - fo).max() <= tol * np.abs(fo).max()
    assert np.array_equal(xg, x)
    # the same physics as the original labelling
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(net.system_view(**extra))
        e0, _, f0 = ff.evaluate(net.flat_coords())
    assert abs(e - e0) <= 1e-12 * abs(e0)
    assert np.abs(f.reshape(-1, 3)[perm] - f0.reshape(-1, 3)).max() <= tol * np.abs(f0).max()


def test_short_minimization(gpu_lib, oracle):
    net, extra, sv, x, perm = shuffled(oracle, cfg=0, seed=3)
    p = cgp(grad_tol=1e-4, energy_rel_tol=1e-14, energy_call_limit=40)
    so, xo, fo, ro = oracle.minimize(sv, x, p)
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(sv)
        sg, xg, fg, rg = ff.minimize(x, p)
    assert sg == so == 0
    assert (rg.num_energy_call, rg.num_force_call, rg.num_iter) == (ro.num_energy_call, ro.num_force_call, ro.num_iter)
    assert np.abs(xg - xo).max() <= 1e-7
    assert abs(rg.energy_after_total - ro.energy_after_total) <= 1e-10 * abs(ro.energy_after_total)
    assert np.abs(fg - fo).max() <= 1e-7 * np.abs(fo).max()


def test_neighbor_list(gpu_lib, oracle):
    net, extra, sv, x, perm = shuffled(oracle)
    no_excl = {k: v for k, v in sv.arrays.items() if not k.startswith(("excl_", "boundary_", "plane_"))}
    cvn = CylindersView(perm[net.cyl_bead1], perm[net.cyl_bead2], net.cyl_id, net.cyl_fil, net.cyl_pos,
                        net.cyl_type, net.cyl_branching, net.cyl_minus_end, net.cyl_eqlen, net.cyl_exclk)
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(SystemView(net.n_beads, branch_ff_mask=sv.branch_ff_mask, **no_excl))
        ff.set_coords(x)
        bp, planes = net.boundary_params()
        ff.set_cylinders(cvn, net.nl_params(), bp)
        ne, nbd = ff.rebuild_neighbor_lists()
        beads, krs, _ = ff.excluded_volume_interactions()
        e, per, f = ff.evaluate(x)
    want = sorted(map(tuple, sv.arrays["excl_beads"].reshape(-1, 4).tolist()))
    assert ne == len(want) and nbd == sv.arrays["boundary_beads"].size
    assert sorted(map(tuple, beads.tolist())) == want
    eo, _ = oracle.energy(sv, x)
    fo = oracle.forces(sv, x)
    assert abs(e - eo) <= 1e-12 * abs(eo)
    assert np.abs(f - fo).max() <= 1e-12 * np.abs(fo).max()
