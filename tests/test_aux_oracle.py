"""The oracle's restatements of the after-minimization quantities on CPU:
BoundaryCylinderRepulsion::computeLoadForces (BoundaryCylinderRepulsion.cpp:125-196)
against its closed form for a filament facing one plane, and the force
magnitudes of assignallforcemags (ForceFieldManager.cpp:346-351) against
the tensions and forces they stand for."""
import numpy as np

from tests.aux_nets import tip_network


def test_load_forces_closed_form(oracle):
    sv, x, cv, nlp, bp, planes, tips, plus = tip_network(seed=1, n_fil=3)
    n_mon, mon = np.full(len(tips), 40), np.full(len(tips), 2.7)
    loads = oracle.boundary_load_forces(cv, x, bp, tips, plus, n_mon, mon)
    xb = x.reshape(-1, 3)
    for t, (c, p) in enumerate(zip(tips, plus)):
        b1, b2 = cv.arrays["bead1"][c], cv.arrays["bead2"][c]
        bo, bd = (xb[b1], xb[b2]) if p else (xb[b2], xb[b1])
        d = (bd - bo) / np.linalg.norm(bd - bo)
        mid = 0.5 * (xb[b1] + xb[b2])
        want = np.zeros(40)
        for pl in planes.reshape(-1, 4):
            if not (pl[:3] @ mid + pl[3]) / np.linalg.norm(pl[:3]) < 300.0:
                continue
            proj = max(-(pl[:3] @ d), 0.0)
            for i in range(40):
                q = bd + i * 2.7 * d
                r = (pl[:3] @ q + pl[3]) / np.linalg.norm(pl[:3])
                want[i] += proj * 41.0 * np.exp(-r / 2.7) / 2.7
        assert np.allclose(loads[t], want, rtol=1e-12, atol=0), t
    # the plus tips of filaments growing towards a plane feel a load
    assert any(l[0] > 1e-3 for l in loads[:3])


def test_force_magnitudes_meaning(oracle):
    rng = np.random.default_rng(2)
    from medyan_b200._abi import SystemView
    x = rng.uniform(0, 100, size=(8, 3)).reshape(-1)
    sv = SystemView(8, linker_beads=[[0, 3, 6, 9]], linker_k=[5.0], linker_l0=[30.0], linker_pos1=[0.25],
                    linker_pos2=[0.75], motor_beads=[[12, 15, 18, 21]], motor_k=[2.0], motor_l0=[10.0],
                    motor_pos1=[0.5], motor_pos2=[0.1])
    lin, mot, br = oracle.force_magnitudes(sv, x)
    xb = x.reshape(-1, 3)
    v1, v2 = 0.75 * xb[0] + 0.25 * xb[1], 0.25 * xb[2] + 0.75 * xb[3]
    assert np.isclose(lin[0], 5.0 * (np.linalg.norm(v2 - v1) - 30.0), rtol=1e-13)
    v1, v2 = 0.5 * xb[4] + 0.5 * xb[5], 0.9 * xb[6] + 0.1 * xb[7]
    assert np.isclose(mot[0], 2.0 * (np.linalg.norm(v2 - v1) - 10.0), rtol=1e-13)
    assert br.shape == (0, 3)
