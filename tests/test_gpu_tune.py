"""Launch shapes and the autotuner (medyan_mech_set_shapes / autotune): every
shape gives the oracle's energies and forces (FP64 1e-12, as
test_gpu_forcefield), the minimizer keeps its call counts, and the
autotuner returns one of the allowed shapes and leaves a working handle."""
import itertools

import numpy as np
import pytest

from medyan_b200.forcefield import ForceFieldManager, conjugate_gradient_params as cgp
from medyan_b200.lib import MedyanError
from medyan_b200.network import make_workload

pytestmark = pytest.mark.gpu


def net(oracle):
    n = make_workload(0, n_fil=12, cyl_per_fil=6, box=700.0, n_linker=16, seed=3)
    st, extra = oracle.complete(n)
    assert st == 0
    return n.system_view(**extra), n.flat_coords()


def close(e, f, eo, fo):
    assert abs(e - eo) <= 1e-12 * abs(eo)
    assert np.abs(f - fo).max() <= 1e-12 * np.abs(fo).max()


SHAPES = [dict(bonded_threads=b, excl_threads=x, chain_threads=c, chain_energy_blocks_per_sm=g, pass_layout=p)
          for b, x, c, g, p in [(128, 32, 128, 2, 1), (512, 128, 512, 8, 0), (256, 64, 256, 4, 1),
                                (128, 128, 512, 2, 0), (256, 32, 256, 4, 0), (256, 64, 256, 4, 2),
                                (512, 128, 128, 2, 2)]]


@pytest.mark.parametrize("shape", SHAPES)
def test_shapes_match_oracle(gpu_lib, oracle, shape):
    sv, x = net(oracle)
    eo, _ = oracle.energy(sv, x)
    fo = oracle.forces(sv, x)
    p = cgp(grad_tol=1e-4, energy_rel_tol=1e-14, energy_call_limit=30)
    so, xo, _, ro = oracle.minimize(sv, x, p)
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(sv)
        ff.set_shapes(**shape)
        assert ff.get_shapes() == shape
        e, per, f = ff.evaluate(x)
        close(e, f, eo, fo)
        sg, xg, fg, rg = ff.minimize(x, p)
    assert (rg.num_energy_call, rg.num_force_call) == (ro.num_energy_call, ro.num_force_call)
    assert np.abs(xg - xo).max() <= 1e-7


def test_autotune(gpu_lib, oracle):
    sv, x = net(oracle)
    eo, _ = oracle.energy(sv, x)
    fo = oracle.forces(sv, x)
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(sv)
        ff.set_coords(x)
        chosen = ff.autotune(reps=5)
        assert chosen == ff.get_shapes()
        assert chosen["bonded_threads"] in (128, 256, 512) and chosen["excl_threads"] in (32, 64, 128)
        assert chosen["chain_threads"] in (128, 256, 512) and chosen["chain_energy_blocks_per_sm"] in (2, 4, 8)
        assert chosen["pass_layout"] in (0, 1, 2)
        e, per, f = ff.evaluate(x)
        close(e, f, eo, fo)
        with pytest.raises(MedyanError):
            ff.set_shapes(bonded_threads=100)
