"""How far apart two valid minimizations of a filament network can end.

The oracle is the reference's CGMethod bit for bit (tests/test_oracle_pins.py).
Started from coordinates that differ by one ulp, it converges on the gradient
(max|F| < gradTol) on every network here, yet to minima whose energies differ
by 1e-4 to 1e-2 relative: the landscape is rough, and trajectories that
differ in the last bit separate. This bounds any comparison of final
energies between precisions or summation orders; the device tests of
converged minimizations use bounds taken from here."""
import numpy as np
import pytest

from medyan_b200.forcefield import conjugate_gradient_params as cgp
from medyan_b200.network import make_workload

NETS = [("12x6", dict(n_fil=12, cyl_per_fil=6, box=700.0, n_linker=16, seed=3)),
        ("30x8", dict(n_fil=30, cyl_per_fil=8, box=1000.0, n_linker=60, seed=11)),
        ("cfg0", {})]


@pytest.mark.parametrize("name,kw", NETS)
def test_one_ulp_start_changes_the_minimum(oracle, name, kw):
    net = make_workload(0, **kw)
    st, extra = oracle.complete(net)
    assert st == 0
    sv, x = net.system_view(**extra), net.flat_coords()
    p = cgp(grad_tol=1.0)
    sa, xa, fa, ra = oracle.minimize(sv, x, p)
    sb, xb, fb, rb = oracle.minimize(sv, np.nextafter(x, np.inf), p)
    assert sa == sb == 0
    # both converge on the gradient criterion
    assert ra.grad_inf_norm < 1.0 and rb.grad_inf_norm < 1.0
    rel = abs(ra.energy_after_total - rb.energy_after_total) / abs(ra.energy_after_total)
    # measured: 1.7e-4 (12x6), 1.4e-2 (30x8), 3.6e-3 (cfg0)
    assert 1e-6 < rel < 5e-2, rel
