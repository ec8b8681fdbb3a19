"""Derivatives (medyan_mech_param_grad, medyan_mech_hvp) against finite
differences of the oracle's FP64 energy and forces, and an implicit-adjoint
sensitivity of a minimized network, d L(x*) / d theta, wrapped in a
torch.autograd.Function here in the tests, against differences of
re-minimized networks.

The Hessian-vector product and the directional parameter gradient are
forward mode on the device (exact to rounding), so they are checked against
Richardson-extrapolated central differences: D(h) = (f(x + h v) - f(x - h v))
/ 2h, R = (4 D(h) - D(2h)) / 3, whose truncation error is O(h^4)."""
import numpy as np
import pytest

from medyan_b200._abi import SystemView
from medyan_b200.forcefield import ForceFieldManager, conjugate_gradient_params as cgp
from medyan_b200.network import make_workload

pytestmark = pytest.mark.gpu

FF_STRETCH, FF_BEND, FF_LINKER, FF_MOTOR, FF_EXCL, FF_BOUNDARY = 0, 1, 2, 3, 8, 9


def diff_net_moved(oracle):
    """diff_net with the beads moved off the generated geometry (straight
    filaments and linkers at their rest length make several gradients
    vanish)."""
    arrays, nb, x = diff_net(oracle)
    return arrays, nb, x + np.random.default_rng(5).normal(0, 0.5, x.size)


def diff_net(oracle):
    # the differentiation workload's composition at reduced size: 80 x 20
    # cylinders, 160 linkers, 16 motors in a 3 um cube, with excluded volume
    # and boundary repulsion
    net = make_workload(3, seed=3, n_fil=80, n_linker=160, n_motor=16)
    st, extra = oracle.complete(net)
    assert st == 0
    arrays = dict(net.ff)
    arrays.update(extra)
    return arrays, net.n_beads, net.flat_coords()


def scaled(arrays, n_beads, key, h, per=None):
    a = dict(arrays)
    v = np.array(a[key], float)
    if per is None:
        v = v * (1.0 + h)
    else:
        v[per] += h
    a[key] = v
    return SystemView(n_beads, **a)


# (force-field slot, parameter array, which output)
CASES = [(FF_STRETCH, "stretch_k", 0), (FF_STRETCH, "stretch_l0", 1), (FF_BEND, "bend_k", 0),
         (FF_LINKER, "linker_k", 0), (FF_LINKER, "linker_l0", 1), (FF_MOTOR, "motor_k", 0),
         (FF_MOTOR, "motor_l0", 1), (FF_BOUNDARY, "boundary_k", 0), (FF_BOUNDARY, "boundary_slen", 1)]


@pytest.mark.parametrize("slot,key,which", CASES)
def test_param_grad_vs_fd(gpu_lib, oracle, slot, key, which):
    arrays, nb, x = diff_net_moved(oracle)
    n = np.asarray(arrays[key]).size
    assert n > 0
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(SystemView(nb, **arrays))
        ff.set_coords(x)
        g = ff.param_grad(slot, n)[which]
    theta = np.asarray(arrays[key], float)
    # differences of this force field's own energy (the total is dominated by
    # others and would bury the difference in its rounding)
    # scaling every parameter of the type: d/ds E(theta (1 + s)) = sum theta_i dE/dtheta_i
    h = 1e-6
    ep = oracle.energy(scaled(arrays, nb, key, h), x)[1][slot]
    em = oracle.energy(scaled(arrays, nb, key, -h), x)[1][slot]
    fd = (ep - em) / (2 * h)
    an = float(np.dot(theta, g))
    assert abs(an - fd) <= 1e-6 * abs(fd) + 1e-12, (an, fd)
    # one interaction at a time
    for i in np.random.default_rng(0).choice(n, size=min(3, n), replace=False):
        hi = 1e-6 * max(abs(theta[i]), 1.0)
        ep = oracle.energy(scaled(arrays, nb, key, hi, per=i), x)[1][slot]
        em = oracle.energy(scaled(arrays, nb, key, -hi, per=i), x)[1][slot]
        fdi = (ep - em) / (2 * hi)
        assert abs(g[i] - fdi) <= 1e-5 * abs(fdi) + 1e-9, (i, g[i], fdi)


BRANCH_CASES = [(4, "branch_stretch_k", 0), (4, "branch_stretch_l0", 1), (5, "branch_bend_k", 0),
                (5, "branch_bend_theta0", 1), (6, "branch_dihedral_k", 0), (7, "branch_position_k", 0)]


def branched_net(oracle):
    net = make_workload(1, n_fil=80, cyl_per_fil=8, box=1600.0, n_linker=60, n_motor=12, n_branch=16,
                        br_position_k=20.0)
    st, extra = oracle.complete(net)
    assert st == 0
    arrays = dict(net.ff)
    arrays.update(extra)
    x = net.flat_coords() + np.random.default_rng(9).normal(0, 0.3, net.n_beads * 3)
    return arrays, net.n_beads, x


@pytest.mark.parametrize("slot,key,which", BRANCH_CASES)
def test_branching_param_grad_vs_fd(gpu_lib, oracle, slot, key, which):
    """dE/dtheta of the four branching potentials (BranchingStretchingHarmonic,
    BranchingBendingCosine, BranchingDihedralCosine, BranchingPositionCosine)
    against central differences of that force field's oracle energy."""
    arrays, nb, x = branched_net(oracle)
    n = np.asarray(arrays[key]).size
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(SystemView(nb, **arrays))
        ff.set_coords(x)
        g = ff.param_grad(slot, n)[which]
    theta = np.asarray(arrays[key], float)
    for i in range(n):
        hi = 1e-6 * max(abs(theta[i]), 1.0)
        ep = oracle.energy(scaled(arrays, nb, key, hi, per=i), x)[1][slot]
        em = oracle.energy(scaled(arrays, nb, key, -hi, per=i), x)[1][slot]
        fdi = (ep - em) / (2 * hi)
        assert abs(g[i] - fdi) <= 1e-6 * max(abs(fdi), 1e-3), (i, g[i], fdi)


def test_bending_theta0_and_excluded_volume(gpu_lib, oracle):
    arrays, nb, x = diff_net_moved(oracle)
    arrays["bend_theta0"] = np.full(np.asarray(arrays["bend_k"]).size, 0.1)
    nbend = arrays["bend_theta0"].size
    nex = np.asarray(arrays["excl_k"]).size
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(SystemView(nb, **arrays))
        ff.set_coords(x)
        gk, gt = ff.param_grad(FF_BEND, nbend)
        ge, _ = ff.param_grad(FF_EXCL, nex)
    h = 1e-6
    ep = oracle.energy(scaled(arrays, nb, "bend_theta0", h), x)[1][FF_BEND]
    em = oracle.energy(scaled(arrays, nb, "bend_theta0", -h), x)[1][FF_BEND]
    fd = (ep - em) / (2 * h)
    assert abs(0.1 * gt.sum() - fd) <= 1e-6 * abs(fd)
    # excluded volume: d_k = dE/dkRS; scaling krep scales kRS
    krs = np.asarray(arrays["excl_k"]) * np.asarray(arrays["excl_eqlen"]).reshape(-1, 2).prod(axis=1)
    ep = oracle.energy(scaled(arrays, nb, "excl_k", h), x)[1][FF_EXCL]
    em = oracle.energy(scaled(arrays, nb, "excl_k", -h), x)[1][FF_EXCL]
    fd = (ep - em) / (2 * h)
    assert abs(np.dot(krs, ge) - fd) <= 1e-6 * abs(fd)


def richardson(f, x, v, h):
    """(4 D(h) - D(2h)) / 3 of f along v, D the central difference."""
    d1 = (f(x + h * v) - f(x - h * v)) / (2 * h)
    d2 = (f(x + 2 * h * v) - f(x - 2 * h * v)) / (4 * h)
    return (4 * d1 - d2) / 3


@pytest.mark.parametrize("slot,key", [(FF_STRETCH, "stretch_k"), (FF_BEND, "bend_k"), (FF_LINKER, "linker_k"),
                                      (FF_MOTOR, "motor_k"), (FF_EXCL, "excl_k"), (FF_BOUNDARY, "boundary_k")])
def test_param_grad_directional(gpu_lib, oracle, slot, key):
    """v . d2E/dx dtheta (forward mode) against differences of the analytic
    gradient along v."""
    arrays, nb, x = diff_net_moved(oracle)
    if slot == FF_BEND:
        arrays["bend_theta0"] = np.full(np.asarray(arrays["bend_k"]).size, 0.1)
    v = np.random.default_rng(1).normal(size=x.size)
    n = np.asarray(arrays[key]).size
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(SystemView(nb, **arrays))
        ff.set_coords(x)
        dk, dp = ff.param_grad(slot, n, v=v)

        def grads(xx):
            ff.set_coords(xx)
            return np.concatenate(ff.param_grad(slot, n))

        want = richardson(grads, x, v, 1e-3 / np.abs(v).max())
    got = np.concatenate([dk, dp])
    # bending: d sin(theta) = -cos d cos / sin is steep for nearly straight
    # filaments, which bounds what the differences resolve
    tol = 1e-6 if slot == FF_BEND else 1e-8
    assert np.abs(got - want).max() <= tol * np.abs(want).max(), np.abs(got - want).max() / np.abs(want).max()


def hvp_check(oracle, sv, x, seed, tol, sym_tol):
    """hv = -dF/dx v against Richardson differences of the oracle's forces
    along v (the definition), and u . Hv against v . Hu. The reference's
    forces are not the exact gradient of its energy everywhere (the
    excluded-volume force moves a bead out of plane when the two cylinders
    are near coplanar; the cosine potentials with theta0 != 0 rescale cos by
    0.999 near +-1), so the product is not exactly symmetric: sym_tol is the
    network's measured asymmetry with margin."""
    rng = np.random.default_rng(seed)
    u, v = rng.normal(size=x.size), rng.normal(size=x.size)
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(sv)
        ff.set_coords(x)
        hv, hu = ff.hvp(v), ff.hvp(u)
    want = -richardson(lambda xx: oracle.forces(sv, xx), x, v, 1e-3 / np.abs(v).max())
    err = np.abs(hv - want).max() / np.abs(want).max()
    asym = abs(u @ hv - v @ hu) / abs(u @ hv)
    assert err <= tol, (err, asym)
    assert asym <= sym_tol, (err, asym)


def test_hvp(gpu_lib, oracle):
    arrays, nb, x = diff_net(oracle)
    hvp_check(oracle, SystemView(nb, **arrays), x, 2, tol=1e-8, sym_tol=1e-6)


def test_hvp_differentiation_workload(gpu_lib, oracle):
    """The differentiation workload at full size: 500 filaments x 20
    cylinders, 1,000 linkers, 100 motors, excluded volume and boundary."""
    net = make_workload(3)
    st, extra = oracle.complete(net)
    assert st == 0
    hvp_check(oracle, net.system_view(**extra), net.flat_coords(), 6, tol=1e-8, sym_tol=1e-4)


def test_hvp_branched(gpu_lib, oracle):
    """Branch points with all four branching potentials (stretching, bending,
    dihedral, position)."""
    net = make_workload(1, n_fil=80, cyl_per_fil=8, box=1600.0, n_linker=60, n_motor=12, n_branch=16,
                        br_position_k=20.0)
    st, extra = oracle.complete(net)
    assert st == 0
    sv = net.system_view(**extra)
    assert sv.branch_ff_mask == 15
    x = net.flat_coords() + np.random.default_rng(9).normal(0, 0.3, net.n_beads * 3)
    hvp_check(oracle, sv, x, 8, tol=1e-8, sym_tol=1e-2)


def test_hvp_exact_for_springs(gpu_lib):
    # a random spring network: H is known in closed form
    rng = np.random.default_rng(3)
    nb = 40
    x = rng.uniform(0, 50, size=(nb, 3))
    pairs = np.array([(i, j) for i in range(nb) for j in range(i + 1, nb) if rng.random() < 0.1])
    k = rng.uniform(1, 10, len(pairs))
    l0 = np.linalg.norm(x[pairs[:, 1]] - x[pairs[:, 0]], axis=1) * rng.uniform(0.8, 1.2, len(pairs))
    H = np.zeros((3 * nb, 3 * nb))
    for (i, j), kk, ll in zip(pairs, k, l0):
        r = x[j] - x[i]
        L = np.linalg.norm(r)
        n = r / L
        B = kk * ((1 - ll / L) * np.eye(3) + (ll / L) * np.outer(n, n))
        for a, b, sgn in ((i, i, 1), (j, j, 1), (i, j, -1), (j, i, -1)):
            H[3 * a:3 * a + 3, 3 * b:3 * b + 3] += sgn * B
    sv = SystemView(nb, linker_beads=np.stack([3 * pairs[:, 0], 3 * pairs[:, 0], 3 * pairs[:, 1], 3 * pairs[:, 1]], 1),
                    linker_k=k, linker_l0=l0, linker_pos1=np.zeros(len(pairs)), linker_pos2=np.zeros(len(pairs)))
    v = rng.normal(size=3 * nb)
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(sv)
        ff.set_coords(x.reshape(-1))
        hv = ff.hvp(v)
    want = H @ v
    assert np.abs(hv - want).max() <= 1e-10 * np.abs(want).max()


# ------------------------------------------------------------ implicit adjoint
def adjoint_net():
    """Four filaments of five cylinders along the edges of a square prism,
    every pair braced by linkers between cylinder midpoints (rungs and
    diagonals): a stiff truss whose only zero modes are rigid motions, with a
    smooth energy (no excluded volume)."""
    rng = np.random.default_rng(4)
    nf, nc = 4, 5
    corners = [(100.0, 100.0), (130.0, 100.0), (100.0, 130.0), (130.0, 130.0)]
    xs, sb, bb = [], [], []
    for f, (cx, cz) in enumerate(corners):
        for b in range(nc + 1):
            xs.append(np.array([cx, 100.0 + 20.0 * b, cz]) + rng.normal(0, 0.5, 3))
        b0 = f * (nc + 1)
        sb += [(3 * (b0 + b), 3 * (b0 + b + 1)) for b in range(nc)]
        bb += [(3 * (b0 + b), 3 * (b0 + b + 1), 3 * (b0 + b + 2)) for b in range(nc - 1)]
    x = np.array(xs).reshape(-1)
    lb = []
    for f in range(nf):
        for g in range(f + 1, nf):
            for c in range(nc):
                for c2 in ((c, c + 1) if c + 1 < nc else (c,)):
                    a, b = f * (nc + 1) + c, g * (nc + 1) + c2
                    lb.append((3 * a, 3 * (a + 1), 3 * b, 3 * (b + 1)))
    nl = len(lb)
    base = dict(stretch_beads=np.array(sb), stretch_k=np.full(len(sb), 100.0), stretch_l0=np.full(len(sb), 20.0),
                bend_beads=np.array(bb), bend_k=np.full(len(bb), 672.0), bend_theta0=np.zeros(len(bb)),
                linker_beads=np.array(lb), linker_k=np.full(nl, 8.0), linker_l0=np.full(nl, 25.0),
                linker_pos1=np.full(nl, 0.5), linker_pos2=np.full(nl, 0.5))
    return base, nf * (nc + 1), x


def system_for(base, nb, s_k, s_l0):
    a = dict(base)
    a["linker_k"] = base["linker_k"] * (1.0 + s_k)
    a["linker_l0"] = base["linker_l0"] * (1.0 + s_l0)
    return SystemView(nb, **a)


CG_PARAMS = cgp(grad_tol=1e-3, energy_rel_tol=1e-13)


def minimized(base, nb, x0, s_k, s_l0):
    """The device minimizer, then Newton steps (forces, and Hessian solves by
    CG on the HVP) to push the residual force to rounding level, so that
    central differences of minimized coordinates resolve 1e-6."""
    with ForceFieldManager("fp64") as ff:
        ff.vectorize_all_force_fields(system_for(base, nb, s_k, s_l0))
        st, x, f, r = ff.minimize(x0, CG_PARAMS)
        assert st == 0, st
        for _ in range(10):
            f = ff.compute_forces(x)
            fn = np.abs(f).max()
            if fn < 1e-9:
                break
            step = cg_solve(ff.hvp, f, tol=1e-9, maxit=500)
            # damped: the truss's near-null rotation modes can make a full
            # Newton step overshoot; halve until the residual force drops
            t = 1.0
            while True:
                xt = x + t * step
                if np.abs(ff.compute_forces(xt)).max() < fn or t < 1e-6:
                    break
                t *= 0.5
            x = xt
        assert np.abs(ff.compute_forces(x)).max() < 1e-7
    return x


def loss(x):
    # squared distance between the first bead of filament 0 and the last bead
    # of filament 3 (across the prism)
    return float(np.sum((x[-3:] - x[0:3]) ** 2))


def cg_solve(hvp, b, tol=1e-10, maxit=2000):
    lam = np.zeros_like(b)
    r = b.copy()
    p = r.copy()
    rr = r @ r
    for _ in range(maxit):
        hp = hvp(p)
        a = rr / (p @ hp)
        lam += a * p
        r -= a * hp
        rn = r @ r
        if np.sqrt(rn) <= tol * np.linalg.norm(b):
            break
        p = r + (rn / rr) * p
        rr = rn
    return lam


def test_implicit_adjoint_autograd(gpu_lib):
    torch = pytest.importorskip("torch")
    base, nb, x0 = adjoint_net()
    nl = base["linker_k"].size

    class MinimizedCoords(torch.autograd.Function):
        """x*(s_k, s_l0): the minimized coordinates with the linker
        stiffness and rest length scaled by (1 + s). Backward: implicit
        adjoint, H lam = dL/dx*, dL/ds = -sum_i theta_i lam . d2E/(dx dtheta_i)."""

        @staticmethod
        def forward(ctx, s_k, s_l0):
            x = minimized(base, nb, x0, float(s_k), float(s_l0))
            ctx.save_for_backward(s_k, s_l0)
            ctx.x = x
            return torch.from_numpy(x.copy())

        @staticmethod
        def backward(ctx, g):
            s_k, s_l0 = ctx.saved_tensors
            with ForceFieldManager("fp64") as ff:
                ff.vectorize_all_force_fields(system_for(base, nb, float(s_k), float(s_l0)))
                ff.set_coords(ctx.x)
                lam = cg_solve(ff.hvp, g.numpy(), tol=1e-9, maxit=500)
                dk, dl = ff.param_grad(FF_LINKER, nl, v=lam)
            kk = base["linker_k"] * (1.0 + float(s_k))
            ll = base["linker_l0"] * (1.0 + float(s_l0))
            # d theta_i / d s = theta_i / (1 + s)
            gk = -float(np.dot(dk, kk)) / (1.0 + float(s_k))
            gl = -float(np.dot(dl, ll)) / (1.0 + float(s_l0))
            return torch.tensor(gk, dtype=torch.float64), torch.tensor(gl, dtype=torch.float64)

    s_k = torch.tensor(0.0, dtype=torch.float64, requires_grad=True)
    s_l0 = torch.tensor(0.0, dtype=torch.float64, requires_grad=True)
    x = MinimizedCoords.apply(s_k, s_l0)
    L = ((x[-3:] - x[0:3]) ** 2).sum()
    L.backward()
    # Richardson differences of re-minimized networks
    h = 1e-3

    def fd(which):
        def at(s):
            return loss(minimized(base, nb, x0, s, 0.0) if which == 0 else minimized(base, nb, x0, 0.0, s))
        d1 = (at(h) - at(-h)) / (2 * h)
        d2 = (at(2 * h) - at(-2 * h)) / (4 * h)
        return (4 * d1 - d2) / 3

    fd_k, fd_l = fd(0), fd(1)
    assert abs(s_k.grad.item() - fd_k) <= 1e-6 * abs(fd_k) + 1e-9, (s_k.grad.item(), fd_k)
    assert abs(s_l0.grad.item() - fd_l) <= 1e-6 * abs(fd_l) + 1e-9, (s_l0.grad.item(), fd_l)
