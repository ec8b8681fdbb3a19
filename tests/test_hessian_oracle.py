"""The oracle's restatement of ForceFieldManager::computeHessian
(ForceFieldManager.cpp:354-398) and the eigenmode analysis (:400-480), on CPU:
the finite-difference Hessian of a spring network against its closed form,
entries rounded to float as the reference stores them, and the participation
ratios of hessian_modes."""
import numpy as np

from medyan_b200._abi import SystemView
from medyan_b200.forcefield import hessian_modes


def spring_network(seed=3, nb=30):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0, 50, size=(nb, 3))
    pairs = np.array([(i, j) for i in range(nb) for j in range(i + 1, nb) if rng.random() < 0.15])
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
    return sv, x.reshape(-1), H


def test_oracle_hessian_springs(oracle):
    sv, x, H = spring_network()
    Ho = oracle.hessian(sv, x, 1e-4)
    # entries are floats
    assert np.array_equal(Ho, Ho.astype(np.float32).astype(np.float64))
    # central differences of springs: O(delta^2) plus force rounding / delta
    assert np.abs(Ho - H).max() <= 1e-5 * np.abs(H).max()
    assert np.abs(Ho - Ho.T).max() <= 1e-5 * np.abs(H).max()


def test_hessian_modes():
    sv, x, H = spring_network(seed=5)
    m = hessian_modes(H)
    n = H.shape[0]
    assert np.all(np.diff(m.evalues) >= -1e-9 * np.abs(m.evalues).max())
    # eigenvectors are orthonormal, and H v = lambda v
    assert np.abs(m.evectors.T @ m.evectors - np.eye(n)).max() < 1e-9
    assert np.abs(H @ m.evectors - m.evectors * m.evalues).max() < 1e-8 * np.abs(H).max()
    # a spring network is translation invariant: three zero modes
    assert np.sum(np.abs(m.evalues) < 1e-8 * np.abs(m.evalues).max()) >= 3
    # participation ratios: 1/n <= IPRI <= 1, 1/(n/3) <= IPRII <= 1
    assert np.all(m.IPRI <= 1 + 1e-12) and np.all(m.IPRI >= 1 / n - 1e-12)
    assert np.all(m.IPRII <= 1 + 1e-12) and np.all(m.IPRII >= 3 / n - 1e-12)
    v = m.evectors[:, 0]
    assert np.isclose(m.IPRI[0], np.sum(v ** 4))
    assert np.isclose(m.IPRII[0], np.sum(np.sum(v.reshape(-1, 3) ** 2, axis=1) ** 2))
