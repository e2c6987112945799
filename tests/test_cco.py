"""GetCCO's potential (modules_b200.cco): the v(k) shapes and constraint set of apps/CCOptimization/main.cpp:262-318
and RepulsiveCCPotential (apps/CCOptimization/RepulsiveCCPotential.h:21-159, plain and S2 kernels) against the
reference's own class compiled into the oracle. Tolerance 1e-10 of the scales sum|V| N^2 / vol + e0 N (energy) and
4 sum|V| N kmax / vol + 20 e0 / sigma (force): the collective-coordinate scales of the reference's tests plus a
contact term of O(1) per particle.
"""
import numpy as np
import pytest

import oracle

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built")
RTOL = 1e-10


def test_alpha_5d_is_the_references_polynomial():
    from modules_b200.cco import alpha
    x = 0.4
    assert float(alpha(5, x)) == 1.0 - 1.875 * x + 1.25 * x * x * x - 0.875 * x ** 5
    assert float(alpha(5, 0.0)) == 1.0


@pytest.mark.parametrize("d", [1, 2, 3, 4])
def test_alpha_ends_and_monte_carlo(d):
    """alpha(d, x): 1 at x = 0, 0 from x = 1 on, and the lens volume fraction of two balls of diameter 1 (Monte Carlo
    over one ball, 4e5 points)."""
    from modules_b200.cco import alpha
    assert abs(float(alpha(d, 0.0)) - 1.0) < 1e-15 and abs(float(alpha(d, 1.0))) < 1e-15
    assert float(alpha(d, 1.5)) == 0.0
    rng = np.random.default_rng(d)
    p = rng.normal(size=(400000, d))
    p *= (0.5 * rng.random(len(p)) ** (1.0 / d) / np.linalg.norm(p, axis=1))[:, None]
    for x in (0.2, 0.55, 0.9):
        c = np.zeros(d)
        c[0] = x
        frac = np.mean(np.linalg.norm(p - c, axis=1) < 0.5)
        assert abs(frac - float(alpha(d, x))) < 5e-3, (d, x, frac, alpha(d, x))


def test_cco_constraints_shapes():
    from modules_b200 import cco
    basis = np.eye(2) * 20.0
    k1, k2 = 0.5, 1.2
    modes, V, S0 = cco.cco_constraints(2, basis, k1, k2, "power-law", m=3)
    k = oracle.lattice_k(basis, modes)
    kl = np.sqrt((k * k).sum(1))
    assert S0 is None and len(modes) > 10
    assert np.all(kl * kl > k1 * k1 - 1e-12) and np.all(kl < k2)
    assert np.allclose(V, (1 - kl / k2) ** 3, rtol=1e-12, atol=0)
    _, V2, _ = cco.cco_constraints(2, basis, k1, k2, "overlap")
    assert np.allclose(V2, cco.alpha(2, kl / k2), rtol=1e-12, atol=0)
    _, V3, S3 = cco.cco_constraints(2, basis, k1, k2, S0=0.7)
    assert np.all(V3 == 1.0) and np.all(S3 == 0.7)
    with pytest.raises(ValueError):
        cco.cco_constraints(2, basis, k1, k2, "triangle")


def jittered(d, N, seed):
    rng = np.random.default_rng(seed)
    side = int(np.ceil(N ** (1.0 / d)))
    grid = np.stack(np.meshgrid(*[np.arange(side)] * d, indexing="ij"), -1).reshape(-1, d)[:N] / side
    return np.ascontiguousarray((grid + rng.normal(0, 0.25 / side, grid.shape)) % 1.0)


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("d,N,k1,vtilde,S0", [(2, 400, 0.0, "flat", 0.0), (2, 500, 0.3, "power-law", 0.0),
                                              (3, 343, 0.0, "overlap", 0.0), (2, 400, 0.0, "flat", 0.6),
                                              (3, 216, 0.2, "flat", 1.3), (1, 64, 0.0, "overlap", 0.0)])
def test_gpu_repulsive_matches_reference(gpu, d, N, k1, vtilde, S0):
    from modules_b200 import cco
    L = N ** (1.0 / d)                 # unit density
    basis = np.eye(d) * L
    if d >= 2:
        basis[1, 0] = 0.2 * L
    k2 = 2.0 * np.pi * 1.6
    e0, sigma = 1.5, 0.85
    modes, V, S0s = cco.cco_constraints(d, basis, k1, k2, vtilde, m=2, S0=S0)
    frac = jittered(d, N, 17 + d)
    kc = oracle.lattice_k(basis, modes)
    Eref, Fref = oracle.ref_repulsive_eval(d, basis, kc, V, e0, sigma, frac, S0=S0s)
    p = cco.RepulsiveCCPotential(d, basis, modes, V, e0, sigma, S0=S0s)
    p.set_configuration(frac)
    E, F = p.energy_and_forces()
    vol = abs(np.linalg.det(basis))
    kmax = np.sqrt((kc * kc).sum(1)).max()
    sE = np.abs(V).sum() * N * N / vol + e0 * N
    sF = 4 * np.abs(V).sum() * N * kmax / vol + 20 * e0 / sigma
    assert abs(E - Eref) <= RTOL * sE, (E, Eref)
    assert np.abs(F - Fref).max() <= RTOL * sF
