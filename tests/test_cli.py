"""The command-line program's potential Types (modules_b200.cli, apps/CollectiveCoordinateCLI/
CollectiveCoordinateCLI.cpp:180-565).

CPU: the lattice enumeration equals the reference's own (PeriodicCellList::IterateThroughNeighbors with the half-space
rule, reached through its varBox class at radius R); the selection and weight rules of Types 4-17 equal a brute-force
restatement over all lattice points. GPU: the potentials built for the Types equal the reference's ShiftedCCPotential,
ShiftedCCPotential_S2 and ShiftedCCPotential_S2_MultiConfig on the same constraint sets (1e-10 of the scales).
"""
import numpy as np
import pytest

import oracle

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built")


def cell(d, N):
    L = N ** (1.0 / d) * 2 * np.pi / 6.0   # a few dozen points inside |k| < 1
    b = np.eye(d) * L
    if d >= 2:
        b[1, 0] = 0.3 * L
    return b


def brute(d, basis, R):
    """All half-space lattice points with |k| < R, by brute force over a box of modes."""
    B = 2 * np.pi * np.linalg.inv(basis).T
    lim = int(np.ceil(R * np.sqrt((basis ** 2).sum(1)).max() / (2 * np.pi))) + 1
    g = np.stack(np.meshgrid(*[np.arange(-lim, lim + 1)] * d, indexing="ij"), -1).reshape(-1, d)
    first = np.array([next((x for x in row if x != 0), 0) for row in g])
    g = g[first > 0]
    k = g @ B
    k2 = (k * k).sum(1)
    keep = k2 < R * R
    return g[keep], k2[keep]


def as_set(modes):
    return {tuple(int(x) for x in m) for m in modes}


@needs_ref
@pytest.mark.parametrize("d,R", [(1, 1.0), (2, 1.0), (2, 1.1), (3, 1.21), (3, 1.0)])
def test_enumeration_is_the_references(d, R):
    from modules_b200 import cli
    basis = cell(d, 300)
    modes, k2 = cli.half_space_points(d, basis, R)
    ref = oracle.RefVarBox("K2Potential", d, basis, R)
    ref.set_positions(np.random.default_rng(0).random((5, d)))
    kref, _ = ref.constraints()
    n = np.rint(kref @ basis.T / (2 * np.pi)).astype(int)
    assert as_set(modes) == as_set(n) and len(modes) == len(n) > 0


@pytest.mark.parametrize("type_", [4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17])
@pytest.mark.parametrize("d", [2, 3])
def test_selection_and_weights(type_, d):
    from modules_b200 import cli
    basis = cell(d, 300)
    S0p, n = 0.8, 1.5
    modes, V, S0, M = cli.constraint_set(type_, d, basis, 300, S0=S0p, n=n)
    assert M == len(modes)   # one growing step here, so no repeated points
    g, k2 = brute(d, basis, 3.0)
    lookup = {tuple(m): q for m, q in zip(g, k2)}
    mk2 = np.array([lookup[tuple(int(x) for x in m)] for m in modes])
    if type_ < 9:
        assert as_set(modes) == as_set(g[k2 < 1.0])
        K = np.sqrt(np.sort(k2)[len(modes)])
        want = {4: 1.0 + 0 * mk2, 8: 1.0 + 0 * mk2, 5: (1 - np.sqrt(mk2) / K) ** 2, 6: (1 - np.sqrt(mk2) / K) ** 6,
                7: 1 - np.sqrt(mk2)}[type_]
        assert S0 is None and np.allclose(V, want, rtol=1e-12, atol=1e-15)
        return
    shells = np.unique(np.round(k2, 12))
    outer = shells[shells > 1.0][0]
    inside = k2 <= 1.0
    if type_ in (9, 10):
        inside = inside | (np.abs(k2 - outer) <= 1e-12)
    assert as_set(modes) == as_set(g[inside])
    kl = np.sqrt(mk2)
    if type_ == 9:
        assert S0 is None and np.array_equal(V, np.where(mk2 > 1.0, -1e-4, 1.0))
        return
    assert np.all(V == 1.0)
    want = {10: np.where(mk2 > 1.0, S0p, 0.0), 11: 1.0 + 0 * kl, 12: S0p + 0 * kl, 13: kl / 2, 14: kl * S0p,
            15: kl * S0p, 16: mk2 * S0p, 17: mk2 ** (n / 2) * S0p}[type_]
    assert np.allclose(S0, want, rtol=1e-12, atol=1e-15)


def test_type_arguments_are_checked():
    from modules_b200 import cli
    basis = cell(2, 300)
    for kw in (dict(type_=15, S0=0.5), dict(type_=101), dict(type_=18), dict(type_=14), dict(type_=17, S0=0.5)):
        with pytest.raises(ValueError):
            cli.generate_potential(d=2, basis=basis, N=300, **kw)


def test_repeated_points_merge():
    """A cell whose first points lie beyond |k| = 1.1: the growing collection appends them again at every step; they
    become one constraint each with the weight times the count."""
    from modules_b200 import cli
    basis = np.eye(2) * 2 * np.pi / 1.05   # |b| = 1.05: points at 1.05 (inside 1.1) and beyond
    modes, V, S0, M = cli.constraint_set(9, 2, basis, 50)
    assert M >= len(modes) and len(np.unique(modes, axis=0)) == len(modes)


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("type_,d,N,nsub", [(4, 2, 400, None), (5, 3, 300, None), (9, 2, 500, None),
                                            (10, 2, 400, None), (13, 3, 343, None), (17, 2, 300, None),
                                            (15, 2, 600, 3)])
def test_gpu_types_match_reference(gpu, type_, d, N, nsub):
    from modules_b200 import cli
    basis = cell(d, N)
    pot, chi = cli.generate_potential(type_, d, basis, N, S0=0.8, n=1.5, nsub=nsub)
    modes, V, S0, M = cli.constraint_set(type_, d, basis, N, S0=0.8, n=1.5)
    assert chi == M / ((N - 1) * d)
    frac = np.random.default_rng(type_).random((N, d))
    ref = oracle.Ref(d, basis, V, modes=modes, S0=S0, nsub=nsub)
    ref.set_positions(frac)
    Eref, Fref, _, _ = ref.eval()
    pot.set_configuration(frac)
    E, F = pot.energy_and_forces()
    k = oracle.lattice_k(basis, modes)
    kmax = np.sqrt((k * k).sum(1)).max()
    if S0 is None:
        vol = abs(np.linalg.det(basis))
        sE, sF = np.abs(V).sum() * N * N / vol, 4 * np.abs(V).sum() * N * kmax / vol
    else:   # the S2 rounding scales of test_s2
        from test_s2 import multiconfig_restatement, tol_scales
        _, _, re, im, dS, _ = multiconfig_restatement(basis, frac, modes, V, S0, 0.0, nsub or 1)
        sE, sF = tol_scales(V, dS, np.sqrt((re * re + im * im).sum(0)), 0 * dS, k, N // (nsub or 1))
    assert abs(E - Eref) <= 1e-10 * sE + 1e-12 * abs(Eref), (E, Eref)
    assert np.abs(F - Fref).max() <= 1e-10 * sF
