"""The S2 form (cc_create_s2 / CCPotential(S0=...)) against the reference's ShiftedCCPotential_S2
(potential/CollectiveCoordinatePotential.h:1642-1749): E = sum_k V (|rho|^2 / N - S0)^2 + Shift and
F_i = -(4 / N) sum_k V dS (Im rho cos k.r - Re rho sin k.r) k.

The CPU tests pin a numpy restatement of those formulas to the compiled reference; the GPU tests compare the sm_100a
path with the reference at 1e-10 of the rounding scales below (rho ~ N; an error of eps in rho moves S by about
2 |rho| eps / N, so the energy scale is sum |V| (|dS| + 1)^2 and the force scale (4 / N) sum |V| (|dS| + 1)(|rho| + 1)|k|).
"""
import numpy as np
import pytest

import oracle

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built")
RTOL = 1e-10


def skew_basis(d):
    b = np.eye(d) * 7.0
    if d >= 2:
        b[1, 0] = 1.75
    if d == 3:
        b[2, 1] = -0.9
        b[2, 0] = 0.4
    return b


def case(d, N, kmax, seed):
    """A near-lattice configuration (so that some S(k) are small and the targets matter), distinct modes with both
    k and -k present for some of them, random weights and targets."""
    rng = np.random.default_rng(seed)
    side = int(np.ceil(N ** (1.0 / d)))
    grid = np.stack(np.meshgrid(*[np.arange(side)] * d, indexing="ij"), -1).reshape(-1, d)[:N] / side
    frac = (grid + rng.normal(0, 0.08 / side, grid.shape)) % 1.0
    r = np.arange(-kmax, kmax + 1)
    modes = np.stack(np.meshgrid(*[r] * d, indexing="ij"), -1).reshape(-1, d)
    modes = modes[np.any(modes != 0, axis=1)]
    modes = modes[rng.random(len(modes)) < 0.6]
    rng.shuffle(modes)
    V = rng.uniform(0.2, 2.0, len(modes))
    S0 = rng.uniform(0.0, 1.5, len(modes))
    return skew_basis(d), np.ascontiguousarray(frac), modes.astype(np.int32), V, S0


def restatement(basis, frac, modes, V, S0, shift):
    """The reference's S2 Energy and Force(i) in numpy."""
    N = len(frac)
    k = oracle.lattice_k(basis, modes)
    r = frac @ basis
    ph = r @ k.T
    c, s = np.cos(ph), np.sin(ph)
    re, im = c.sum(0), s.sum(0)
    dS = (re * re + im * im) / N - S0
    E = float((V * dS * dS).sum()) + shift
    coef = (4.0 / N) * V * dS
    F = -((im * c - re * s) * coef) @ k
    return E, F, re, im, dS, k


def tol_scales(V, dS, re, im, k, N):
    kn = np.sqrt((k * k).sum(1))
    rho = np.sqrt(re * re + im * im)
    return (float((np.abs(V) * (np.abs(dS) + 1) ** 2).sum()),
            float((4.0 / N) * (np.abs(V) * (np.abs(dS) + 1) * (rho + 1) * kn).sum()))


@needs_ref
@pytest.mark.parametrize("d,N,kmax", [(1, 40, 25), (2, 300, 6), (3, 200, 3)])
def test_restatement_matches_reference(d, N, kmax):
    basis, frac, modes, V, S0 = case(d, N, kmax, 11 + d)
    ref = oracle.Ref(d, basis, V, modes=modes, shift=0.3, S0=S0)
    ref.set_positions(frac)
    E, F, re, im = ref.eval()
    E2, F2, re2, im2, dS, k = restatement(basis, frac, modes, V, S0, 0.3)
    sE, sF = tol_scales(V, dS, re2, im2, k, N)
    assert abs(E - E2) <= 1e-12 * sE
    assert np.abs(F - F2).max() <= 1e-12 * sF
    assert np.abs(re - re2).max() <= 1e-12 * N and np.abs(im - im2).max() <= 1e-12 * N
    for i in (0, N // 2, N - 1):
        assert np.abs(ref.force_one(i) - F2[i]).max() <= 1e-12 * sF


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("d,N,kmax", [(1, 64, 40), (2, 1000, 9), (3, 2000, 5), (2, 20000, 12)])
def test_gpu_matches_reference(gpu, d, N, kmax):
    basis, frac, modes, V, S0 = case(d, N, kmax, 100 + d + N)
    ref = oracle.Ref(d, basis, V, modes=modes, shift=-0.25, S0=S0)
    ref.set_positions(frac)
    Eref, Fref, re, im = ref.eval()
    k = oracle.lattice_k(basis, modes)
    dS = (re * re + im * im) / N - S0
    sE, sF = tol_scales(V, dS, re, im, k, N)
    p = gpu.CCPotential(d, basis, modes, V, -0.25, S0=S0)
    p.set_configuration(frac)
    for _ in range(3):   # direct, then captured evaluations of the same key
        E, F = p.energy_and_forces()
        assert abs(E - Eref) <= RTOL * sE, (E, Eref)
        assert np.abs(F - Fref).max() <= RTOL * sF
    assert p.energy() == E
    gre, gim = p.rho()
    assert np.abs(gre - re).max() <= RTOL * N and np.abs(gim - im).max() <= RTOL * N
    assert np.array_equal(p.force(N // 3), F[N // 3])


@pytest.mark.gpu
@needs_ref
def test_gpu_repeated_modes_match_reference(gpu):
    """The reference keeps repeated wavevectors as separate constraints; here they share a slot with the summed
    weight, the weighted mean target and the remainder in the shift."""
    basis, frac, modes, V, S0 = case(2, 800, 7, 77)
    rng = np.random.default_rng(5)
    pick = rng.choice(len(modes), 12, replace=False)
    modes2 = np.vstack([modes, modes[pick], modes[pick[:4]]])
    V2 = np.concatenate([V, rng.uniform(0.1, 1.0, 12), rng.uniform(-0.05, 0.5, 4)])
    S02 = np.concatenate([S0, rng.uniform(0.0, 2.0, 16)])
    ref = oracle.Ref(2, basis, V2, modes=modes2, shift=0.2, S0=S02)
    ref.set_positions(frac)
    Eref, Fref, re, im = ref.eval()
    k = oracle.lattice_k(basis, modes2)
    dS = (re * re + im * im) / len(frac) - S02
    sE, sF = tol_scales(V2, dS, re, im, k, len(frac))
    p = gpu.CCPotential(2, basis, modes2, V2, 0.2, S0=S02)
    p.set_configuration(frac)
    E, F = p.energy_and_forces()
    assert abs(E - Eref) <= RTOL * sE, (E, Eref)
    assert np.abs(F - Fref).max() <= RTOL * sF


@pytest.mark.gpu
def test_gpu_fp64_only_and_refusals(gpu):
    basis, frac, modes, V, S0 = case(2, 3000, 8, 5)
    p = gpu.CCPotential(2, basis, modes, V, 0.0, S0=S0)
    p.set_configuration(frac)
    E, F = p.energy_and_forces()
    Em, Fm = p.energy_and_forces(precision=gpu.PREC_MIXED)   # evaluated in FP64 whatever the precision
    assert Em == E and np.array_equal(Fm, F)
    with pytest.raises(gpu.CCError):
        p.set_path(1)                                           # not a path (include/cc_gpu.h cc_set_path)
    with pytest.raises(gpu.CCError):
        p.set_path(gpu.PATH_NUFFT)
    with pytest.raises(gpu.CCError):
        p.try_move(frac[0], (frac[0] + 0.01) % 1.0)
    with pytest.raises(gpu.CCError):
        gpu.CCBatch([p], [len(frac)])
    with pytest.raises(gpu.CCError):   # copies of a mode whose weights cancel have no S2 form
        gpu.CCPotential(2, basis, np.vstack([modes, modes[:1]]), np.append(V, -V[0]), 0.0, S0=np.append(S0, 0.5))
    with pytest.raises(ValueError):
        gpu.CCPotential(2, basis, modes, V, 0.0, S0=S0[:-1])


@pytest.mark.gpu
def test_gpu_minimize_s2(gpu):
    """Stealthy targets (S0 = 0) at a small constrained fraction: the device L-BFGS drives E to its ground state 0,
    and the reported energy is the potential's at the returned positions."""
    basis, frac, modes, V, _ = case(2, 400, 3, 9)
    rng = np.random.default_rng(3)
    start = rng.random((400, 2))
    p = gpu.CCPotential(2, basis, modes, V, 0.0, S0=np.zeros(len(V)))
    p.set_configuration(start)
    E0 = p.energy()
    x, E, evals, iters, status = p.minimize(start, stopval=1e-20, max_evals=20000,
                                            precision=gpu.PREC_SCHEDULE)
    assert evals > 0 and E < 1e-6 * E0
    p.set_configuration(x)
    assert abs(p.energy() - E) <= 1e-12 * E0


def multiconfig_restatement(basis, frac, modes, V, S0, shift, nsub):
    """The reference's ShiftedCCPotential_S2_MultiConfig Energy and Force(i) in numpy
    (potential/CollectiveCoordinatePotential.h:1777-1870)."""
    N = len(frac)
    Np = N // nsub
    k = oracle.lattice_k(basis, modes)
    ph = (frac @ basis) @ k.T
    c, s = np.cos(ph), np.sin(ph)
    re = c.reshape(nsub, Np, -1).sum(1)
    im = s.reshape(nsub, Np, -1).sum(1)
    snow = (re * re + im * im).sum(0) / (Np * nsub)
    dS = snow - S0
    E = float((V * dS * dS).sum()) + shift
    coef = (4.0 / Np) * V * dS / nsub
    sub = np.repeat(np.arange(nsub), Np)
    F = -((im[sub] * c - re[sub] * s) * coef) @ k
    return E, F, re, im, dS, k


@needs_ref
@pytest.mark.parametrize("d,N,kmax,nsub", [(2, 300, 6, 3), (3, 200, 3, 4), (1, 60, 20, 5)])
def test_multiconfig_restatement_matches_reference(d, N, kmax, nsub):
    basis, frac, modes, V, S0 = case(d, N, kmax, 21 + d)
    ref = oracle.Ref(d, basis, V, modes=modes, shift=0.4, S0=S0, nsub=nsub)
    ref.set_positions(frac)
    E, F, _, _ = ref.eval()
    E2, F2, re, im, dS, k = multiconfig_restatement(basis, frac, modes, V, S0, 0.4, nsub)
    sE, sF = tol_scales(V, dS, np.sqrt((re * re + im * im).sum(0)), 0 * dS, k, N // nsub)
    assert abs(E - E2) <= 1e-12 * sE
    assert np.abs(F - F2).max() <= 1e-12 * sF


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("d,N,kmax,nsub", [(2, 1200, 9, 3), (3, 2000, 5, 4), (2, 6000, 10, 2), (1, 100, 30, 5)])
def test_gpu_multiconfig_matches_reference(gpu, d, N, kmax, nsub):
    basis, frac, modes, V, S0 = case(d, N, kmax, 300 + d + nsub)
    ref = oracle.Ref(d, basis, V, modes=modes, shift=0.125, S0=S0, nsub=nsub)
    ref.set_positions(frac)
    Eref, Fref, _, _ = ref.eval()
    _, _, re, im, dS, k = multiconfig_restatement(basis, frac, modes, V, S0, 0.125, nsub)
    sE, sF = tol_scales(V, dS, np.sqrt((re * re + im * im).sum(0)), 0 * dS, k, N // nsub)
    p = gpu.CCPotential(d, basis, modes, V, 0.125, S0=S0, nsub=nsub)
    p.set_configuration(frac)
    for _ in range(3):   # direct, then captured evaluations of the same key
        E, F = p.energy_and_forces()
        assert abs(E - Eref) <= RTOL * sE, (E, Eref)
        assert np.abs(F - Fref).max() <= RTOL * sF
    assert p.energy() == E


@pytest.mark.gpu
def test_gpu_multiconfig_rules(gpu):
    basis, frac, modes, V, S0 = case(2, 600, 6, 41)
    one = gpu.CCPotential(2, basis, modes, V, 0.0, S0=S0, nsub=1)
    s2 = gpu.CCPotential(2, basis, modes, V, 0.0, S0=S0)
    one.set_configuration(frac)
    s2.set_configuration(frac)
    E1, F1 = one.energy_and_forces()
    E2, F2 = s2.energy_and_forces()
    assert E1 == E2 and np.array_equal(F1, F2)          # one sub-configuration is the S2 form
    p = gpu.CCPotential(2, basis, modes, V, 0.0, S0=S0, nsub=4)
    with pytest.raises(gpu.CCError):
        p.set_configuration(frac[:598])                  # not a multiple of the sub-configuration count
    p.set_configuration(frac)
    with pytest.raises(gpu.CCError):
        p.rho()                                          # rho is per sub-configuration
    E, F = p.energy_and_forces()
    x, Em, evals, iters, status = p.minimize(frac, max_evals=300)
    assert Em < E
    p.set_configuration(x)
    assert abs(p.energy() - Em) <= 1e-12 * E
    with pytest.raises(ValueError):
        gpu.CCPotential(2, basis, modes, V, 0.0, nsub=2)
