"""The varBox potentials (modules_b200.varbox) against the reference's own classes (potential/CCPotential_varBox.h,
potential/CCPotential_Kernels.h), compiled into the oracle.

CPU: the constrained wavevectors, weights tildeV(k), targets S0(k) and shifts equal the reference's for every named
potential. GPU: energies and forces of the plain kinds (K2Potential, KM3Potential) equal the reference classes' own
Energy / AllForce; for the S2 kinds, whose reference classes leave S0 empty, they equal the reference's
ShiftedCCPotential_S2 given those classes' constraints with S0(k) from the classes' own S0k. Tolerance 1e-10 of the
rounding scales of the plain (rho ~ N, energy ~ sum|V| N^2 / vol, force ~ 4 sum|V| N kmax / vol) and S2 forms
(energy ~ sum|V| (|dS| + 1)^2, force ~ (4 / N) sum|V| (|dS| + 1)(|rho| + 1)|k|).
"""
import numpy as np
import pytest

import oracle

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built")

RTOL = 1e-10
CELLS = {
    1: np.array([[23.0]]),
    2: np.array([[21.0, 0.0], [5.5, 19.0]]),
    3: np.array([[11.0, 0.0, 0.0], [1.5, 10.0, 0.0], [-2.0, 2.5, 12.0]]),
}


def modes_of(basis, k):
    """Integer modes n_e = k . a_e / (2 pi) of Cartesian wavevectors."""
    n = np.asarray(k) @ np.asarray(basis).T / (2 * np.pi)
    r = np.rint(n)
    assert np.abs(n - r).max() < 1e-9
    return r.astype(np.int32)


def keyed(modes, *cols):
    order = np.lexsort(modes.T[::-1])
    return (modes[order],) + tuple(c[order] for c in cols)


@needs_ref
@pytest.mark.parametrize("d,rK", [(1, 2.0), (1, 2 * np.pi / 23.0 * 7), (2, 1.6), (3, 2.1), (2, 1.0)])
def test_wavevectors_and_plain_shift(d, rK):
    """The lattice points within rK (strict, half space) and the K2Potential shift N(N-1)/2V - N/V sum tildeV."""
    from modules_b200 import varbox
    basis = CELLS[d]
    frac = np.random.default_rng(d).random((37, d))
    ref = oracle.RefVarBox("K2Potential", d, basis, rK)
    ref.set_positions(frac)
    kref, Vref = ref.constraints()
    modes, V, S0, shift = varbox.constraints(d, basis, 37, "K2", rK=rK)
    assert S0 is None and len(modes) == len(kref) > 0
    a = keyed(modes, V)
    b = keyed(modes_of(basis, kref), Vref)
    assert np.array_equal(a[0], b[0])
    assert np.abs(a[1] - b[1]).max() <= 1e-13 * max(1.0, np.abs(b[1]).max())
    assert abs(shift - ref.state()[1]) <= 1e-12 * abs(ref.state()[1])


@needs_ref
@pytest.mark.parametrize("name", oracle.VARBOX_KINDS)
def test_weights_and_targets(name):
    """tildeV(k) and S0(k) of every named potential equal the class's own at its constraints."""
    from modules_b200 import varbox
    d = 3 if "KMLog" in name else 2
    basis = CELLS[d]
    n = 1.5
    ref = oracle.RefVarBox(name, d, basis, 1.3, n)
    ref.set_positions(np.random.default_rng(1).random((20, d)))
    kref, Vref = ref.constraints()
    Vw, S0w = ref.weights(kref)
    assert np.array_equal(Vw, Vref)
    weight, target, form = varbox.NAMED[name]
    modes, V, S0, shift = varbox.constraints(d, basis, 20, weight, target, form, 1.3, n)
    m, V, S0 = keyed(modes, V, np.zeros(len(V)) if S0 is None else S0)
    mr, Vr, S0r = keyed(modes_of(basis, kref), Vref, S0w)
    assert np.array_equal(m, mr)
    assert np.abs(V - Vr).max() <= 1e-12 * np.abs(Vr).max()
    if form == "plain":
        assert np.all(np.isnan(S0r))
    else:
        assert np.abs(S0 - S0r).max() <= 1e-12 * np.abs(S0r).max()
        if form == "S2_noV0":
            assert abs(shift + ((S0r - 1) ** 2 * Vr).sum()) <= 1e-12 * abs(shift)


@needs_ref
def test_reference_s2_classes_leave_S0_empty():
    """The defect that decides how the S2 kinds are checked: after SetConfiguration the reference's S2 varBox classes
    hold no S0 (and the noV0 class no shift), because the base marks the cell as cached before they test it."""
    for name in ("K2K2Potential", "K2K2Potential_noV0", "KM3KnPotential"):
        ref = oracle.RefVarBox(name, 2, CELLS[2], 1.3, 1.5)
        ref.set_positions(np.random.default_rng(2).random((10, 2)))
        M, shift, nS0 = ref.state()
        assert M > 0 and nS0 == 0 and shift == 0.0


def test_forms_are_checked():
    from modules_b200 import varbox
    with pytest.raises(ValueError):
        varbox.constraints(2, CELLS[2], 10, "K2", None, "S2")
    with pytest.raises(ValueError):
        varbox.constraints(2, CELLS[2], 10, "K2", "K2", "plain")
    with pytest.raises(ValueError):
        varbox.constraints(2, CELLS[2], 10, "KM3", "Kn", "S2")
    with pytest.raises(ValueError):
        varbox.constraints(3, CELLS[3], 10, "Lemniscate", None, "plain")


def test_unbound_potential_raises():
    """Energy, forces and minimisation before a cell is bound, or after close(), raise a clear error (no GPU call)."""
    from modules_b200 import varbox
    v = varbox.VarBoxPotential("K2Potential", d=2)
    for call in (v.energy, v.energy_and_forces, lambda: v.minimize(np.zeros((4, 2)))):
        with pytest.raises(RuntimeError, match="no bound cell"):
            call()
    v.close()
    with pytest.raises(RuntimeError, match="no bound cell"):
        v.energy()


def near_lattice(d, N, seed):
    rng = np.random.default_rng(seed)
    side = int(np.ceil(N ** (1.0 / d)))
    grid = np.stack(np.meshgrid(*[np.arange(side)] * d, indexing="ij"), -1).reshape(-1, d)[:N] / side
    return np.ascontiguousarray((grid + rng.normal(0, 0.1 / side, grid.shape)) % 1.0)


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("name,d,N,rK", [("K2Potential", 2, 1500, 1.6), ("KM3Potential", 3, 800, 2.1),
                                         ("K2Potential", 1, 200, 2.0)])
def test_gpu_plain_kinds_match_reference(gpu, name, d, N, rK):
    from modules_b200 import varbox
    basis = CELLS[d]
    frac = near_lattice(d, N, 7)
    ref = oracle.RefVarBox(name, d, basis, rK)
    ref.set_positions(frac)
    Eref, Fref, _, _ = ref.eval()
    kref, Vref = ref.constraints()
    vol = abs(np.linalg.det(basis))
    sE = np.abs(Vref).sum() * N * N / vol
    sF = 4 * np.abs(Vref).sum() * N * np.sqrt((kref ** 2).sum(1)).max() / vol
    p = varbox.VarBoxPotential(name, d, rK)
    p.set_configuration(basis, frac)
    E, F = p.energy_and_forces()
    assert abs(E - Eref) <= RTOL * sE + 1e-12 * abs(Eref), (E, Eref)
    assert np.abs(F - Fref).max() <= RTOL * sF


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("name,d,N", [("K2K2Potential", 2, 1200), ("K2K2Potential_noV0", 2, 700),
                                      ("KM3KnPotential", 3, 900), ("KM4KlcPotential", 2, 1000),
                                      ("KM3KMLogPotential", 3, 600), ("KM3K2Potential_noV0", 1, 150)])
def test_gpu_s2_kinds_match_reference_s2(gpu, name, d, N):
    from modules_b200 import varbox
    basis, rK, n = CELLS[d], 1.7, 1.5
    frac = near_lattice(d, N, 8)
    kind = oracle.RefVarBox(name, d, basis, rK, n)
    kind.set_positions(frac)
    kref, Vref = kind.constraints()
    _, S0ref = kind.weights(kref)
    shift = 0.0 if "noV0" not in name else -float(((S0ref - 1) ** 2 * Vref).sum())
    ref = oracle.Ref(d, basis, Vref, modes=modes_of(basis, kref), shift=shift, S0=S0ref)
    ref.set_positions(frac)
    Eref, Fref, re, im = ref.eval()
    dS = (re * re + im * im) / N - S0ref
    kn = np.sqrt((kref ** 2).sum(1))
    sE = float((np.abs(Vref) * (np.abs(dS) + 1) ** 2).sum())
    sF = float((4.0 / N) * (np.abs(Vref) * (np.abs(dS) + 1) * (np.sqrt(re * re + im * im) + 1) * kn).sum())
    p = varbox.VarBoxPotential(name, d, rK, n)
    p.set_configuration(basis, frac)
    E, F = p.energy_and_forces()
    assert abs(E - Eref) <= RTOL * sE + 1e-12 * abs(shift), (E, Eref)
    assert np.abs(F - Fref).max() <= RTOL * sF


@pytest.mark.gpu
def test_gpu_varbox_rebinds_on_cell_and_count(gpu):
    """A new cell regenerates the constraints; a new N changes the plain form's shift only."""
    from modules_b200 import varbox
    p = varbox.VarBoxPotential("K2Potential", 2, 1.6)
    frac = near_lattice(2, 400, 3)
    p.set_configuration(CELLS[2], frac)
    M0, s0 = len(p.V), p.shift
    p.set_configuration(CELLS[2], frac[:300])
    assert len(p.V) == M0 and p.shift != s0
    p.set_configuration(CELLS[2] * 1.5, frac[:300])
    assert len(p.V) > M0
    E, F = p.energy_and_forces()
    assert np.isfinite(E) and F.shape == (300, 2)
