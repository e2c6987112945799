"""Isotropic structure factor (IsotropicStructureFactor, pairstat/StructureFactor.cpp:79-260) against golden vectors
made by the reference's own implementation (tests/golden/make_golden_isotropic.py).

CPU: the wavevector list (GetKs, core/PeriodicCellList.cpp:509-735) of cc_kset_isotropic, in the reference's order.
GPU: the binned rows (k, S, dk, dS) of cc_isotropic_structure_factor. Bin means of k and S must agree to 1e-9 relative;
the spreads dk and dS come from a difference of two nearly equal sums (one-wavevector bins give sqrt of a rounding
residue), so they are held to 1e-7 of the column's scale; option 2's counts must be equal.
"""
import numpy as np
import pytest

from conftest import load_golden

G = load_golden("isotropic_sk")
NAMES = [str(n) for n in G["names"]]


def _case(name):
    d = int(G[name + "__d"])
    bases = G[name + "__bases"]
    Ns = G[name + "__N"]
    frac = G[name + "__frac"]
    fracs = np.split(frac, np.cumsum(Ns)[:-1])
    circ, lin, kprec, p, option, kmin = G[name + "__params"]
    return d, bases, fracs, circ, lin, kprec, p, int(option), kmin


@pytest.mark.parametrize("name", NAMES)
def test_wavevectors_match_reference(ccgpu, name):
    d, bases, _fr, circ, lin, _kp, p, _opt, kmin = _case(name)
    ref = G[name + "__ks"]
    modes, kamp = ccgpu.isotropic_kset(d, bases[0], circ, lin, p, kmin)
    assert len(modes) == len(ref)
    if len(ref) == 0:
        return
    B = 2 * np.pi * np.linalg.inv(bases[0]).T
    k = modes.astype(np.float64) @ B
    scale = np.abs(ref).max()
    assert np.abs(k - ref).max() <= 1e-12 * scale
    assert np.abs(kamp - np.sqrt((ref ** 2).sum(1))).max() <= 1e-12 * scale
    # half space: first nonzero index positive
    first = np.array([m[np.nonzero(m)[0][0]] for m in modes])
    assert np.all(first > 0)


def test_wavevector_arguments(ccgpu):
    with pytest.raises(ccgpu.CCError):
        ccgpu.isotropic_kset(1, -np.eye(1), 1.0, 2.0)          # a 1D cell of negative length
    m, k = ccgpu.isotropic_kset(2, np.eye(2) * 5, -1.0, 2.0)    # no circle: no wavevector, as the reference
    assert len(m) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_isotropic_sk_matches_reference(gpu, name):
    d, bases, fracs, circ, lin, kprec, p, option, kmin = _case(name)
    ref = G[name + "__rows"]
    got = gpu.isotropic_structure_factor(d, bases, fracs, circ, lin, kprec, p, option, kmin)
    assert got.shape == ref.shape
    if option == 2:
        # one row per wavevector, sorted by |k|: rows of equal |k| may come in either order
        key = lambda r: np.lexsort((r[:, 1], np.round(r[:, 0], 10)))
        got, ref = got[key(got)], ref[key(ref)]
    kscale, sscale = max(lin, 1e-300), max(np.abs(ref[:, 1]).max(), 1.0)
    assert np.allclose(got[:, 0], ref[:, 0], rtol=1e-9, atol=1e-12 * kscale)
    assert np.allclose(got[:, 1], ref[:, 1], rtol=1e-9, atol=1e-12 * sscale)
    assert np.abs(got[:, 2] - ref[:, 2]).max() <= 1e-7 * kscale
    if option == 2:
        assert np.array_equal(got[:, 3], ref[:, 3])
    else:
        assert np.abs(got[:, 3] - ref[:, 3]).max() <= 1e-7 * sscale


@pytest.mark.gpu
def test_isotropic_sk_edge_cases(gpu):
    f = [np.random.default_rng(3).random((50, 2))]
    # the reference returns no rows for these
    assert len(gpu.isotropic_structure_factor(2, [np.eye(2) * 7], f, 0.0, 1.0)) == 0
    assert len(gpu.isotropic_structure_factor(2, [np.eye(2) * 7], f, 1.0, 2.0, circular_kmin=1.5)) == 0
    with pytest.raises(gpu.CCError):
        gpu.isotropic_structure_factor(2, [np.eye(2) * 7], f, 1.0, 1.0, option=3)
