"""The multi-species stealthy potential with soft-core contact (cc_multi_*, MultiStealthyPotential of
apps/CCOptimization) against golden vectors made by the reference's own implementation
(tests/golden/make_golden_multi.py). Tolerances as the reference's test_fused_contact.cpp: the energy within 1e-10
relative, forces within 1e-10 times max(1, max |F|)."""
import numpy as np
import pytest

from conftest import load_golden

G = load_golden("multi_stealthy")
NAMES = [str(n) for n in G["names"]]


def _build(gpu, name):
    d = int(G[name + "__d"])
    M = G[name + "__M"]
    cuts = np.cumsum(M)[:-1]
    modes = np.split(G[name + "__modes"], cuts)
    Vs = np.split(G[name + "__V"], cuts)
    pot = gpu.CCMulti(d, G[name + "__basis"], modes, Vs, u0=float(G[name + "__u0"]), e0=float(G[name + "__e0"]))
    radii = G[name + "__radii"]
    pot.set_configuration(G[name + "__frac"], G[name + "__species"], radii if len(radii) else None)
    return pot


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_multi_matches_reference(gpu, name):
    pot = _build(gpu, name)
    E, F = pot.energy_and_forces()
    Er, Fr = float(G[name + "__E"]), G[name + "__F"]
    assert abs(E - Er) <= 1e-10 * abs(Er), (E, Er)
    assert np.abs(F - Fr).max() <= 1e-10 * max(1.0, np.abs(Fr).max()), np.abs(F - Fr).max()
    # the energy-only call gives the same energy bitwise
    E2, _ = pot.energy_and_forces(forces=False)
    assert E2 == E


@pytest.mark.gpu
def test_multi_arguments(gpu):
    d = 2
    pot = gpu.CCMulti(d, np.eye(2) * 5, [np.array([[1, 0]], np.int32)], [np.array([1.0])])
    frac = np.random.default_rng(0).random((10, 2))
    with pytest.raises(gpu.CCError):
        pot.set_configuration(frac, np.full(10, 1, np.int32))          # species out of range
    with pytest.raises(gpu.CCError):
        pot.set_configuration(frac, np.zeros(10, np.int32), radii=-np.ones(10))
    with pytest.raises(gpu.CCError):
        pot.energy_and_forces()                                          # nothing bound yet
    pot.set_configuration(frac, np.zeros(10, np.int32))
    E, F = pot.energy_and_forces()
    assert np.isfinite(E) and F.shape == (10, 2)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES[:3])
def test_multi_from_mspb_snapshot(gpu, name, tmp_path):
    """A configuration stored as an MSPB snapshot (the reference optimiser's export format), read back and bound with
    CCMulti.set_snapshot, evaluates like the configuration bound directly and within 1e-10 of the reference."""
    from modules_b200 import mspb
    direct = _build(gpu, name)
    E0, F0 = direct.energy_and_forces()
    d = int(G[name + "__d"])
    n = len(G[name + "__frac"])
    radii = G[name + "__radii"] if len(G[name + "__radii"]) else np.full(n, 0.5)
    snap = mspb.Snapshot.create(G[name + "__basis"].reshape(d, d), G[name + "__frac"], species=G[name + "__species"],
                                radii=radii, ids=np.arange(n)[::-1] + 100, species_count=len(G[name + "__M"]))
    path = tmp_path / "conf.mspb"
    mspb.write(path, snap)
    direct.set_snapshot(mspb.read(path))
    E, F = direct.energy_and_forces()
    assert E == E0 and np.array_equal(F, F0)
    Er, Fr = float(G[name + "__E"]), G[name + "__F"]
    assert abs(E - Er) <= 1e-10 * abs(Er)
    assert np.abs(F - Fr).max() <= 1e-10 * max(1.0, np.abs(Fr).max())
