"""Failures made on the host, never on the GPU: non-finite inputs, the objective's NaN sentinel. Every case checks the
returned status and that the same handle evaluates correctly afterwards.

The reference's conventions: non-finite coordinates are refused by the setters (std::invalid_argument in the
reference; CC_ERR_ARG here), and a NaN first variable of the Switch-0 objective is NotANumberFound
(potential/StructureOptimization.cpp:460-461), which its Objective does not catch (:571 catches InvalidStructure).
"""
import numpy as np
import pytest

from conftest import load_golden, scales


def test_nan_status_maps_to_not_a_number_found(ccgpu):
    """CPU: status -8 raises NotANumberFound (a CCError), other statuses plain CCError."""
    from modules_b200 import ccgpu as b
    with pytest.raises(ccgpu.NotANumberFound) as e:
        b._check(-8)
    assert e.value.code == -8 and isinstance(e.value, ccgpu.CCError)
    with pytest.raises(ccgpu.CCError) as e:
        b._check(-1)
    assert not isinstance(e.value, ccgpu.NotANumberFound)


def _pot(gpu, r):
    return gpu.CCPotential(int(r["d"]), r["basis"], r["modes"], r["V"], float(r["shift"]))


def _check_eval(p, r):
    s = scales(r)
    E, F = p.energy_and_forces()
    assert abs(E - float(r["E"])) <= 1e-10 * abs(float(r["E"]))
    assert np.abs(F - r["F"]).max() <= 1e-10 * s["force"]


@pytest.mark.gpu
@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_nonfinite_positions_rejected(gpu, bad):
    r = load_golden("lattice_2d_skew")
    p = _pot(gpu, r)
    p.set_configuration(r["frac"])
    _check_eval(p, r)
    x = r["frac"].copy()
    x[7, 1] = bad
    with pytest.raises(gpu.CCError) as e:
        p.set_configuration(x)
    assert e.value.code == -1
    with pytest.raises(gpu.CCError) as e:   # nothing is bound after a refused configuration
        p.energy_and_forces()
    assert e.value.code in (-1, -6)
    p.set_configuration(r["frac"])
    _check_eval(p, r)


@pytest.mark.gpu
def test_objective_nan_first_variable(gpu):
    r = load_golden("lattice_2d_skew")
    p = _pot(gpu, r)
    x = r["frac"].reshape(-1) * 10.0
    f0, g0 = p.objective(x, 10.0)
    bad = x.copy()
    bad[0] = np.nan
    with pytest.raises(gpu.NotANumberFound):
        p.objective(bad, 10.0)
    bad = x.copy()
    bad[3] = np.inf
    with pytest.raises(gpu.CCError) as e:
        p.objective(bad, 10.0)
    assert e.value.code == -1
    f1, g1 = p.objective(x, 10.0)
    assert f1 == f0 and np.array_equal(g1, g0)
    assert abs(f0 - float(r["E"])) <= 1e-10 * abs(float(r["E"]))


@pytest.mark.gpu
def test_batch_bounded_wait_runs_out_and_recovers(gpu):
    """The fused batch kernel's bounded wait, made to run out from the host (the first instance's reduce items wait
    for one rho item that does not exist, 2000 polls): the evaluation reports CC_ERR_TIMEOUT (-4), and the next
    evaluation of the same batch, with the hook off, is bitwise the one before."""
    rng = np.random.default_rng(3)
    pots, N, fracs = [], [], []
    for d, n, chi in [(2, 300, 0.3), (3, 400, 0.25), (2, 150, 0.4)]:
        basis = np.eye(d) * n ** (1.0 / d)
        modes, V = gpu.stealthy_kset(d, basis, n, chi)
        pots.append(gpu.CCPotential(d, basis, modes, V))
        N.append(n)
        fracs.append(rng.random((n, d)))
    batch = gpu.CCBatch(pots, N)
    batch.set_positions(fracs)
    E0, F0 = batch.energy_and_forces()
    batch.set_wait_test(polls=2000, phantom=1)
    with pytest.raises(gpu.CCError) as e:
        batch.energy_and_forces()
    assert e.value.code == -4
    batch.set_wait_test(0, 0)
    E1, F1 = batch.energy_and_forces()
    assert np.array_equal(E0, E1) and all(np.array_equal(a, b) for a, b in zip(F0, F1))
