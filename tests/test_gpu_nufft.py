"""The non-uniform FFT path (cc_set_path(CC_PATH_NUFFT)) against the reference's own FP64 results and against the
direct path. The reference holds its own FINUFFT backend to rtol 1e-9 of the Direct sums
(potential/tests/finufft_type1/test_finufft_type1.cpp CompareBackends); here the bar is the direct path's: 1e-10 of
the reference tests' scales (rho ~ N, energy ~ sum|V| N^2/vol, force ~ 4 sum|V| N kmax/vol)."""
import numpy as np
import pytest

from conftest import golden_eval_cases, load_golden, scales

pytestmark = pytest.mark.gpu

RTOL = 1e-10


@pytest.mark.parametrize("name", golden_eval_cases())
def test_nufft_matches_reference(gpu, name):
    r = load_golden(name)
    if not len(r["V"]):
        pytest.skip("no constraints: nothing to transform")
    s = scales(r)
    p = gpu.CCPotential(int(r["d"]), r["basis"], r["modes"], r["V"], float(r["shift"]))
    p.set_path(gpu.PATH_NUFFT)
    p.set_configuration(r["frac"])
    E, F = p.energy_and_forces()
    Eref = float(r["E"])
    assert abs(E - Eref) <= RTOL * abs(Eref) + 1e-13 * max(s["energy"], 1.0), (E, Eref)
    if len(r["frac"]):
        assert np.abs(F - r["F"]).max() <= RTOL * s["force"]
    re, im = p.rho()
    assert np.abs(re - r["rho_re"]).max() <= RTOL * s["rho"]
    assert np.abs(im - r["rho_im"]).max() <= RTOL * s["rho"]


def test_nufft_large_2d_against_direct(gpu):
    """2D N=1e5 chi=0.20 (M=40002): NUFFT against the direct path, and bitwise repeatable."""
    d, N, chi = 2, 100000, 0.20
    basis = np.eye(d) * np.sqrt(N)
    modes, V = gpu.stealthy_kset(d, basis, N, chi)
    frac = np.random.default_rng(21).random((N, d))
    p = gpu.CCPotential(d, basis, modes, V)
    p.set_path(gpu.PATH_SPLIT)
    p.set_configuration(frac)
    E0, F0 = p.energy_and_forces()
    p.set_path(gpu.PATH_NUFFT)
    E1, F1 = p.energy_and_forces()
    E2, F2 = p.energy_and_forces()
    assert E1 == E2 and np.array_equal(F1, F2)
    kmax = np.sqrt(((2 * np.pi * modes / np.sqrt(N)) ** 2).sum(1)).max()
    sE, sF = V.sum() * N * N / N, 4 * V.sum() * N * kmax / N
    assert abs(E1 - E0) <= RTOL * abs(E0) + 1e-13 * sE, (E1, E0)
    assert np.abs(F1 - F0).max() <= RTOL * sF
    assert np.abs(F1.sum(0)).max() <= 1e-9 * sF   # Newton's third law
    p.set_path(gpu.PATH_AUTO)   # the default picks the NUFFT path at this size
    E3, F3 = p.energy_and_forces()
    assert E3 == E1 and np.array_equal(F3, F1)


def test_nufft_minimisation_reaches_ground_state(gpu):
    """The device L-BFGS on the NUFFT path reaches the 2D N=100 stealthy ground state (Phi/N < 1e-20)."""
    d, N = 2, 100
    modes, V = gpu.stealthy_kset(d, np.eye(2), N, 0.30)
    p = gpu.CCPotential(d, np.eye(2), modes, V)
    p.set_path(gpu.PATH_NUFFT)
    x, E, evals, iters, status = p.minimize(np.random.default_rng(5).random((N, d)), stopval=1e-20 * N)
    print(f"NUFFT minimisation: E/N={E / N:.2e} evals={evals}")
    assert E / N < 1e-20
