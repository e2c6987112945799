"""The oracle (CPU checker) against the reference's golden vectors and, where built, the reference itself."""
import numpy as np
import pytest

import oracle
from conftest import golden_eval_cases, load_golden, scales


@pytest.mark.parametrize("name", golden_eval_cases())
def test_port_matches_golden(name):
    """The C restatement reproduces the reference's E, F, rho (pinned at 1e-13 of the test scales)."""
    r = load_golden(name)
    E, F, re, im = oracle.port_eval(int(r["d"]), r["basis"], r["frac"], r["kcart"], r["V"], float(r["shift"]))
    s = scales(r)
    assert abs(E - r["E"]) <= 1e-13 * max(s["energy"], abs(r["E"]), 1.0)
    if len(r["V"]):
        assert np.abs(re - r["rho_re"]).max() <= 1e-13 * s["rho"]
        assert np.abs(im - r["rho_im"]).max() <= 1e-13 * s["rho"]
    if len(r["frac"]) and len(r["V"]):
        assert np.abs(F - r["F"]).max() <= 1e-13 * s["force"]


def test_sign_kats():
    """Analytic phase/sign checks of the reference test (TestSign): rho(k) = sum_j exp(+i k.r_j)."""
    r = load_golden("sign_1d")
    assert abs(r["rho_re"][0]) < 1e-12 and abs(r["rho_im"][0] - 1.0) < 1e-12
    assert abs(r["rho_im"][1] + 1.0) < 1e-12 and abs(r["rho_re"][2] - 1.0) < 1e-12
    r = load_golden("sign_2d_skew")
    p0, p1 = 2 * np.pi * (0.25 + 0.125), 2 * np.pi * (-2 * 0.25 + 3 * 0.125)
    assert np.allclose([r["rho_re"][0], r["rho_im"][0], r["rho_re"][1], r["rho_im"][1]],
                       [np.cos(p0), np.sin(p0), np.cos(p1), np.sin(p1)], atol=1e-10)


def test_empty_kats():
    r = load_golden("empty_constraints")
    assert r["E"] == 0.7 and np.all(r["F"] == 0)
    r = load_golden("empty_particles")
    assert r["E"] == 0.0 and np.all(r["rho_re"] == 0) and np.all(r["rho_im"] == 0)


def test_port_structure_factor_matches_golden():
    r = load_golden("stealthy_3d_n2000")
    s = load_golden("sk_3d_n2000")
    k = oracle.lattice_k(r["basis"], s["sk_modes"])
    S = oracle.port_sk(3, r["basis"], r["frac"], k)
    assert np.abs(S - s["S"]).max() <= 1e-11 * max(1.0, s["S"].max())


def test_minimised_golden_is_ground_state():
    m = load_golden("min_2d_n100")
    assert m["E"] / 100 < 1e-20
    # stealthy window: S(k) ~ 0 for |k| <= K on the final configuration
    r = load_golden("stealthy_2d_n100")
    k = np.sqrt((oracle.lattice_k(np.eye(2), m["sk_modes"]) ** 2).sum(1))
    assert m["S"][k <= m["K"] * (1 + 1e-12)].max() < 1e-10


@pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built (needs the reference tree)")
def test_reference_reproduces_golden():
    """Re-running the reference on the stored inputs gives the stored outputs bitwise (fixtures are current)."""
    for name in ["lattice_2d_skew", "lattice_3d_skew", "stealthy_2d_n100"]:
        r = load_golden(name)
        ref = oracle.Ref(int(r["d"]), r["basis"], r["V"], modes=r["modes"], shift=float(r["shift"]))
        ref.set_positions(r["frac"])
        E, F, re, im = ref.eval()
        assert np.array_equal(F, r["F"]) and np.array_equal(re, r["rho_re"]) and np.array_equal(im, r["rho_im"])
        assert abs(E - r["E"]) <= 4e-16 * abs(r["E"])   # thread-order energy partials


@pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built (needs the reference tree)")
def test_port_matches_reference_random():
    rng = np.random.default_rng(7)
    for d, basis in [(1, [[1.7]]), (2, [[1.2, 0.1], [-0.3, 0.9]]), (3, [[1.0, 0.2, 0.0], [0.0, 1.1, 0.3],
                                                                        [0.1, 0.0, 0.8]])]:
        basis = np.array(basis)
        modes = rng.integers(-6, 7, size=(40, d)).astype(np.int32)
        V = rng.uniform(-0.5, 1.5, 40)
        frac = rng.random((37, d)) * 3 - 1   # unwrapped on purpose: both wrap by floor twice
        ref = oracle.Ref(d, basis, V, modes=modes, shift=0.1)
        ref.set_positions(frac)
        E, F, re, im = ref.eval()
        E2, F2, re2, im2 = oracle.port_eval(d, basis, frac, ref.kcart(), V, 0.1)
        assert abs(E - E2) <= 1e-14 * abs(E)
        assert np.array_equal(F, F2) and np.array_equal(re, re2) and np.array_equal(im, im2)
