"""Device-resident L-BFGS to the stealthy ground state, checked against the reference.

Parity is on the final state, not on iterates (the method is L-BFGS in compact form, not NLopt's PLIS): from the
same start as the reference's own minimisation (tests/golden/min_2d_n100.npz, made by running the reference's
LuksanPLIS through the restated three-pass driver), the GPU reaches Phi/N < 1e-20, the reference's FP64 energy of the
GPU result is below 1e-20 N too, and S(k) in the stealthy window |k| <= K vanishes (<= 1e-10) as it does for the
reference's result.
"""
import numpy as np
import pytest

import oracle
from conftest import load_golden

pytestmark = pytest.mark.gpu


def _window_max_S(basis, frac, modes_window):
    k = oracle.lattice_k(basis, modes_window)
    return oracle.port_sk(len(basis), basis, frac, k).max()


def test_ground_state_2d_n100(gpu):
    r = load_golden("stealthy_2d_n100")
    mref = load_golden("min_2d_n100")
    N = 100
    p = gpu.CCPotential(2, r["basis"], r["modes"], r["V"])
    x, E, evals, iters, status = p.minimize(mref["frac0"], stopval=1e-20 * N)
    print(f"2D N=100: E={E:.3e} evals={evals} iters={iters} status={status} (reference: E={float(mref['E']):.3e} "
          f"evals={int(mref['evals'])})")
    assert status == 1 and E / N < 1e-20
    # the reference's own FP64 energy of the GPU result
    ref = oracle.Ref(2, r["basis"], r["V"], modes=r["modes"])
    ref.set_positions(x)
    Eref, _, _, _ = ref.eval(forces=False)
    assert Eref / N < 1e-20
    # stealthy window on both results
    K = float(mref["K"])
    kk = np.sqrt((oracle.lattice_k(r["basis"], mref["sk_modes"]) ** 2).sum(1))
    win = mref["sk_modes"][kk <= K * (1 + 1e-12)]
    assert _window_max_S(r["basis"], x, win) < 1e-10
    assert mref["S"][kk <= K * (1 + 1e-12)].max() < 1e-10


def test_ground_state_repeats_bitwise(gpu):
    r = load_golden("stealthy_2d_n100")
    mref = load_golden("min_2d_n100")
    p = gpu.CCPotential(2, r["basis"], r["modes"], r["V"])
    a = p.minimize(mref["frac0"], stopval=1e-20 * 100)
    b = p.minimize(mref["frac0"], stopval=1e-20 * 100)
    assert np.array_equal(a[0], b[0]) and a[1] == b[1] and a[2] == b[2]


def test_ground_state_3d_n2000(gpu):
    r = load_golden("stealthy_3d_n2000")
    N = 2000
    p = gpu.CCPotential(3, r["basis"], r["modes"], r["V"])
    x, E, evals, iters, status = p.minimize(r["frac"], stopval=1e-20 * N, max_evals=20000)
    print(f"3D N=2000: E={E:.3e} evals={evals} iters={iters} status={status}")
    assert E / N < 1e-20
    # S(k) in the window from the GPU, and a reference spot check of the window's largest values
    S = p.structure_factor(r["modes"])
    assert S.max() < 1e-10
    worst = r["modes"][np.argsort(S)[-50:]]
    assert _window_max_S(r["basis"], x, worst) < 1e-10


def test_precision_schedule_reaches_ground_state(gpu):
    """Mixed precision while far from the ground state, FP64 near it: the FP64 energy of the result is < 1e-20 N."""
    r = load_golden("stealthy_3d_n2000")
    N = 2000
    p = gpu.CCPotential(3, r["basis"], r["modes"], r["V"])
    x, E, evals, iters, status = p.minimize(r["frac"], stopval=1e-20 * N, max_evals=20000,
                                            precision=gpu.PREC_SCHEDULE, switch_energy_per_particle=1e-10)
    print(f"3D N=2000 schedule: E={E:.3e} evals={evals} iters={iters} status={status}")
    assert E / N < 1e-20


@pytest.mark.parametrize("history", [3, 64])
def test_ground_state_history_sizes(gpu, history):
    """The history at its smallest sizes (the ring wraps every few iterations) and at its largest (64 pairs, four
    full quarters of the update's history sum): alone and in a batch the configuration reaches its ground state,
    the reference's FP64 energy of the result agrees, and the batch of one ends bitwise where the mixed batch does
    (one instance takes the four-lane update, a batch the one-lane one: the same arithmetic)."""
    r = load_golden("stealthy_2d_n100")
    mref = load_golden("min_2d_n100")
    N = 100
    p = gpu.CCPotential(2, r["basis"], r["modes"], r["V"])
    x, E, evals, iters, status = p.minimize(mref["frac0"], stopval=1e-20 * N, history=history)
    print(f"history {history}: E={E:.3e} evals={evals} status={status}")
    assert E / N < 1e-20
    ref = oracle.Ref(2, r["basis"], r["V"], modes=r["modes"])
    ref.set_positions(x)
    Eref, _, _, _ = ref.eval(forces=False)
    assert Eref / N < 1e-20
    # in a batch with another instance, and alone in a batch of one
    basis2 = np.eye(3) * 300 ** (1.0 / 3.0)
    modes2, V2 = gpu.stealthy_kset(3, basis2, 300, 0.2, 3)
    other = gpu.CCPotential(3, basis2, modes2, V2)
    f2 = np.random.default_rng(4).random((300, 3))
    mix = gpu.CCBatch([p, other], [N, 300])
    xs, Es, es, its, sts = mix.minimize([mref["frac0"], f2], history=history)
    assert np.all(Es / np.array([N, 300]) < 1e-20)
    one = gpu.CCBatch([p], [N])
    xa, Ea, ea, ia, sa = one.minimize([mref["frac0"]], history=history)
    assert np.array_equal(xa[0], xs[0]) and Ea[0] == Es[0] and ea[0] == es[0]
