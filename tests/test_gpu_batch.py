"""Batches of uneven configurations in one launch per dimension: same results as each configuration alone."""
import numpy as np
import pytest

from conftest import load_golden, scales

pytestmark = pytest.mark.gpu


def _instances(gpu, specs, seed=11):
    rng = np.random.default_rng(seed)
    pots, N, fracs = [], [], []
    for d, n, chi, typ in specs:
        basis = np.eye(d) * n ** (1.0 / d)
        modes, V = gpu.stealthy_kset(d, basis, n, chi, typ)
        pots.append(gpu.CCPotential(d, basis, modes, V))
        N.append(n)
        fracs.append(rng.random((n, d)))
    return pots, N, fracs


SPECS = [(2, 200, 0.3, 3), (3, 300, 0.12, 3), (2, 1000, 0.45, 3), (3, 700, 0.25, 3), (2, 64, 0.40, 0),
         (3, 2000, 0.45, 0)]


def test_batch_matches_each_instance(gpu):
    pots, N, fracs = _instances(gpu, SPECS)
    batch = gpu.CCBatch(pots, N)
    batch.set_positions(fracs)
    E, F = batch.energy_and_forces()
    for p, f, e, fb in zip(pots, fracs, E, F):
        p.set_configuration(f)
        e1, f1 = p.energy_and_forces()
        assert abs(e - e1) <= 1e-10 * abs(e1)
        assert np.abs(fb - f1).max() <= 1e-10 * np.abs(f1).max()


def test_batch_ensemble_of_one_potential(gpu):
    """Many configurations of one potential in one fused launch (the ensemble form of the benchmark's
    configuration): each instance's energy and forces equal those of the same instance in a batch of one, bitwise,
    and agree with the three-kernel evaluation of the potential to rounding."""
    d, n, chi = 3, 400, 0.40
    basis = np.eye(d) * n ** (1.0 / d)
    modes, V = gpu.stealthy_kset(d, basis, n, chi)
    B = 24
    pots = [gpu.CCPotential(d, basis, modes, V) for _ in range(B)]
    fracs = list(np.random.default_rng(21).random((B, n, d)))
    ens = gpu.CCBatch(pots, [n] * B)
    ens.set_positions(fracs)
    E, F = ens.energy_and_forces()
    for k in (0, 7, B - 1):
        one = gpu.CCBatch([pots[k]], [n])
        one.set_positions([fracs[k]])
        e1, f1 = one.energy_and_forces()
        assert e1[0] == E[k] and np.array_equal(f1[0], F[k])
        pots[k].set_configuration(fracs[k])
        e2, f2 = pots[k].energy_and_forces()
        assert abs(E[k] - e2) <= 1e-10 * abs(e2)
        assert np.abs(F[k] - f2).max() <= 1e-10 * np.abs(f2).max()


def test_batch_golden_parity(gpu):
    """A batch of the golden cases (1D-3D, skew cells, repeated modes) against the reference's results."""
    names = ["lattice_1d", "lattice_2d_skew", "lattice_3d_skew", "weighted_3d_n300", "stealthy_3d_n2000"]
    recs = [load_golden(n) for n in names]
    pots = [gpu.CCPotential(int(r["d"]), r["basis"], r["modes"], r["V"], float(r["shift"])) for r in recs]
    batch = gpu.CCBatch(pots, [len(r["frac"]) for r in recs])
    batch.set_positions([r["frac"] for r in recs])
    E, F = batch.energy_and_forces()
    for r, e, f in zip(recs, E, F):
        s = scales(r)
        assert abs(e - float(r["E"])) <= 1e-10 * abs(float(r["E"])) + 1e-13 * s["energy"]
        assert np.abs(f - r["F"]).max() <= 1e-10 * s["force"]


def test_batch_minimize_same_alone_and_in_mix(gpu):
    """Continuous batching must not change results: an instance minimised in a mixed batch ends bitwise where it
    ends when minimised alone, and every instance reaches its ground state (Phi/N < 1e-20)."""
    pots, N, fracs = _instances(gpu, SPECS[:5], seed=3)
    batch = gpu.CCBatch(pots, N)
    xs, E, evals, iters, status = batch.minimize(fracs)
    print("batch:", [f"{e / n:.1e}" for e, n in zip(E, N)], evals.tolist())
    assert np.all(E / np.array(N) < 1e-20)
    for k in (0, 3):
        alone = gpu.CCBatch([pots[k]], [N[k]])
        xa, Ea, ea, ia, sa = alone.minimize([fracs[k]])
        assert np.array_equal(xa[0], xs[k]) and Ea[0] == E[k] and ea[0] == evals[k]


def test_batch_precision_schedule_reaches_ground_states(gpu):
    """Mixed precision first, FP64 per instance once E/N <= 1e-10 or the mixed stage stalls: every instance ends
    at Phi/N < 1e-20 (FP64 energy of the result)."""
    pots, N, fracs = _instances(gpu, SPECS[:5], seed=8)
    batch = gpu.CCBatch(pots, N)
    xs, E, evals, iters, status = batch.minimize(fracs, precision=gpu.PREC_SCHEDULE, switch_energy_per_particle=1e-10)
    print("schedule:", [f"{e / n:.1e}" for e, n in zip(E, N)], evals.tolist(), status.tolist())
    assert np.all(E / np.array(N) < 1e-20)


def test_batch_autotune_keeps_results(gpu):
    """The autotuner picks one of the candidate tile shapes; results before and after agree to rounding, and a tuned
    batch still evaluates every instance as before within 1e-12 relative."""
    pots, N, fracs = _instances(gpu, SPECS, seed=11)
    batch = gpu.CCBatch(pots, N)
    batch.set_positions(fracs)
    E0, F0 = batch.energy_and_forces()
    ps, sg = batch.autotune(reps=1)
    cands = (32, 64, 128, 256, 512, 1024)   # include/cc_gpu.h cc_batch_autotune: 6 x 6 candidate shapes
    assert ps in cands and sg in cands
    E1, F1 = batch.energy_and_forces()
    for e0, e1, f0, f1 in zip(E0, E1, F0, F1):
        assert abs(e1 - e0) <= 1e-12 * abs(e0)
        assert np.abs(f1 - f0).max() <= 1e-12 * max(np.abs(f0).max(), 1.0)


@pytest.mark.parametrize("precision", ["fp64", "schedule"])
def test_batch_ground_states_against_reference(gpu, precision):
    """The north star's bar on batched ground states: the reference's own FP64 energy of each final configuration
    (oracle/_ref, potential/CollectiveCoordinatePotential.h:1351-1372) is below 1e-20 per particle and within 1e-12
    per particle of the GPU's energy."""
    import oracle
    if not oracle.ref_available():
        pytest.skip("reference oracle not built")
    pots, N, fracs = _instances(gpu, SPECS[:5], seed=21)
    batch = gpu.CCBatch(pots, N)
    prec = gpu.PREC_FP64 if precision == "fp64" else gpu.PREC_SCHEDULE
    xs, E, evals, iters, status = batch.minimize(fracs, precision=prec, switch_energy_per_particle=1e-10)
    for (d, n, chi, typ), x, e in zip(SPECS[:5], xs, E):
        basis = np.eye(d) * n ** (1.0 / d)
        modes, V = gpu.stealthy_kset(d, basis, n, chi, typ)
        ref = oracle.Ref(d, basis, V, modes=modes)
        ref.set_positions(x)
        Er = ref.eval(forces=False)[0]
        print(f"d={d} N={n}: GPU E/N={e / n:.3e} reference E/N={Er / n:.3e}")
        # the stop rule is the GPU's E <= 1e-20 N; the reference's sum of the same configuration differs by rounding
        # (|rho| ~ 1e-10 near the ground state, its rounding ~1e-15: ~1e-5 relative in E)
        assert Er / n < 1.001e-20 and abs(e - Er) / n <= 1e-12


def test_batch_counts_survive_finished_instances(gpu):
    """A batched minimisation in which instances finish at very different times (skipped item by item while the others
    run), then a second minimisation of the same batch from new starts: every instance ends where it ends alone. The
    fused launch's per-instance counts must be zero again after every launch, whatever instances were skipped."""
    specs = [(2, 64, 0.40, 0), (3, 700, 0.25, 3), (2, 250, 0.40, 3), (3, 120, 0.25, 0)]
    pots, N, fracs = _instances(gpu, specs, seed=4)
    batch = gpu.CCBatch(pots, N)
    for seed in (4, 6):
        rng = np.random.default_rng(seed)
        starts = [rng.random((n, p.d)) for n, p in zip(N, pots)]
        xs, E, evals, iters, status = batch.minimize(starts)
        assert np.all(E / np.array(N) < 1e-20), (E / np.array(N), evals)
        for k in range(len(pots)):
            alone = gpu.CCBatch([pots[k]], [N[k]])
            xa, Ea, ea, ia, sa = alone.minimize([starts[k]])
            assert np.array_equal(xa[0], xs[k]) and Ea[0] == E[k] and ea[0] == evals[k]
