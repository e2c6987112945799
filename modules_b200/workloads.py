"""Synthetic workloads shared by the benchmark and the profiling entry point (seeded, so both see the same inputs)."""
import numpy as np


def batched_workload(cc, count, seed=2024):
    """`count` independent stealthy configurations: d in {2,3}, N log-uniform in [200, 5000], chi U[0.10, 0.49],
    v(k) = (1 - |k|/K)^2 (GeneratePotential Type 3), unit density, uniform random positions.
    Returns (potentials, N per instance, fractional positions, particle-k pairs of one evaluation of all)."""
    rng = np.random.default_rng(seed)
    pots, Ns, fracs, pairs = [], [], [], 0
    for _ in range(count):
        d = int(rng.choice([2, 3]))
        n = int(round(np.exp(rng.uniform(np.log(200), np.log(5000)))))
        chi = float(rng.uniform(0.10, 0.49))
        basis = np.eye(d) * n ** (1.0 / d)
        modes, V = cc.stealthy_kset(d, basis, n, chi, 3)
        pots.append(cc.CCPotential(d, basis, modes, V))
        Ns.append(n)
        fracs.append(rng.random((n, d)))
        pairs += n * len(V)
    return pots, Ns, fracs, pairs
