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


def served_stream(count, rate=60.0, nmax=4000, chimax=0.40, seed=99):
    """`count` ground-state requests with Poisson arrivals at `rate` per second: d in {2,3}, N log-normal (median
    1000, sigma 0.6) clipped to [100, nmax], chi U[0.05, chimax], v(k) = 1 or (1 - |k|/K)^2, uniform random start.
    Returns a list of request dicts for modules_b200.serve (seeded: the same arguments give the same stream)."""
    rng = np.random.default_rng(seed)
    reqs, t = [], 0.0
    for _ in range(count):
        t += rng.exponential(1.0 / rate)
        d = int(rng.choice([2, 3]))
        n = int(np.clip(np.exp(rng.normal(np.log(1000), 0.6)), 100, nmax))
        chi = float(rng.uniform(0.05, chimax))
        reqs.append(dict(d=d, N=n, chi=chi, vtype=int(rng.choice([0, 3])), frac0=rng.random((n, d)), arrival_s=t))
    return reqs
