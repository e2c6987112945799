"""Evaluate one synthetic stealthy configuration a few times (for profiling a single kernel launch sequence).

    python -m modules_b200.evalcase --d 2 --N 20000 --chi 0.2 --evals 3 [--mixed] [--path split|nufft|auto]
    python -m modules_b200.evalcase --batch 512 --evals 3 [--mixed] [--autotune]
    python -m modules_b200.evalcase --serve 120
    python -m modules_b200.evalcase --d 3 --N 2000 --chi 0.45 --minimize [--mixed]

The configuration: N uniform random points (seed 1) in a periodic cube of unit density, the CLI's Type 0 k-set.
With --batch: the seeded batch of uneven instances of the benchmark (modules_b200.workloads.batched_workload),
evaluated as one batch (the fused batch kernel) with the default tile shape, or with --autotune the shape the
autotuner picks (as the benchmark does).
With --serve: the seeded served stream of the benchmark (modules_b200.workloads.served_stream: arrivals at 60/s,
N <= 4000, chi <= 0.40) through modules_b200.serve with 16 iterations per round.
With --minimize: one L-BFGS minimisation of the configuration to Phi/N < 1e-20 (FP64, or with --mixed the precision
schedule).
"""
import argparse

import numpy as np

import modules_b200 as cc


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--d", type=int, default=2)
    ap.add_argument("--N", type=int, default=20000)
    ap.add_argument("--chi", type=float, default=0.2)
    ap.add_argument("--evals", type=int, default=3)
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--path", default="split", choices=["split", "nufft", "auto"])
    ap.add_argument("--batch", type=int, default=0, help="evaluate the seeded batch of this many instances")
    ap.add_argument("--serve", type=int, default=0, help="serve the seeded stream of this many requests")
    ap.add_argument("--minimize", action="store_true", help="minimise the configuration to its ground state")
    ap.add_argument("--autotune", action="store_true", help="with --batch: autotune the tile shape first")
    a = ap.parse_args()
    if a.serve > 0:
        from .workloads import served_stream
        reqs = served_stream(a.serve)
        res, wall = cc.serve(reqs, iters_per_round=16)
        reached = sum(r["E"] / q["N"] < 1e-20 for r, q in zip(res, reqs))
        print(f"served {a.serve} requests in {wall:.2f} s, {reached} reached E/N < 1e-20")
        return
    if a.batch > 0:
        from .workloads import batched_workload
        pots, Ns, fracs, pairs = batched_workload(cc, a.batch)
        batch = cc.CCBatch(pots, Ns)
        batch.set_positions(fracs)
        if a.autotune:
            print("tile", batch.autotune(reps=2))
        for _ in range(a.evals):
            E, _F = batch.energy_and_forces(precision=cc.PREC_MIXED if a.mixed else cc.PREC_FP64)
        print(f"batch of {a.batch}: {pairs} particle-k pairs, sum E={float(np.sum(E)):.12e}")
        return
    basis = np.eye(a.d) * a.N ** (1.0 / a.d)
    modes, V = cc.stealthy_kset(a.d, basis, a.N, a.chi)
    pot = cc.CCPotential(a.d, basis, modes, V)
    paths = {"split": cc.PATH_SPLIT, "nufft": cc.PATH_NUFFT, "auto": cc.PATH_AUTO}
    pot.set_path(paths[a.path])
    frac = np.random.default_rng(1).random((a.N, a.d))
    if a.minimize:
        prec = cc.PREC_SCHEDULE if a.mixed else cc.PREC_FP64
        x, E, ev, it, st = pot.minimize(frac, stopval=1e-20 * a.N, precision=prec)
        print(f"d={a.d} N={a.N} M={len(V)} minimised: E/N={E / a.N:.3e} evals={ev} iters={it} status={st}")
        return
    pot.set_configuration(frac)
    E = None
    for _ in range(a.evals):
        E, _F = pot.energy_and_forces(precision=cc.PREC_MIXED if a.mixed else cc.PREC_FP64)
    print(f"d={a.d} N={a.N} M={len(V)} E={E:.12e}")


if __name__ == "__main__":
    main()
