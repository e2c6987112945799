"""Evaluate one synthetic stealthy configuration a few times (for profiling a single kernel launch sequence).

    python -m modules_b200.evalcase --d 2 --N 20000 --chi 0.2 --evals 3 [--mixed] [--fused]

The configuration: N uniform random points (seed 1) in a periodic cube of unit density, the CLI's Type 0 k-set.
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
    ap.add_argument("--fused", action="store_true")
    a = ap.parse_args()
    basis = np.eye(a.d) * a.N ** (1.0 / a.d)
    modes, V = cc.stealthy_kset(a.d, basis, a.N, a.chi)
    pot = cc.CCPotential(a.d, basis, modes, V)
    pot.set_path(1 if a.fused else 0)
    pot.set_configuration(np.random.default_rng(1).random((a.N, a.d)))
    E = None
    for _ in range(a.evals):
        E, _F = pot.energy_and_forces(precision=cc.PREC_MIXED if a.mixed else cc.PREC_FP64)
    print(f"d={a.d} N={a.N} M={len(V)} E={E:.12e}")


if __name__ == "__main__":
    main()
