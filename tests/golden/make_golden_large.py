"""Golden vectors of the large 2D workload, made by running the REFERENCE ITSELF (oracle/_ref/libccref.so, the
reference's ShiftedCCPotential Direct path compiled from its own sources by oracle/Makefile).

Workload: N = 100000 points uniform (seed 11, numpy PCG64) in a periodic square of unit density (side sqrt(N)), the
CLI's Type 0 k-set at chi = 0.20 (GeneratePotential, apps/CollectiveCoordinateCLI/CollectiveCoordinateCLI.cpp:180-300:
M = 40002 half-space wavevectors, v(k) = 1): about 4e9 particle-k pairs. One Energy + AllForce + GetRho of the
reference (potential/CollectiveCoordinatePotential.h:1255-1394, 1434-1448) on all host cores; about a minute on 8.

Run where the reference tree exists:  python tests/golden/make_golden_large.py
Writes tests/golden/large_2d_n100000.npz: d, basis, modes, V, frac, E, F (Cartesian), rho_re, rho_im, volume, seconds.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

D, N, CHI, SEED = 2, 100000, 0.20, 11


def main():
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libccref.so is not built (python -c 'import oracle; oracle.build(ref_tree=...)')")
    basis = np.eye(D) * np.sqrt(float(N))
    modes, V = oracle.ref_kset(D, basis, N, CHI, 0)
    frac = np.random.default_rng(SEED).random((N, D))
    ref = oracle.Ref(D, basis, V, modes=modes)
    ref.set_positions(frac)
    t0 = time.time()
    E, F, re, im = ref.eval()
    dt = time.time() - t0
    np.savez_compressed(os.path.join(HERE, "large_2d_n100000.npz"), d=D, basis=basis, modes=modes, V=V, frac=frac,
                        E=E, F=F, rho_re=re, rho_im=im, volume=ref.volume(), seconds=dt, chi=CHI, seed=SEED)
    print(f"large_2d_n100000: N={N} M={len(V)} E={E:.17g} ({dt:.1f} s on {os.cpu_count()} threads)")


if __name__ == "__main__":
    main()
