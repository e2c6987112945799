"""Golden vectors of the multi-species stealthy potential with soft-core contact, made by running the REFERENCE's own
MultiStealthyPotential (apps/CCOptimization/MultiStealthyPotential.{h,cpp}, compiled from the reference tree into
oracle/_ref/libccref.so).

Run in a container where the reference tree exists:  python tests/golden/make_golden_multi.py
Inputs are seeded here (numpy PCG64). The cases follow the reference's test_fused_contact.cpp: dimensions 1-3,
orthogonal and skew cells, 1, 2 and 5 species interleaved in particle order, equal and unequal radii (0.7-1.3 times
the mean radius of packing fraction 0.2 at unit number density), contact on and off, a small cell where a particle
touches several images of one neighbour and its own images, and coincident particles. Each species carries the CLI's
stealthy k-set (Type 0, or Type 3 weights) for its own particle count.
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

VD = {1: 2.0, 2: math.pi, 3: 4.0 * math.pi / 3.0}


def cell(d, N, skew):
    L = N ** (1.0 / d)
    A = np.eye(d) * L
    if skew and d >= 2:
        A[1, 0] = 0.3 * L
        if d == 3:
            A[2, 0], A[2, 1] = -0.2 * L, 0.25 * L
    return A


CASES = [
    # name, d, N, skew, species, chi, e0, u0, radii ("none" | "equal" | "unequal"), kset type, coincident, side
    ("d1_s2_equal", 1, 60, False, 2, 0.2, 1.0, 1.0, "equal", 0, 0, None),
    ("d2_s1_default_radii", 2, 120, False, 1, 0.25, 1.0, 1.0, "none", 0, 0, None),
    ("d2_s2_skew_unequal", 2, 150, True, 2, 0.2, 1.0, 1.0, "unequal", 0, 0, None),
    ("d2_s5_contact_off", 2, 200, False, 5, 0.15, 0.0, 1.0, "equal", 3, 0, None),
    ("d3_s2_unequal", 3, 160, False, 2, 0.2, 0.5, 2.5, "unequal", 0, 0, None),
    ("d3_s5_skew", 3, 250, True, 5, 0.1, 1.0, 1.0, "equal", 3, 0, None),
    ("d2_small_cell_images", 2, 6, False, 2, 0.3, 1.0, 1.0, "equal", 0, 0, 1.2),
    ("d3_coincident", 3, 40, False, 2, 0.2, 1.0, 1.0, "equal", 0, 2, None),
]


def main():
    if not oracle.ref_available():
        oracle.build(ref=True)
    rng = np.random.default_rng(20261204)
    rec = {}
    for name, d, N, skew, S, chi, e0, u0, rkind, ktype, coincident, side in CASES:
        A = np.eye(d) * side if side else cell(d, N, skew)
        frac = rng.random((N, d))
        for k in range(coincident):
            frac[N - 1 - k] = frac[k]
        species = (np.arange(N) % S).astype(np.int32)
        R0 = (0.2 / VD[d]) ** (1.0 / d) if not side else 0.5
        radii = None
        if rkind == "equal":
            radii = np.full(N, R0)
        elif rkind == "unequal":
            radii = R0 * rng.uniform(0.7, 1.3, N)
        modes, Vs, ks = [], [], []
        for s in range(S):
            Ns = int((species == s).sum())
            m, V = oracle.ref_kset(d, A, max(Ns, 1), chi, ktype)
            modes.append(m)
            Vs.append(V)
            ks.append(oracle.lattice_k(A, m))
        E, F = oracle.ref_multi_eval(d, A, ks, Vs, u0, e0, frac, species, radii)
        rec.update({f"{name}__d": d, f"{name}__basis": A, f"{name}__frac": frac, f"{name}__species": species,
                    f"{name}__radii": radii if radii is not None else np.zeros(0), f"{name}__u0": u0,
                    f"{name}__e0": e0, f"{name}__M": np.array([len(v) for v in Vs], np.int64),
                    f"{name}__modes": np.concatenate(modes), f"{name}__V": np.concatenate(Vs), f"{name}__E": E,
                    f"{name}__F": F})
        print(f"{name}: N={N} S={S} M={[len(v) for v in Vs]} E={E:.6e} max|F|={np.abs(F).max():.3e}")
    rec["names"] = np.array([c[0] for c in CASES])
    np.savez_compressed(os.path.join(HERE, "multi_stealthy.npz"), **rec)


if __name__ == "__main__":
    main()
