"""Generate the golden vectors of the CC path by running the REFERENCE ITSELF (oracle/_ref/libccref.so: the reference's
ShiftedCCPotential, Configuration and LuksanPLIS compiled from its own sources by oracle/Makefile).

Run in a container where the reference tree exists:  python tests/golden/make_golden.py
Inputs are seeded here (numpy PCG64); the case shapes follow the reference's own tests
(potential/tests/finufft_type1/test_finufft_type1.cpp: TestSign :387-440, TestEmpty :442-487, TestLatticeCases
:489-521, TestFiniteDifference :660-703, TestSmokeN500 :804-846) and the workloads named for this path
(2D N=100 chi=0.30; 3D N=2000 chi=0.45; a (1-|k|/K)^2 weighted instance; 2D N=1e5 chi=0.20 k-set).
Each case file holds: d, basis, modes, V, shift, frac, and the reference's E, F (Cartesian), rho_re, rho_im.
"""
import hashlib
import itertools
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402


def all_modes(d, K):
    """All integer modes in [-K, K]^d (the reference test's AllModes, first index fastest)."""
    out = []
    for t in itertools.product(range(-K, K + 1), repeat=d):
        out.append(t[::-1])
    return np.array(out, np.int32).reshape(-1, d)


def scramble(modes, dups, rng):
    modes = modes[rng.permutation(len(modes))]
    for _ in range(dups):
        c = modes[rng.integers(len(modes))]
        pos = rng.integers(len(modes) + 1)
        modes = np.insert(modes, pos, c, axis=0)
    return modes


def run_case(name, d, basis, modes, V, frac, shift=0.0, extra=None):
    basis = np.asarray(basis, np.float64).reshape(d, d)
    ref = oracle.Ref(d, basis, V, modes=modes, shift=shift)
    ref.set_positions(frac)
    E, F, re, im = ref.eval()
    rec = dict(d=d, basis=basis, modes=np.asarray(modes, np.int32).reshape(-1, d), V=np.asarray(V, np.float64),
               shift=shift, frac=np.asarray(frac, np.float64).reshape(-1, d), E=E, F=F, rho_re=re, rho_im=im,
               kcart=ref.kcart(), volume=ref.volume())
    if extra:
        rec.update(extra)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **rec)
    print(f"{name}: d={d} N={len(rec['frac'])} M={len(V)} E={E:.17g}")
    return ref, rec


def main():
    oracle.build()
    rng = np.random.default_rng(20261203)

    # analytic sign checks (TestSign)
    run_case("sign_1d", 1, [[1.0]], [[1], [-1], [0]], [1.0, 1.0, 1.0], [[0.25]])
    run_case("sign_2d_skew", 2, [[1.0, 0.0], [0.4, 0.9]], [[1, 1], [-2, 3]], [1.0, 1.0], [[0.25, 0.125]])

    # empty constraint list / empty particle list (TestEmpty)
    run_case("empty_constraints", 2, [[1.0, 0.0], [0.3, 1.1]], np.zeros((0, 2), np.int32), np.zeros(0),
             rng.random((12, 2)), shift=0.7)
    m = all_modes(3, 1)
    run_case("empty_particles", 3, np.eye(3), m, rng.uniform(0.5, 1.5, len(m)), np.zeros((0, 3)))

    # lattice cases: scrambled full mode cubes with duplicates, random V in [-0.5, 1.5], Shift 0.25
    cases = [
        ("lattice_1d", 1, [[2.7]], 64, 25),
        ("lattice_2d_orthogonal", 2, [[1.3, 0.0], [0.0, 0.8]], 100, 7),
        ("lattice_2d_skew", 2, [[1.3, 0.0], [0.45, 0.9]], 100, 7),
        ("lattice_2d_rotated_skew", 2, [[1.0, 0.3], [-0.4, 1.1]], 100, 6),
        ("lattice_3d_orthogonal", 3, [[1.0, 0.0, 0.0], [0.0, 1.2, 0.0], [0.0, 0.0, 0.9]], 60, 3),
        ("lattice_3d_skew", 3, [[1.1, 0.0, 0.0], [0.3, 0.95, 0.1], [0.2, -0.25, 1.2]], 60, 3),
    ]
    for name, d, basis, n, K in cases:
        modes = scramble(all_modes(d, K), 7, rng)
        run_case(name, d, basis, modes, rng.uniform(-0.5, 1.5, len(modes)), rng.random((n, d)), shift=0.25)

    # finite-difference case (TestFiniteDifference): 2D skew, N=30, modes |n|<=4 with duplicates, V in [0.2,1.2]
    modes = scramble(all_modes(2, 4), 2, rng)
    run_case("fd_2d_skew", 2, [[1.3, 0.0], [0.45, 0.9]], modes, rng.uniform(0.2, 1.2, len(modes)),
             rng.random((30, 2)))

    # seeded N=500 2D smoke (TestSmokeN500): the 299 shortest half-plane modes ordered by (|m|^2, m1, m0), V=1
    R = 16
    sm = [(m0, m1) for m1 in range(-R, R + 1) for m0 in range(-R, R + 1)
          if m0 * m0 + m1 * m1 <= R * R and (m1 > 0 or (m1 == 0 and m0 > 0))]
    sm.sort(key=lambda t: (t[0] ** 2 + t[1] ** 2, t[1], t[0]))
    L = np.sqrt(500.0)
    run_case("smoke_n500_2d", 2, [[L, 0.0], [0.0, L]], np.array(sm[:299], np.int32), np.ones(299),
             rng.random((500, 2)))

    # the stealthy workloads: the CLI k-set (GeneratePotential Type 0 / Type 3) on unit-density or unit cells
    ks = {}
    for name, d, N, chi, side, typ in [("ks_2d_n100_chi030", 2, 100, 0.30, 1.0, 0),
                                       ("ks_3d_n2000_chi045", 3, 2000, 0.45, 2000 ** (1 / 3), 0),
                                       ("ks_3d_n300_chi030_t3", 3, 300, 0.30, 300 ** (1 / 3), 3),
                                       ("ks_2d_n100000_chi020", 2, 100000, 0.20, np.sqrt(1e5), 0)]:
        basis = np.eye(d) * side
        modes, V = oracle.ref_kset(d, basis, N, chi, typ)
        order = np.lexsort(modes.T[::-1])
        key = np.ascontiguousarray(modes[order])
        ks[name] = dict(d=d, N=N, chi=chi, side=side, type=typ, M=len(V), sha=hashlib.sha256(key.tobytes()).hexdigest(),
                        modes=modes if len(V) <= 5000 else np.zeros((0, d), np.int32), V=V if len(V) <= 5000 else
                        np.zeros(0))
        print(f"{name}: M={len(V)}")
    np.savez_compressed(os.path.join(HERE, "ksets.npz"), **{f"{k}__{f}": v for k, r in ks.items() for f, v in r.items()})

    # 2D N=100 chi=0.30 (unit square): random start, then the reference's minimisation to Phi/N < 1e-20
    r = ks["ks_2d_n100_chi030"]
    frac = rng.random((100, 2))
    ref, rec = run_case("stealthy_2d_n100", 2, np.eye(2), r["modes"], r["V"], frac)
    t = time.time()
    Emin, xmin, evals = ref.minimize(frac, emin=1e-20 * 100)
    print(f"  minimise: E={Emin:.3e} evals={evals} ({time.time() - t:.2f}s)")
    ref.set_positions(xmin)
    # S(k) of the final configuration on every half-space lattice k with |k| <= 1.5 K
    K = np.sqrt((oracle.lattice_k(np.eye(2), r["modes"]) ** 2).sum(1)).max()
    sk_modes = halfspace_ball(2, np.eye(2), 1.5 * K)
    Sfin = ref.structure_factor(oracle.lattice_k(np.eye(2), sk_modes))
    np.savez_compressed(os.path.join(HERE, "min_2d_n100.npz"), frac0=frac, frac=xmin, E=Emin, evals=evals,
                        sk_modes=sk_modes, S=Sfin, K=K)

    # 3D N=2000 chi=0.45 (unit density): one evaluation at a random start
    r = ks["ks_3d_n2000_chi045"]
    side = r["side"]
    ref, rec = run_case("stealthy_3d_n2000", 3, np.eye(3) * side, r["modes"], r["V"], rng.random((2000, 3)))
    # S(k) at the same configuration on |k| <= 1.5 K (pairstat StructureFactor), reference values
    K = np.sqrt((oracle.lattice_k(np.eye(3) * side, r["modes"]) ** 2).sum(1)).max()
    sk_modes = halfspace_ball(3, np.eye(3) * side, 1.5 * K)
    S = ref.structure_factor(oracle.lattice_k(np.eye(3) * side, sk_modes))
    np.savez_compressed(os.path.join(HERE, "sk_3d_n2000.npz"), sk_modes=sk_modes, S=S, K=K)
    print(f"sk_3d_n2000: K_S={len(S)}")

    # (1-|k|/K)^2 weighted 3D instance (GeneratePotential Type 3)
    r = ks["ks_3d_n300_chi030_t3"]
    run_case("weighted_3d_n300", 3, np.eye(3) * r["side"], r["modes"], r["V"], rng.random((300, 3)))


def halfspace_ball(d, basis, kmax):
    """All half-space lattice modes (first nonzero index > 0) with |k| <= kmax, ordered by |k| then index."""
    B = 2 * np.pi * np.linalg.inv(np.asarray(basis, np.float64)).T
    bound = [int(np.floor(kmax * np.linalg.norm(basis[e]) / (2 * np.pi))) + 1 for e in range(d)]
    grids = np.meshgrid(*[np.arange(-b, b + 1) for b in bound], indexing="ij")
    n = np.stack([g.reshape(-1) for g in grids], 1).astype(np.int32)
    first = np.zeros(len(n), np.int64)
    for e in range(d - 1, -1, -1):
        first = np.where(n[:, e] != 0, n[:, e], first)
    n = n[first > 0]
    k2 = ((n @ B) ** 2).sum(1)
    n = n[k2 <= kmax * kmax * (1 + 1e-12)]
    k2 = ((n @ B) ** 2).sum(1)
    order = np.lexsort(tuple(n.T[::-1]) + (k2,))
    return np.ascontiguousarray(n[order])


if __name__ == "__main__":
    main()
