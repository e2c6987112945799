"""Golden vectors of the isotropic structure factor, made by running the REFERENCE's own IsotropicStructureFactor
(pairstat/StructureFactor.cpp:79-260, compiled from the reference tree into oracle/_ref/libccref.so) and the
oracle's GetKs restatement (oracle/sk_oracle.cpp, after core/PeriodicCellList.cpp:509-735).

Run in a container where the reference tree exists:  python tests/golden/make_golden_isotropic.py
Inputs are seeded here (numpy PCG64): uniform random fractional positions in square, skew, cubic and 1D cells; the
parameters cover the three averaging options, the circle-only and the linear (multiples of each direction) wavevector
lists, a lower cut, sampling, an automatic bin width and cells that change between configurations.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

CASES = [
    # name, d, bases (one per configuration), N per configuration, circ, lin, kprec, p, option, kmin
    ("sq2d_opt0", 2, [np.eye(2) * np.sqrt(200)] * 3, [200, 200, 200], 4.0, 4.0, 0.1, 1.0, 0, 0.0),
    ("sq2d_opt1", 2, [np.eye(2) * np.sqrt(200)] * 3, [200, 200, 200], 4.0, 4.0, 0.1, 1.0, 1, 0.0),
    ("skew2d_linear", 2, [np.array([[15.0, 0.0], [4.0, 13.0]])] * 2, [180, 180], 1.0, 6.0, 0.05, 1.0, 0, 0.0),
    ("skew2d_linear_opt1", 2, [np.array([[15.0, 0.0], [4.0, 13.0]])] * 2, [180, 180], 1.0, 6.0, 0.05, 1.0, 1, 0.0),
    ("cube3d_opt2", 3, [np.eye(3) * 300 ** (1 / 3)] * 2, [300, 300], 5.0, 5.0, 0.1, 1.0, 2, 0.0),
    ("cube3d_kmin_sampled", 3, [np.eye(3) * 300 ** (1 / 3)] * 2, [300, 300], 2.0, 6.0, 0.2, 0.6, 0, 0.5),
    ("cells_change_2d", 2, [np.eye(2) * 12.0, np.eye(2) * 13.0], [150, 160], 3.0, 3.0, 0.1, 1.0, 0, 0.0),
    ("auto_width_2d", 2, [np.eye(2) * 14.0] * 2, [196, 196], 5.0, 5.0, 0.0, 1.0, 1, 0.0),
    ("line1d", 1, [np.eye(1) * 100.0] * 2, [100, 100], 1.0, 5.0, 0.05, 0.6, 0, 0.3),
    ("line1d_plain", 1, [np.eye(1) * 100.0] * 2, [100, 100], 1.0, 5.0, 0.05, 1.0, 0, 0.0),
]


def main():
    if not oracle.ref_available():
        oracle.build(ref=True)
    rng = np.random.default_rng(20261203)
    rec = {}
    for name, d, bases, Ns, circ, lin, kprec, p, option, kmin in CASES:
        fracs = [rng.random((n, d)) for n in Ns]
        rows = oracle.ref_isotropic_sk(d, bases, fracs, circ, lin, kprec, p, option, kmin)
        ks = oracle.ref_getks(d, bases[0], circ, lin, p, kmin)
        rec.update({f"{name}__d": d, f"{name}__bases": np.asarray(bases, np.float64),
                    f"{name}__N": np.asarray(Ns, np.int64), f"{name}__frac": np.concatenate(fracs),
                    f"{name}__params": np.array([circ, lin, kprec, p, option, kmin], np.float64),
                    f"{name}__rows": rows, f"{name}__ks": ks})
        print(f"{name}: {len(rows)} rows, {len(ks)} wavevectors of the first cell")
    rec["names"] = np.array([c[0] for c in CASES])
    np.savez_compressed(os.path.join(HERE, "isotropic_sk.npz"), **rec)


if __name__ == "__main__":
    main()
