"""The potentials of the reference's collective-coordinate command-line program, built on the GPU.

GeneratePotential (apps/CollectiveCoordinateCLI/CollectiveCoordinateCLI.cpp:180-565) turns a cell, a particle count,
chi and a potential Type into a constrained wavevector set and a potential class:
  0-3     stealthy sets of ceil(chi N d) points completed to the shell, weights of Types 0-3 (the library's
          cc_kset_stealthy);
  4-8     half-space lattice points with |k| < 1, weight 1 (Type 4, 8), or, with K the |k| of the first point left
          out, (1 - |k|/K)^2 (5), (1 - |k|/K)^6 (6), 1 - |k| (7)            (:268-362);
  9-17    the points up to |k|^2 <= 1 (for 9 and 10 also the first shell beyond 1), collected by growing the radius
          from 1.1 by factors of 1.1 until the largest point reaches |k|^2 >= 1 (:363-542):
            9   weight 1 inside, -1e-4 on the outer shell;
            10  S2, S0 = 0 inside and S0out on the outer shell;
            11  S2, S0 = 1;   12  S2, S0 = a given constant;   13  S2, S0 = |k| / 2;
            14  S2, S0 = S0 |k|;   16  S2, S0 = S0 |k|^2;   17  S2, S0 = S0 |k|^n;
            15  S2 over Nc sub-configurations, S0 = S0 |k|;
  100     K2K2Potential (rK = 1), 101 KM3KnPotential(n) (rK = 1) (:543-556), the variable-cell classes of
          potential/CCPotential_Kernels.h at the bound cell (modules_b200.varbox).
The reference reads the extra parameters from its input stream; here they are keyword arguments (S0 for Types 10, 12,
14, 15, 16 and 17, n for 17 and 101, nsub for 15). As in the reference, chi is recomputed from the constraint count:
M / ((N - 1) d).

Growing the radius for Types 9-17 appends every point again at each step (the reference's list is not cleared); a
repeated point is one constraint here with its weight multiplied by its count, which leaves the energy and forces
unchanged. Thresholds compare |k|^2 formed from the reference's reciprocal basis; only a point within an ulp of
|k|^2 = 1 could fall on the other side.
"""
import math

import numpy as np

from .ccgpu import CCPotential, isotropic_kset, stealthy_kset
from .varbox import VarBoxPotential


def half_space_points(d, basis, R):
    """Integer modes and |k|^2 of the half-space lattice points with |k|^2 < R^2, by |k|^2."""
    modes, kamp = isotropic_kset(d, basis, R, R)
    k2 = kamp * kamp
    if d == 1:
        keep = k2 < R * R
        modes, k2 = modes[keep], k2[keep]
    return modes, k2


def _merge(modes, V, S0=None):
    """One constraint per distinct mode, its weight multiplied by the number of copies (targets are per mode); the
    count before merging is the reference's constraint count."""
    if len(modes) == 0:
        return modes, V, S0, 0
    u, first, counts = np.unique(modes, axis=0, return_index=True, return_counts=True)
    return (np.ascontiguousarray(u, np.int32), V[first] * counts,
            None if S0 is None else np.ascontiguousarray(S0[first]), len(modes))


def constraint_set(type_, d, basis, N, chi=0.0, S0=None, n=None):
    """(modes, V, S0 or None, M) of GeneratePotential for Types 0-17; M counts the reference's constraints (repeated
    points included)."""
    basis = np.ascontiguousarray(basis, np.float64).reshape(d, d)
    if type_ < 4:
        modes, V = stealthy_kset(d, basis, N, chi, type_)
        return modes, V, None, len(V)
    if type_ < 9:
        modes, k2 = half_space_points(d, basis, 1.0)
        V = np.ones(len(modes))
        if type_ in (5, 6, 7):
            M = len(modes)
            R = 1.2
            while True:
                _, k2all = half_space_points(d, basis, R)
                if len(k2all) > M:
                    break
                R *= 1.2
            K2 = np.partition(k2all, M)[M]
            kl = np.sqrt(k2)
            if type_ == 5:
                V = (1.0 - np.sqrt(k2 / K2)) ** 2
            elif type_ == 6:
                V = (1.0 - np.sqrt(k2 / K2)) ** 6
            else:
                V = 1.0 - kl
        return modes, V, None, len(V)
    if type_ > 17:
        raise ValueError("GeneratePotential types are 0-17, 100 and 101")
    if type_ in (10, 12, 14, 15, 16, 17) and S0 is None:
        raise ValueError("Type %d takes S0" % type_)
    if type_ == 17 and n is None:
        raise ValueError("Type 17 takes n")
    # the growing collection of :374-398
    parts_m, parts_k2 = [], []
    R = 1.1
    while True:
        m, k2 = half_space_points(d, basis, R)
        parts_m.append(m)
        parts_k2.append(k2)
        k2all = np.concatenate(parts_k2)
        if len(k2all) and k2all.max() >= 1.0:
            break
        R *= 1.1
    modes = np.concatenate(parts_m)
    order = np.argsort(k2all, kind="stable")
    modes, k2 = modes[order], k2all[order]
    if type_ in (9, 10):
        keep = np.ones(len(k2), bool)
        prev = 0.0
        for i, q in enumerate(k2):
            if prev > 1.0 and (q - prev) / prev > 1e-9:
                keep[i:] = False
                break
            prev = q
    else:
        keep = k2 <= 1.0
    modes, k2 = modes[keep], k2[keep]
    kl = np.sqrt(k2)
    if type_ == 9:
        return _merge(modes, np.where(k2 > 1.0, -1e-4, 1.0))
    ones = np.ones(len(modes))
    if type_ == 10:
        target = np.where(k2 > 1.0, float(S0), 0.0)
    elif type_ == 11:
        target = ones.copy()
    elif type_ == 12:
        target = np.full(len(modes), float(S0))
    elif type_ == 13:
        target = kl / 2
    elif type_ in (14, 15):
        target = kl * S0
    elif type_ == 16:
        target = k2 * S0
    else:
        target = k2 ** (n * 0.5) * S0
    return _merge(modes, ones, target)


def generate_potential(type_, d, basis, N, chi=0.0, S0=None, n=None, nsub=None):
    """(potential, chi) for a GeneratePotential Type: a CCPotential (plain, S2, or S2 over nsub sub-configurations for
    Type 15) or, for Types 100 and 101, a VarBoxPotential to bind with set_configuration(basis, frac)."""
    basis = np.ascontiguousarray(basis, np.float64).reshape(d, d)
    if type_ == 100:
        return VarBoxPotential("K2K2Potential", d, 1.0), None
    if type_ == 101:
        if n is None:
            raise ValueError("Type 101 takes n")
        return VarBoxPotential("KM3KnPotential", d, 1.0, n), None
    if type_ == 15 and not nsub:
        raise ValueError("Type 15 takes the sub-configuration count nsub")
    modes, V, target, M = constraint_set(type_, d, basis, N, chi, S0, n)
    chi_out = M / ((N - 1) * d) if N > 1 else math.nan
    if target is None:
        return CCPotential(d, basis, modes, V, 0.0), chi_out
    return CCPotential(d, basis, modes, V, 0.0, S0=target, nsub=nsub if type_ == 15 else 1), chi_out
