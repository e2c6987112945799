"""The one-component collective-coordinate optimiser's potential (GetCCO, apps/CCOptimization/main.cpp:135-590) on
the GPU: its constraint set and v(k) shapes, and RepulsiveCCPotential (apps/CCOptimization/RepulsiveCCPotential.h:
21-159), a soft-core contact e0 (1 - r / sigma)^2 for r < sigma plus a ShiftedCCPotential, or a
ShiftedCCPotential_S2 when S0 != 0 ("equiluminous patterns").

Constraints (main.cpp:262-318): the wavevectors of GetKs(cell, k2, k2, 1) with |k|^2 > k1^2; for S0 == 0 the weight
v(|k|) is flat (1), overlap (alpha(d, |k| / k2), the intersection volume fraction of two d-balls of diameter 1 at
distance |k| / k2, core/etc.cpp:76-101) or power-law ((1 - |k| / k2)^m); for S0 != 0 the weight is 1 and every
target is S0. The potential runs as a one-species CCMulti (u0 = 1, radii sigma / 2), whose contact sum and
collective-coordinate part are the reference's two terms.
"""
import numpy as np

from .ccgpu import CCMulti, isotropic_kset


def alpha(d, x):
    """Intersection volume of two d-balls of diameter 1 whose centres are x apart, over one ball's volume (core/etc.cpp:
    76-101): 0 for x > 1; d = 1..5. The d = 5 polynomial is the reference's, whose x^5 coefficient (0.875) differs
    from the lens volume's (0.375): alpha(5, 1) = -0.5 there. The GPU potentials take d <= 3."""
    x = np.asarray(x, np.float64)
    if np.any(x < 0):
        raise ValueError("alpha: negative argument")
    with np.errstate(invalid="ignore"):
        if d == 1:
            v = 1.0 - x
        elif d == 2:
            v = 2.0 / np.pi * (np.arccos(np.minimum(x, 1.0)) - x * np.sqrt(np.maximum(1.0 - x * x, 0.0)))
        elif d == 3:
            v = 1.0 - 1.5 * x + 0.5 * x * x * x
        elif d == 4:
            v = 2.0 / np.pi * (np.arccos(np.minimum(x, 1.0)) -
                               (5.0 * x - 2.0 * x * x * x) / 3.0 * np.sqrt(np.maximum(1 - x * x, 0.0)))
        elif d == 5:
            v = 1.0 - 1.875 * x + 1.25 * x * x * x - 0.875 * x ** 5
        else:
            raise ValueError("alpha: dimension out of range")
    return np.where(x > 1.0, 0.0, v)


def cco_constraints(d, basis, k1, k2, vtilde="flat", m=None, S0=0.0):
    """(modes, V, S0 list or None) of GetCCO's collective-coordinate part for a cell."""
    if S0 == 0.0 and vtilde not in ("flat", "overlap", "power-law"):
        raise ValueError("unknown vtilde function '%s'" % vtilde)
    if S0 == 0.0 and vtilde == "power-law" and m is None:
        raise ValueError("the power-law v(k) takes the exponent m")
    modes, kamp = isotropic_kset(d, basis, k2, k2, 1.0)
    keep = kamp * kamp > k1 * k1
    modes, kamp = modes[keep], kamp[keep]
    if S0 != 0.0:
        return modes, np.ones(len(modes)), np.full(len(modes), float(S0))
    if vtilde == "flat":
        V = np.ones(len(modes))
    elif vtilde == "overlap":
        V = alpha(d, kamp / k2)
    else:
        V = (1.0 - kamp / k2) ** m
    return modes, np.ascontiguousarray(V, np.float64), None


class RepulsiveCCPotential:
    """RepulsiveCCPotential on the GPU: contact strength e0 and distance sigma, constraints (integer modes, weights V)
    and, for the S2 kernel, targets S0 (one per mode)."""

    def __init__(self, d, basis, modes, V, e0, sigma, S0=None):
        self.d, self.sigma = int(d), float(sigma)
        self._m = CCMulti(d, basis, [modes], [V], u0=1.0, e0=e0,
                          S0_per_species=None if S0 is None else [S0])

    def set_configuration(self, frac):
        frac = np.ascontiguousarray(frac, np.float64).reshape(-1, self.d)
        self._m.set_configuration(frac, np.zeros(len(frac), np.int32), np.full(len(frac), 0.5 * self.sigma))

    def energy_and_forces(self, forces=True):
        return self._m.energy_and_forces(forces)
