"""The variable-cell collective-coordinate potentials of the reference, evaluated at a given cell on the GPU.

Reference: potential/CCPotential_varBox.h (ShiftedCCPotential_varBoxable:32-213, ShiftedCCPotential_varBox:216-293,
ShiftedCCPotential_S2_varBox:300-386, ShiftedCCPotential_S2_varBox_noV0:389-470) and the weight / target catalogue of
potential/CCPotential_Kernels.h (K2, KM2, KM3, KM4, Lemniscate weights :18-188; K2, Kn, Klc, KM2, KMLog targets
:196-334; the named typedefs at :190-191 and :339-358).

For a cell with reciprocal basis b_e the constraints are every lattice point k = sum_e n_e b_e with |k|^2 < rK^2 in
the half space whose first non-zero index is positive (varBoxable::SetConfiguration :129-202), weighted by tildeV(k):
  plain form  E = sum_k tildeV(k) |rho(k)|^2 / V + N (N - 1) / (2 V) - (N / V) sum_k tildeV(k)     (:228-246)
  S2 form     E = sum_k tildeV(k) (|rho(k)|^2 / N - S0(k))^2                                       (:320-331)
  S2 noV0     E = sum_k tildeV(k) (|rho(k)|^2 / N - S0(k))^2 - sum_k tildeV(k) (S0(k) - 1)^2       (:409-424)
The wavevectors come from the library's lattice enumeration (the reference's reciprocal basis and |k|^2 rounding,
so the same points are in or out); the energies and forces run on the GPU through CCPotential (plain form) or its
S2 form. The cell derivatives (dBi, dki, EnergyDerivativeToBasisVectors) are not provided: cells are fixed here.

In the reference as shipped, the S2 classes never fill S0 or the noV0 shift: varBoxable::SetConfiguration sets
SameBasisVector before the S2 classes test it (:201 against :325 and :414), which leaves S0 empty for their Energy and
Force to read past. This module gives S0(k) and the shift the values those SetConfiguration bodies compute.
"""
import numpy as np

from .ccgpu import CCPotential, isotropic_kset


def _kl(k):
    return np.sqrt((k * k).sum(1))


def _km(p):
    def w(k, rK):
        t = 1.0 / _kl(k) - 1.0
        return t ** p
    return w


def _lemniscate(k, rK):
    """LemniscateVkTemplate (CCPotential_Kernels.h:140-188), d = 2: (|k|^4 / (rK^2 (kx^2 - ky^2)) - 1)^4 inside the
    lemniscate, 0 outside."""
    if k.shape[1] != 2:
        raise ValueError("the lemniscate weight is two-dimensional")
    k2 = (k * k).sum(1)
    x2my2 = k[:, 0] * k[:, 0] - k[:, 1] * k[:, 1]
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = k2 * k2 / (rK * rK) / x2my2
    inside = (ratio < 1) & (x2my2 > 0)
    return np.where(inside, (ratio - 1) ** 4, 0.0)


# tildeV(k), CCPotential_Kernels.h:18-188
WEIGHTS = {
    "K2": lambda k, rK: (1.0 - _kl(k)) ** 2,
    "KM2": _km(2),
    "KM3": _km(3),
    "KM4": _km(4),
    "Lemniscate": _lemniscate,
}

# S0(k), CCPotential_Kernels.h:196-334 (n: the exponent of Kn and Klc)
TARGETS = {
    "K2": lambda k, n: (k * k).sum(1),
    "Kn": lambda k, n: (k * k).sum(1) ** (0.5 * n),
    "Klc": lambda k, n: 0.5 * ((k * k).sum(1) ** (0.5 * n) + 1),
    "KM2": lambda k, n: (1.0 / _kl(k) - 1.0) ** 2,
    "KMLog": lambda k, n: -0.5 * np.log((k * k).sum(1)),
}

# The reference's named potentials (CCPotential_Kernels.h:190-191, 339-358): (weight, target, form)
NAMED = {
    "K2Potential": ("K2", None, "plain"),
    "KM3Potential": ("KM3", None, "plain"),
    "K2K2Potential": ("K2", "K2", "S2"),
    "K2K2Potential_noV0": ("K2", "K2", "S2_noV0"),
    "KM3K2Potential_noV0": ("KM3", "K2", "S2_noV0"),
    "KM2K2Potential": ("KM2", "K2", "S2"),
    "KM3K2Potential": ("KM3", "K2", "S2"),
    "KM4K2Potential": ("KM4", "K2", "S2"),
    "KM3KM2Potential": ("KM3", "KM2", "S2"),
    "KM3KMLogPotential": ("KM3", "KMLog", "S2"),
    "KM2KnPotential": ("KM2", "Kn", "S2"),
    "KM3KnPotential": ("KM3", "Kn", "S2"),
    "KM4KnPotential": ("KM4", "Kn", "S2"),
    "KM2KlcPotential": ("KM2", "Klc", "S2"),
    "KM3KlcPotential": ("KM3", "Klc", "S2"),
    "KM4KlcPotential": ("KM4", "Klc", "S2"),
}


def lattice_ks(d, basis, rK):
    """The constrained lattice points of a cell: integer modes (M x d) of the half-space points with |k|^2 < rK^2
    (the strict test of PeriodicCellList::IterateThroughNeighbors), ordered by (|k|^2, k_x)."""
    modes, kamp = isotropic_kset(d, basis, rK, rK)
    if d == 1:   # the 1D enumeration includes |k| = rK; IterateThroughNeighbors does not
        modes = modes[kamp * kamp < rK * rK]
    return modes


def cartesian(basis, modes):
    """k = sum_e n_e b_e with b = 2 pi inv(A)^T (A rows = basis vectors)."""
    basis = np.asarray(basis, np.float64)
    return np.asarray(modes, np.float64) @ (2 * np.pi * np.linalg.inv(basis).T)


def constraints(d, basis, N, weight, target=None, form="plain", rK=1.0, n=None):
    """(modes, V, S0 or None, shift) of a varBox potential at the cell `basis` with N particles."""
    if form not in ("plain", "S2", "S2_noV0"):
        raise ValueError("form must be 'plain', 'S2' or 'S2_noV0'")
    if (target is None) != (form == "plain"):
        raise ValueError("the S2 forms take a target S0(k); the plain form none")
    if target in ("Kn", "Klc") and n is None:
        raise ValueError("the Kn and Klc targets take the exponent n")
    basis = np.ascontiguousarray(basis, np.float64).reshape(d, d)
    modes = lattice_ks(d, basis, rK)
    k = cartesian(basis, modes)
    V = np.ascontiguousarray(WEIGHTS[weight](k, rK), np.float64)
    if form == "plain":
        vol = abs(float(np.linalg.det(basis)))
        return modes, V, None, N * (N - 1) / vol / 2.0 - N / vol * float(V.sum())
    S0 = np.ascontiguousarray(TARGETS[target](k, n), np.float64)
    shift = 0.0 if form == "S2" else -float(((S0 - 1) * (S0 - 1) * V).sum())
    return modes, V, S0, shift


class VarBoxPotential:
    """A named varBox potential of the reference (``NAMED``), or one assembled from ``weight`` / ``target`` / ``form``,
    bound to a cell and a configuration. Constraints are regenerated when the cell changes (and, for the plain form,
    the shift when N changes), as the reference's SetConfiguration does."""

    def __init__(self, name=None, d=3, rK=1.0, n=None, weight=None, target=None, form=None):
        if name is not None:
            weight, target, form = NAMED[name]
        self.name, self.d, self.rK, self.n = name, int(d), float(rK), n
        self.weight, self.target, self.form = weight, target, form or "plain"
        self._key = None
        self.pot = None
        self.modes = self.V = self.S0 = None
        self.shift = 0.0

    def set_configuration(self, basis, frac):
        basis = np.ascontiguousarray(basis, np.float64).reshape(self.d, self.d)
        frac = np.ascontiguousarray(frac, np.float64).reshape(-1, self.d)
        N = len(frac)
        key = (basis.tobytes(), N if self.form == "plain" else None)
        if key != self._key:
            self.modes, self.V, self.S0, self.shift = constraints(self.d, basis, N, self.weight, self.target,
                                                                  self.form, self.rK, self.n)
            if self.pot is not None:
                self.pot.close()
            self.pot = CCPotential(self.d, basis, self.modes, self.V, self.shift, S0=self.S0)
            self._key = key
        self.pot.set_configuration(frac)

    def _bound(self):
        if self.pot is None:
            raise RuntimeError("VarBoxPotential has no bound cell (closed, or set_configuration not called)")
        return self.pot

    def energy_and_forces(self, forces=True):
        return self._bound().energy_and_forces(forces=forces)

    def energy(self):
        return self._bound().energy()

    def minimize(self, frac, **kw):
        """Device L-BFGS over the positions at the bound cell (see CCPotential.minimize)."""
        return self._bound().minimize(frac, **kw)

    def close(self):
        if self.pot is not None:
            self.pot.close()
            self.pot = None
            self._key = None
