"""ctypes binding of libccgpu.so (include/cc_gpu.h).

``CCPotential`` mirrors the reference's ShiftedCCPotential (potential/CollectiveCoordinatePotential.h): a constraint
set {k, V(k)} plus Shift, bound to one configuration at a time (SetConfiguration), with Energy / AllForce / Force /
GetRho and the structure optimiser's objective. Errors raise ``CCError`` carrying the ABI status code, as the
reference's setters raise std::invalid_argument / std::logic_error.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

PREC_FP64 = 0
PREC_MIXED = 1

_STATUS = {0: "CC_OK", -1: "CC_ERR_ARG", -2: "CC_ERR_OOM", -3: "CC_ERR_CUDA", -4: "CC_ERR_TIMEOUT",
           -5: "CC_ERR_NONLATTICE", -6: "CC_ERR_STATE", -7: "CC_ERR_NOGPU", -8: "CC_ERR_NAN"}


class CCError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_STATUS.get(code, code)}: {msg}")
        self.code = code


class NotANumberFound(CCError):
    """The objective's first variable is NaN (the reference's NotANumberFound, StructureOptimization.h:47)."""


def library_path():
    return os.path.join(_HERE, "libccgpu.so")


_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_d = ctypes.c_double
_i = ctypes.c_int

class LbfgsOpts(ctypes.Structure):
    _fields_ = [("history", ctypes.c_int), ("max_evals", ctypes.c_int64), ("stopval", ctypes.c_double),
                ("gtol", ctypes.c_double), ("ftol", ctypes.c_double), ("precision", ctypes.c_int),
                ("switch_energy_per_particle", ctypes.c_double), ("iters_per_check", ctypes.c_int)]


class LbfgsResult(ctypes.Structure):
    _fields_ = [("E", ctypes.c_double), ("evals", ctypes.c_int64), ("iters", ctypes.c_int64),
                ("status", ctypes.c_int)]


class ServeRequest(ctypes.Structure):
    _fields_ = [("d", ctypes.c_int), ("N", ctypes.c_int64), ("chi", ctypes.c_double), ("vtype", ctypes.c_int),
                ("frac0", ctypes.c_void_p), ("arrival_s", ctypes.c_double), ("max_evals", ctypes.c_int64),
                ("frac_out", ctypes.c_void_p)]


class ServeResult(ctypes.Structure):
    _fields_ = [("E", ctypes.c_double), ("evals", ctypes.c_int64), ("status", ctypes.c_int),
                ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double)]


class ServeOpts(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_size_t), ("max_slots", ctypes.c_int), ("iters_per_round", ctypes.c_int),
                ("history", ctypes.c_int), ("max_bypass_s", ctypes.c_double)]


PREC_SCHEDULE = 2
PATH_SPLIT, PATH_NUFFT, PATH_AUTO = 0, 2, 3
STOPVAL_GROUND_STATE = -1.0

_SIGS = {
    "cc_last_error": (ctypes.c_char_p, []),
    "cc_device_available": (_i, []),
    "cc_create": (_i, [_i, _vp, _i64, _vp, _vp, _d, ctypes.POINTER(_vp)]),
    "cc_create_cartesian": (_i, [_i, _vp, _i64, _vp, _vp, _d, ctypes.POINTER(_vp)]),
    "cc_create_s2": (_i, [_i, _vp, _i64, _vp, _vp, _vp, _d, ctypes.POINTER(_vp)]),
    "cc_create_s2_multiconfig": (_i, [_i, _vp, _i64, _vp, _vp, _vp, _d, _i, ctypes.POINTER(_vp)]),
    "cc_destroy": (_i, [_vp]),
    "cc_info": (_i, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i), ctypes.POINTER(_d), _vp]),
    "cc_set_rho_offset": (_i, [_vp, _d]),
    "cc_set_positions": (_i, [_vp, _i64, _vp]),
    "cc_energy_grad": (_i, [_vp, ctypes.POINTER(_d), _vp, _i]),
    "cc_rho": (_i, [_vp, _vp, _vp, _i]),
    "cc_force_one": (_i, [_vp, _i64, _vp]),
    "cc_structure_factor": (_i, [_vp, _i64, _vp, _vp, _i]),
    "cc_objective": (_i, [_vp, _i64, _vp, _d, ctypes.POINTER(_d), _vp, _i]),
    "cc_energy_grad_device": (_i, [_vp, _i64, _vp, _vp, _vp, _vp, _i, _vp]),
    "cc_energy_grad_many": (_i, [_vp, _i64, _i64, _vp, _vp, _vp, _i]),
    "cc_kset_stealthy": (_i, [_i, _vp, _i64, _d, _i, _i64, _vp, _vp, ctypes.POINTER(_i64)]),
    "cc_kset_isotropic": (_i, [_i, _vp, _d, _d, _d, _d, _i64, _vp, _vp, ctypes.POINTER(_i64)]),
    "cc_multi_create": (_i, [_i, _vp, _i, _vp, _vp, _vp, _d, _d, ctypes.POINTER(_vp)]),
    "cc_multi_create_s2": (_i, [_i, _vp, _i, _vp, _vp, _vp, _vp, _d, _d, ctypes.POINTER(_vp)]),
    "cc_multi_set_configuration": (_i, [_vp, _i64, _vp, _vp, _vp]),
    "cc_multi_energy_grad": (_i, [_vp, ctypes.POINTER(_d), _vp]),
    "cc_multi_destroy": (_i, [_vp]),
    "cc_isotropic_structure_factor": (_i, [_i, _i64, _vp, _vp, _vp, _d, _d, _d, _d, _i, _d, _vp, _i64,
                                           ctypes.POINTER(_i64)]),
    "cc_set_timing": (_i, [_vp, _i]),
    "cc_set_independent_positions": (_i, [_vp, _i]),
    "cc_get_timing": (_i, [_vp, ctypes.POINTER(_d), ctypes.POINTER(_d), ctypes.POINTER(_d), ctypes.POINTER(_i64)]),
    "cc_plan_info": (_i, [_vp, _i64, ctypes.POINTER(_i), ctypes.POINTER(_i64), ctypes.POINTER(_i),
                          ctypes.POINTER(_i)]),
    "cc_probe_fma_peak": (_i, [_i, ctypes.POINTER(_d)]),
    "cc_lbfgs_defaults": (_i, [ctypes.POINTER(LbfgsOpts)]),
    "cc_minimize": (_i, [_vp, _i64, _vp, ctypes.POINTER(LbfgsOpts), ctypes.POINTER(LbfgsResult)]),
    "cc_batch_create": (_i, [_i, ctypes.POINTER(_vp), ctypes.POINTER(_i64), ctypes.POINTER(_vp)]),
    "cc_batch_destroy": (_i, [_vp]),
    "cc_batch_set_positions": (_i, [_vp, ctypes.POINTER(_vp)]),
    "cc_batch_energy_grad": (_i, [_vp, _vp, ctypes.POINTER(_vp), _i]),
    "cc_batch_eval_device": (_i, [_vp, _i, _vp]),
    "cc_batch_autotune": (_i, [_vp, _i, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "cc_batch_set_wait_test": (_i, [_vp, ctypes.c_uint, _i]),
    "cc_batch_minimize": (_i, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(LbfgsOpts), ctypes.POINTER(LbfgsResult)]),
    "cc_serve": (_i, [ctypes.POINTER(ServeRequest), _i, ctypes.POINTER(ServeOpts), ctypes.POINTER(ServeResult),
                      ctypes.POINTER(_d)]),
    "cc_serve_last_error": (ctypes.c_char_p, []),
    "cc_mc_try_move": (_i, [_vp, _vp, _vp, ctypes.POINTER(_d)]),
    "cc_mc_accept_move": (_i, [_vp]),
    "cc_set_path": (_i, [_vp, _i]),
    "cc_eval_path": (_i, [_vp, _i64, _i, ctypes.POINTER(_i)]),
    "cc_check_device_error": (_i, [_vp]),
    "cc_energy_noalloc": (_i, [_i, _vp, _i64, _vp, _vp, _d, _i64, _vp, _vp, _vp, _vp]),
    "cc_noalloc_last_error": (ctypes.c_char_p, []),
}


def load_library():
    """Load libccgpu.so (building it first if it is missing and nvcc is present). Raises if it cannot be loaded."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path):
        from . import build
        build.build()
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def _check(rc):
    if rc != 0:
        raise (NotANumberFound if rc == -8 else CCError)(rc, load_library().cc_last_error().decode())


def _ptr(a):
    # the address as a plain int (every entry point has c_void_p argtypes): a quarter of data_as's cost per call
    return a.ctypes.data if a is not None else None


def device_available():
    return bool(load_library().cc_device_available())


def stealthy_kset(d, basis, N, chi, type_=0):
    """The reference CLI's stealthy k-set (GeneratePotential Type 0..3): (modes int32 M x d, V float64 M)."""
    lib = load_library()
    basis = np.ascontiguousarray(basis, dtype=np.float64).reshape(d, d)
    M = _i64(0)
    rc = lib.cc_kset_stealthy(d, _ptr(basis), N, chi, type_, 0, None, None, ctypes.byref(M))
    if rc not in (0, -1):
        _check(rc)
    modes = np.zeros((max(M.value, 1), d), np.int32)
    V = np.zeros(max(M.value, 1))
    _check(lib.cc_kset_stealthy(d, _ptr(basis), N, chi, type_, M.value, _ptr(modes), _ptr(V), ctypes.byref(M)))
    return modes[:M.value], V[:M.value]


def isotropic_kset(d, basis, circular_kmax, linear_kmax, sample_probability=1.0, circular_kmin=0.0):
    """The wavevectors of the reference's GetKs for a cell: (modes int32 K x d, |k| float64 K). Host only."""
    lib = load_library()
    basis = np.ascontiguousarray(basis, dtype=np.float64).reshape(d, d)
    K = _i64(0)
    args = (d, _ptr(basis), circular_kmax, linear_kmax, sample_probability, circular_kmin)
    rc = lib.cc_kset_isotropic(*args, 0, None, None, ctypes.byref(K))
    if rc not in (0, -1) or (rc == -1 and K.value == 0):
        _check(rc)
    modes = np.zeros((max(K.value, 1), d), np.int32)
    kamp = np.zeros(max(K.value, 1))
    _check(lib.cc_kset_isotropic(*args, K.value, _ptr(modes), _ptr(kamp), ctypes.byref(K)))
    return modes[:K.value], kamp[:K.value]


def isotropic_structure_factor(d, bases, fracs, circular_kmax, linear_kmax, k_precision=0.01, sample_probability=1.0,
                               option=0, circular_kmin=0.0):
    """IsotropicStructureFactor over configurations (bases[j]: d x d rows a_i; fracs[j]: N_j x d fractional).
    Returns an (R, 4) array of rows (k, S, dk, dS) as the reference's results."""
    lib = load_library()
    n = len(fracs)
    B = np.ascontiguousarray(np.asarray(bases, dtype=np.float64).reshape(n, d, d))
    arrs = [np.ascontiguousarray(f, dtype=np.float64).reshape(-1, d) for f in fracs]
    N = np.array([len(a) for a in arrs], dtype=np.int64)
    ptrs = (_vp * n)(*[a.ctypes.data_as(_vp) for a in arrs])
    cnt = _i64(0)
    args = (d, n, _ptr(B), _ptr(N), ptrs, circular_kmax, linear_kmax, k_precision, sample_probability, option,
            circular_kmin)
    # rows: at most one per bin (options 0, 1) or one per wavevector of the first cell (option 2)
    if option == 2:
        cap = len(isotropic_kset(d, B[0], circular_kmax, linear_kmax, sample_probability, circular_kmin)[1])
    else:
        kp = k_precision if k_precision > 0 else float(np.linalg.norm(2 * np.pi * np.linalg.inv(B[0]).T[0]))
        cap = int(np.floor(linear_kmax / kp)) + 1 if linear_kmax > 0 else 0
    out = np.zeros((max(cap, 1), 4))
    _check(lib.cc_isotropic_structure_factor(*args, _ptr(out), cap, ctypes.byref(cnt)))
    return out[:cnt.value]


class CCMulti:
    """MultiStealthyPotential: species with their own constraint sets (integer modes + weights) over subsets of the
    particles, plus the soft-core contact repulsion of strength e0; u0 scales the collective-coordinate part. With
    ``S0_per_species`` (an array of targets, or None, per species) a species' collective-coordinate part is the S2
    form."""

    def __init__(self, d, basis, modes_per_species, V_per_species, u0=1.0, e0=1.0, S0_per_species=None):
        self._lib = load_library()
        self.d = d
        basis = np.ascontiguousarray(basis, dtype=np.float64).reshape(d, d)
        self._modes = [np.ascontiguousarray(m, dtype=np.int32).reshape(-1, d) for m in modes_per_species]
        self._V = [np.ascontiguousarray(v, dtype=np.float64) for v in V_per_species]
        S = len(self._V)
        M = np.array([len(v) for v in self._V], dtype=np.int64)
        mp = (_vp * S)(*[m.ctypes.data_as(_vp) for m in self._modes])
        vp = (_vp * S)(*[v.ctypes.data_as(_vp) for v in self._V])
        h = _vp()
        if S0_per_species is None:
            _check(self._lib.cc_multi_create(d, _ptr(basis), S, _ptr(M), mp, vp, u0, e0, ctypes.byref(h)))
        else:
            self._S0 = [None if t is None else np.ascontiguousarray(t, dtype=np.float64) for t in S0_per_species]
            if len(self._S0) != S or any(t is not None and len(t) != len(v) for t, v in zip(self._S0, self._V)):
                raise ValueError("one S0 list (or None) per species, one target per mode")
            sp = (_vp * S)(*[None if t is None else t.ctypes.data_as(_vp) for t in self._S0])
            _check(self._lib.cc_multi_create_s2(d, _ptr(basis), S, _ptr(M), mp, vp, sp, u0, e0, ctypes.byref(h)))
        self._h = h
        self.N = None
        self.basis = basis
        self.nspecies = S

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.cc_multi_destroy(self._h)
            self._h = None

    def set_configuration(self, frac, species, radii=None):
        frac = np.ascontiguousarray(frac, dtype=np.float64).reshape(-1, self.d)
        sp = np.ascontiguousarray(species, dtype=np.int32)
        rad = None if radii is None else np.ascontiguousarray(radii, dtype=np.float64)
        _check(self._lib.cc_multi_set_configuration(self._h, len(frac), _ptr(frac), _ptr(sp),
                                                    None if rad is None else _ptr(rad)))
        self.N = len(frac)

    def set_snapshot(self, snapshot):
        """Bind an MSPB snapshot (modules_b200.mspb): its relative coordinates, species labels and radii. The
        snapshot's cell must be the potential's (bitwise) and its labels must name the potential's species."""
        if snapshot.d != self.d or not np.array_equal(snapshot.basis, self.basis):
            raise ValueError("the snapshot's cell is not the potential's")
        if snapshot.N and int(snapshot.species.max()) >= self.nspecies:
            raise ValueError("the snapshot has species labels beyond the potential's species")
        self.set_configuration(snapshot.rel, snapshot.species.astype(np.int32), snapshot.radii)

    def energy_and_forces(self, forces=True):
        E = _d()
        F = np.empty((max(self.N or 0, 1), self.d)) if forces else None
        _check(self._lib.cc_multi_energy_grad(self._h, ctypes.byref(E), _ptr(F) if forces else None))
        return (E.value, F[: self.N]) if forces else (E.value, None)


def probe_fma_peak(precision=PREC_FP64):
    """Measured FMA throughput of the device in TFLOP/s (FP64 or FP32 chains)."""
    t = _d()
    _check(load_library().cc_probe_fma_peak(precision, ctypes.byref(t)))
    return t.value


class CCPotential:
    """GPU ShiftedCCPotential over a cell ``basis`` (rows a_i) with integer ``modes`` (k = sum_e n_e b_e).

    With ``S0`` (one target per mode, integer modes) it is the S2 form, the reference's ShiftedCCPotential_S2
    (potential/CollectiveCoordinatePotential.h:1642-1749): E = sum_k V(k) (|rho(k)|^2 / N - S0(k))^2 + shift. With
    ``nsub`` > 1 as well, ShiftedCCPotential_S2_MultiConfig (:1756-1870): the N particles are nsub consecutive
    sub-configurations and S(k) is their mean."""

    def __init__(self, d, basis, modes=None, V=None, shift=0.0, kcart=None, S0=None, nsub=1):
        self._lib = load_library()
        self.d = int(d)
        self.basis = np.ascontiguousarray(basis, dtype=np.float64).reshape(self.d, self.d)
        h = _vp()
        if kcart is not None and S0 is not None:
            raise ValueError("the S2 form takes integer modes")
        if nsub != 1 and S0 is None:
            raise ValueError("sub-configurations belong to the S2 form")
        if kcart is not None:
            kc = np.ascontiguousarray(kcart, dtype=np.float64).reshape(-1, self.d)
            V = np.ascontiguousarray(V, dtype=np.float64).reshape(-1)
            _check(self._lib.cc_create_cartesian(self.d, _ptr(self.basis), len(V), _ptr(kc), _ptr(V), shift,
                                                 ctypes.byref(h)))
        else:
            modes = np.ascontiguousarray(modes, dtype=np.int32).reshape(-1, self.d)
            V = np.ascontiguousarray(V, dtype=np.float64).reshape(-1)
            if len(V) != len(modes):
                raise ValueError("modes and V differ in length")
            if S0 is not None:
                S0 = np.ascontiguousarray(S0, dtype=np.float64).reshape(-1)
                if len(S0) != len(V):
                    raise ValueError("modes and S0 differ in length")
                _check(self._lib.cc_create_s2_multiconfig(self.d, _ptr(self.basis), len(V), _ptr(modes), _ptr(V),
                                                          _ptr(S0), shift, int(nsub), ctypes.byref(h)))
            else:
                _check(self._lib.cc_create(self.d, _ptr(self.basis), len(V), _ptr(modes), _ptr(V), shift,
                                           ctypes.byref(h)))
        self._h = h
        self.M = len(V)
        self.N = None

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def info(self):
        M, d, vol = _i64(), _i(), _d()
        modes = np.zeros((max(self.M, 1), self.d), np.int32)
        _check(self._lib.cc_info(self._h, ctypes.byref(M), ctypes.byref(d), ctypes.byref(vol), _ptr(modes)))
        return modes[:M.value], vol.value

    def set_rho_offset(self, off):
        _check(self._lib.cc_set_rho_offset(self._h, float(off)))

    def set_configuration(self, frac):
        frac = np.ascontiguousarray(frac, dtype=np.float64).reshape(-1, self.d)
        _check(self._lib.cc_set_positions(self._h, len(frac), _ptr(frac)))
        self.N = len(frac)

    SetConfiguration = set_configuration

    def energy_and_forces(self, precision=PREC_FP64, forces=True):
        E = _d()
        F = np.empty((max(self.N or 0, 1), self.d)) if forces else None
        _check(self._lib.cc_energy_grad(self._h, ctypes.byref(E), _ptr(F) if forces else None, precision))
        return (E.value, F[: self.N]) if forces else (E.value, None)

    def energy(self, precision=PREC_FP64):
        return self.energy_and_forces(precision, forces=False)[0]

    Energy = energy

    def all_force(self, precision=PREC_FP64):
        return self.energy_and_forces(precision)[1]

    AllForce = all_force

    def force(self, i):
        f = np.zeros(self.d)
        _check(self._lib.cc_force_one(self._h, int(i), _ptr(f)))
        return f

    Force = force

    def rho(self, precision=PREC_FP64):
        re = np.zeros(max(self.M, 1))
        im = np.zeros(max(self.M, 1))
        _check(self._lib.cc_rho(self._h, _ptr(re), _ptr(im), precision))
        return re[: self.M], im[: self.M]

    GetRho = rho

    def structure_factor(self, modes, precision=PREC_FP64):
        modes = np.ascontiguousarray(modes, dtype=np.int32).reshape(-1, self.d)
        S = np.zeros(max(len(modes), 1))
        _check(self._lib.cc_structure_factor(self._h, len(modes), _ptr(modes), _ptr(S), precision))
        return S[: len(modes)]

    def objective(self, x, rescale, grad=True, precision=PREC_FP64):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        n = len(x) // self.d
        f = _d()
        g = np.zeros(max(len(x), 1)) if grad else None
        _check(self._lib.cc_objective(self._h, n, _ptr(x), rescale, ctypes.byref(f), _ptr(g) if grad else None,
                                      precision))
        self.N = n
        return (f.value, g[: len(x)]) if grad else f.value

    def minimize(self, frac, stopval=None, history=40, max_evals=100000, precision=PREC_FP64, gtol=0.0,
                 ftol=1e-15, switch_energy_per_particle=1e-12, iters_per_check=32):
        """Device-resident L-BFGS from the fractional start `frac`; returns (frac, E, evals, iters, status)."""
        o = LbfgsOpts()
        _check(self._lib.cc_lbfgs_defaults(ctypes.byref(o)))
        o.history, o.max_evals, o.precision = history, max_evals, precision
        o.gtol, o.ftol, o.switch_energy_per_particle, o.iters_per_check = gtol, ftol, switch_energy_per_particle, \
            iters_per_check
        if stopval is not None:
            o.stopval = stopval
        x = np.ascontiguousarray(frac, dtype=np.float64).reshape(-1, self.d).copy()
        r = LbfgsResult()
        _check(self._lib.cc_minimize(self._h, len(x), _ptr(x), ctypes.byref(o), ctypes.byref(r)))
        self.N = len(x)
        return x, r.E, r.evals, r.iters, r.status

    def try_move(self, s_prev, s_after):
        """Energy change of moving one particle from s_prev to s_after (fractional), as ForMC::TryMove."""
        a = np.ascontiguousarray(s_prev, dtype=np.float64).reshape(self.d)
        b = np.ascontiguousarray(s_after, dtype=np.float64).reshape(self.d)
        dE = _d()
        _check(self._lib.cc_mc_try_move(self._h, _ptr(a), _ptr(b), ctypes.byref(dE)))
        return dE.value

    TryMove = try_move

    def accept_move(self):
        _check(self._lib.cc_mc_accept_move(self._h))

    AcceptMove = accept_move

    def set_path(self, path):
        """PATH_AUTO (default): PATH_NUFFT where it is estimated faster, else PATH_SPLIT; PATH_SPLIT: the three-kernel
        direct path; PATH_NUFFT: non-uniform FFTs (FP64)."""
        _check(self._lib.cc_set_path(self._h, int(path)))

    def eval_path(self, N, precision=PREC_FP64):
        """The path an evaluation of N particles takes: "split" or "nufft"."""
        p = _i()
        _check(self._lib.cc_eval_path(self._h, int(N), precision, ctypes.byref(p)))
        return {PATH_SPLIT: "split", PATH_NUFFT: "nufft"}[p.value]

    def check_device_error(self):
        _check(self._lib.cc_check_device_error(self._h))

    def set_independent_positions(self, on=True):
        """Promise that positions given to energy_grad_device were complete before the kernel enqueued just before
        each call and that nothing in flight writes them (a pool of resident configurations): the rho kernel then
        overlaps its phase sums with the previous kernel's tail. Results are bitwise those of the default (off)."""
        _check(self._lib.cc_set_independent_positions(self._h, 1 if on else 0))

    def set_timing(self, on):
        _check(self._lib.cc_set_timing(self._h, 1 if on else 0))

    def get_timing(self):
        """(rho kernel ms, reduce kernel ms, force kernel ms, evaluations) summed since set_timing(True)."""
        r, q, f, n = _d(), _d(), _d(), _i64()
        _check(self._lib.cc_get_timing(self._h, ctypes.byref(r), ctypes.byref(q), ctypes.byref(f), ctypes.byref(n)))
        return r.value, q.value, f.value, n.value

    def plan_info(self, N):
        L, nseg, ns, nk = _i(), _i64(), _i(), _i()
        _check(self._lib.cc_plan_info(self._h, int(N), ctypes.byref(L), ctypes.byref(nseg), ctypes.byref(ns),
                                      ctypes.byref(nk)))
        return dict(L=L.value, nseg=nseg.value, nsplit=ns.value, nksplit=nk.value)

    def energy_grad_many(self, frac, E=None, F=None, precision=PREC_FP64, forces=True):
        """Energies and forces of many configurations from host memory in one call: frac is (P, N, d). E (P,) and F
        (P, N, d) are filled when given (pass arrays in pinned memory, e.g. numpy views of pinned torch tensors, for
        copies that overlap the evaluations), else allocated. Bitwise the results of P set_configuration +
        energy_and_forces calls. Returns (E, F)."""
        if frac.dtype != np.float64 or not frac.flags.c_contiguous:
            frac = np.ascontiguousarray(frac, dtype=np.float64)
        P, N = frac.shape[0], frac.shape[1]
        if E is None:
            E = np.empty(P)
        if forces and F is None:
            F = np.empty((P, N, self.d))
        for a, n in ((E, P), (F if forces else None, P * N * self.d)):
            if a is not None and (a.dtype != np.float64 or not a.flags.c_contiguous or a.size != n):
                raise ValueError("E must be a contiguous float64 array of P values and F of P x N x d")
        _check(self._lib.cc_energy_grad_many(self._h, P, N, _ptr(frac), _ptr(E), _ptr(F) if forces else None,
                                             precision))
        return E, (F if forces else None)

    def energy_grad_device(self, N, d_frac, d_E, d_F=None, d_gfrac=None, precision=PREC_FP64, stream=None):
        """Enqueue one evaluation on device pointers (ints); no synchronisation."""
        _check(self._lib.cc_energy_grad_device(self._h, int(N), _vp(d_frac), _vp(d_E), _vp(d_F) if d_F else None,
                                               _vp(d_gfrac) if d_gfrac else None, precision,
                                               _vp(stream) if stream else None))


class CCBatch:
    """Many independent configurations evaluated (and minimised) together: per dimension, one persistent launch of
    each multi-instance kernel (rho, reduce, force), the dimensions on parallel streams."""

    def __init__(self, pots, N):
        self._lib = load_library()
        self.pots = list(pots)
        self.N = [int(n) for n in N]
        hs = (_vp * len(self.pots))(*[p.handle for p in self.pots])
        ns = (_i64 * len(self.N))(*self.N)
        b = _vp()
        _check(self._lib.cc_batch_create(len(self.pots), hs, ns, ctypes.byref(b)))
        self._b = b

    def close(self):
        if getattr(self, "_b", None):
            self._lib.cc_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._b

    def _arrays(self, fracs):
        arrs = [np.ascontiguousarray(f, dtype=np.float64).reshape(n, p.d).copy()
                for f, n, p in zip(fracs, self.N, self.pots)]
        return arrs, (_vp * len(arrs))(*[a.ctypes.data_as(_vp) for a in arrs])

    def set_positions(self, fracs):
        arrs, ptrs = self._arrays(fracs)
        _check(self._lib.cc_batch_set_positions(self._b, ptrs))

    def energy_and_forces(self, precision=PREC_FP64, forces=True):
        E = np.zeros(len(self.pots))
        F = [np.zeros((n, p.d)) for n, p in zip(self.N, self.pots)]
        fp = (_vp * len(F))(*[f.ctypes.data_as(_vp) for f in F]) if forces else None
        _check(self._lib.cc_batch_energy_grad(self._b, E.ctypes.data_as(_vp), fp, precision))
        return (E, F) if forces else (E, None)

    def eval_device(self, precision=PREC_FP64, stream=None):
        _check(self._lib.cc_batch_eval_device(self._b, precision, _vp(stream) if stream else None))

    def autotune(self, reps=3):
        """Time every candidate tile shape on the bound positions and keep the fastest: (per_split, segs)."""
        ps, sg = _i(), _i()
        _check(self._lib.cc_batch_autotune(self._b, reps, ctypes.byref(ps), ctypes.byref(sg)))
        return ps.value, sg.value

    def set_wait_test(self, polls=0, phantom=0):
        """Test hook of the fused batch kernel's bounded waits (include/cc_gpu.h cc_batch_set_wait_test)."""
        _check(self._lib.cc_batch_set_wait_test(self._b, int(polls), int(phantom)))

    def minimize(self, fracs, stopval=STOPVAL_GROUND_STATE, history=40, max_evals=100000, precision=PREC_FP64,
                 gtol=0.0, ftol=1e-15, switch_energy_per_particle=1e-12, iters_per_check=32):
        """Minimise every instance from fracs[i]; returns (list of frac, E array, evals, iters, status arrays)."""
        self.set_positions(fracs)
        arrs, ptrs = self._arrays(fracs)
        o = LbfgsOpts()
        _check(self._lib.cc_lbfgs_defaults(ctypes.byref(o)))
        o.history, o.max_evals, o.precision, o.stopval = history, max_evals, precision, stopval
        o.gtol, o.ftol, o.switch_energy_per_particle, o.iters_per_check = gtol, ftol, switch_energy_per_particle, \
            iters_per_check
        res = (LbfgsResult * len(arrs))()
        _check(self._lib.cc_batch_minimize(self._b, ptrs, ctypes.byref(o), res))
        return (arrs, np.array([r.E for r in res]), np.array([r.evals for r in res]),
                np.array([r.iters for r in res]), np.array([r.status for r in res]))


def serve(requests, hbm_budget=16 << 30, max_slots=256, iters_per_round=16, history=40, max_bypass_s=1.0,
          positions=False):
    """Run the continuous-batching ground-state server on `requests`, a list of dicts with keys d, N, chi, vtype,
    frac0 (N x d array), arrival_s. Returns (list of result dicts, wall seconds); with positions=True each result
    also holds "frac", the final positions. A request the server cannot serve comes back with a negative status (the
    CC_ERR_* code: -1 invalid, -2 larger than the budget or out of memory) and E = NaN; the others are served."""
    lib = load_library()
    keep, finals = [], []
    reqs = (ServeRequest * len(requests))()
    for i, r in enumerate(requests):
        f = np.ascontiguousarray(r["frac0"], dtype=np.float64).reshape(int(r["N"]), int(r["d"]))
        keep.append(f)
        fo = np.full_like(f, np.nan) if positions else None
        finals.append(fo)
        reqs[i] = ServeRequest(int(r["d"]), int(r["N"]), float(r["chi"]), int(r.get("vtype", 0)),
                               f.ctypes.data_as(_vp), float(r.get("arrival_s", 0.0)), int(r.get("max_evals", 0)),
                               fo.ctypes.data_as(_vp) if positions else None)
    opts = ServeOpts(hbm_budget, max_slots, iters_per_round, history, max_bypass_s)
    res = (ServeResult * len(requests))()
    wall = _d()
    rc = lib.cc_serve(reqs, len(requests), ctypes.byref(opts), res, ctypes.byref(wall))
    if rc != 0:
        raise CCError(rc, lib.cc_serve_last_error().decode())
    out = [dict(E=x.E, evals=x.evals, status=x.status, t_admit=x.t_admit, t_done=x.t_done) for x in res]
    if positions:
        for o, fo in zip(out, finals):
            o["frac"] = fo
    return out, wall.value
