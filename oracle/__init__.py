"""ORACLE — test infrastructure only (tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg).

Two CPU checkers of the collective-coordinate path:
  * ``Ref``  — the reference's own ShiftedCCPotential / LuksanPLIS compiled from its sources (oracle/_ref/libccref.so,
    built by oracle/Makefile where the reference tree is present), with its S2, multi-configuration, varBox
    (``RefVarBox``), multi-species, RepulsiveCCPotential, IsotropicStructureFactor and MSPB code;
  * ``port`` — the plain-C restatement oracle/cc_oracle.c (oracle/_build/libccoracle.so), pinned to the reference by
    tests/test_oracle.py and the golden vectors in tests/golden/.
Nothing on the product path imports this package.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libccref.so")
PORT_LIB = os.path.join(HERE, "_build", "libccoracle.so")
# The reference's source tree, needed only to BUILD oracle/_ref (the built library then runs without it): the
# CC_REFERENCE_TREE environment variable, or the ref_tree argument of build().
REFERENCE_TREE = os.environ.get("CC_REFERENCE_TREE")

_vp = ctypes.c_void_p
_l = ctypes.c_long
_d = ctypes.c_double


def build(ref=True, ref_tree=None):
    """Build the port (always) and the reference oracle (when a reference tree is given, by ref_tree or
    CC_REFERENCE_TREE, and present)."""
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    tree = ref_tree or REFERENCE_TREE
    if ref and tree and os.path.isdir(tree):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={tree}"], check=True)


def _p(a):
    return a.ctypes.data_as(_vp) if a is not None else None


_REF = None
_PORT = None


def ref_available():
    return os.path.exists(REF_LIB)


def ref_lib():
    global _REF
    if _REF is None:
        lib = ctypes.CDLL(REF_LIB)
        lib.ccref_create.restype = _vp
        lib.ccref_create.argtypes = [ctypes.c_int, _vp, _l, _vp, _vp, _vp, _d, ctypes.c_int]
        lib.ccref_create_s2.restype = _vp
        lib.ccref_create_s2.argtypes = [ctypes.c_int, _vp, _l, _vp, _vp, _vp, _d, ctypes.c_int]
        lib.ccref_create_s2_multiconfig.restype = _vp
        lib.ccref_create_s2_multiconfig.argtypes = [ctypes.c_int, _vp, _l, _vp, _vp, _vp, _d, ctypes.c_int,
                                                    ctypes.c_int]
        lib.ccref_create_varbox.restype = _vp
        lib.ccref_create_varbox.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _d, _d, ctypes.c_int]
        lib.ccref_varbox_state.argtypes = [_vp, _vp, _vp, _vp]
        lib.ccref_constraints.argtypes = [_vp, _vp, _vp]
        lib.ccref_varbox_weights.argtypes = [_vp, _l, _vp, _vp, _vp]
        lib.ccref_destroy.argtypes = [_vp]
        lib.ccref_kcart.argtypes = [_vp, _vp]
        lib.ccref_volume.restype = _d
        lib.ccref_volume.argtypes = [_vp]
        lib.ccref_reciprocal.argtypes = [_vp, _vp]
        lib.ccref_set_positions.argtypes = [_vp, _l, _vp]
        lib.ccref_eval.argtypes = [_vp, ctypes.POINTER(_d), _vp, _vp, _vp]
        lib.ccref_force_one.argtypes = [_vp, _l, _vp]
        lib.ccref_cartesian.argtypes = [_vp, _vp]
        lib.ccref_structure_factor.argtypes = [_vp, _l, _vp, _vp]
        lib.ccref_minimize.restype = _d
        lib.ccref_minimize.argtypes = [_vp, _l, _vp, _d, _l, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_l)]
        lib.ccref_mc_trymove.restype = _d
        lib.ccref_mc_trymove.argtypes = [_vp, _vp, _vp, ctypes.c_int]
        lib.ccref_kset_cli.restype = _l
        lib.ccref_kset_cli.argtypes = [ctypes.c_int, _vp, _l, _d, ctypes.c_int, _l, _vp, _vp]
        lib.ccref_getks.restype = _l
        lib.ccref_getks.argtypes = [ctypes.c_int, _vp, _d, _d, _d, _d, _l, _vp]
        lib.ccref_multi_eval.restype = ctypes.c_int
        lib.ccref_multi_eval.argtypes = [ctypes.c_int, _vp, ctypes.c_int, _vp, _vp, _vp, _d, _d, _l, _vp, _vp, _vp,
                                         ctypes.POINTER(_d), _vp]
        lib.ccref_isotropic_sk.restype = _l
        lib.ccref_isotropic_sk.argtypes = [ctypes.c_int, _l, _vp, _vp, _vp, _d, _d, _d, _d, ctypes.c_int, _d, _l,
                                           _vp]
        _REF = lib
    return _REF


def port_lib():
    global _PORT
    if _PORT is None:
        if not os.path.exists(PORT_LIB):
            build(ref=False)
        lib = ctypes.CDLL(PORT_LIB)
        lib.cco_eval.restype = _d
        lib.cco_eval.argtypes = [ctypes.c_int, _vp, _l, _vp, _l, _vp, _vp, _d, _vp, _vp, _vp]
        lib.cco_sk.argtypes = [ctypes.c_int, _vp, _l, _vp, _l, _vp, _vp]
        lib.cco_volume.restype = _d
        lib.cco_volume.argtypes = [ctypes.c_int, _vp]
        _PORT = lib
    return _PORT


def lattice_k(basis, modes):
    """Cartesian k = sum_e n_e b_e with b = 2 pi inv(A)^T (A rows = basis vectors)."""
    basis = np.asarray(basis, np.float64)
    B = 2 * np.pi * np.linalg.inv(basis).T
    return np.asarray(modes, np.float64) @ B


class Ref:
    """The reference's ShiftedCCPotential (Direct backend) over a cell; modes or Cartesian k. With S0 (integer modes)
    the reference's ShiftedCCPotential_S2 instead (potential/CollectiveCoordinatePotential.h:1642-1749), and with nsub
    its ShiftedCCPotential_S2_MultiConfig (:1756-1870)."""

    def __init__(self, d, basis, V, modes=None, kcart=None, shift=0.0, nthreads=None, S0=None, nsub=None):
        self.lib = ref_lib()
        self.d = d
        self.basis = np.ascontiguousarray(basis, np.float64).reshape(d, d)
        V = np.ascontiguousarray(V, np.float64)
        self.M = len(V)
        m = np.ascontiguousarray(modes, np.int32) if modes is not None else None
        k = np.ascontiguousarray(kcart, np.float64) if kcart is not None else None
        nt = nthreads or os.cpu_count() or 1
        if nsub is not None:   # ShiftedCCPotential_S2_MultiConfig
            S0 = np.ascontiguousarray(S0, np.float64)
            self.h = self.lib.ccref_create_s2_multiconfig(d, _p(self.basis), self.M, _p(m), _p(V), _p(S0), shift,
                                                          int(nsub), nt)
        elif S0 is not None:
            S0 = np.ascontiguousarray(S0, np.float64)
            self.h = self.lib.ccref_create_s2(d, _p(self.basis), self.M, _p(m), _p(V), _p(S0), shift, nt)
        else:
            self.h = self.lib.ccref_create(d, _p(self.basis), self.M, _p(m), _p(k), _p(V), shift, nt)
        if not self.h:
            raise ValueError("ccref_create failed")
        self.N = 0

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ccref_destroy(self.h)
            self.h = None

    def kcart(self):
        out = np.zeros((max(self.M, 1), self.d))
        self.lib.ccref_kcart(self.h, _p(out))
        return out[: self.M]

    def volume(self):
        return self.lib.ccref_volume(self.h)

    def set_positions(self, frac):
        frac = np.ascontiguousarray(frac, np.float64).reshape(-1, self.d)
        self.N = len(frac)
        self.lib.ccref_set_positions(self.h, self.N, _p(frac))

    def eval(self, forces=True):
        E = _d()
        F = np.zeros((max(self.N, 1), self.d)) if forces else None
        re = np.zeros(max(self.M, 1))
        im = np.zeros(max(self.M, 1))
        self.lib.ccref_eval(self.h, ctypes.byref(E), _p(F), _p(re), _p(im))
        return E.value, (F[: self.N] if forces else None), re[: self.M], im[: self.M]

    def force_one(self, i):
        f = np.zeros(self.d)
        self.lib.ccref_force_one(self.h, i, _p(f))
        return f

    def structure_factor(self, kcart):
        kcart = np.ascontiguousarray(kcart, np.float64).reshape(-1, self.d)
        S = np.zeros(max(len(kcart), 1))
        self.lib.ccref_structure_factor(self.h, len(kcart), _p(kcart), _p(S))
        return S[: len(kcart)]

    def mc_try_move(self, s_prev, s_after, accept=False):
        a = np.ascontiguousarray(s_prev, np.float64)
        b = np.ascontiguousarray(s_after, np.float64)
        return self.lib.ccref_mc_trymove(self.h, _p(a), _p(b), 1 if accept else 0)

    def minimize(self, frac, emin=-1.0, maxeval=5000, history=40, fast=0):
        x = np.ascontiguousarray(frac, np.float64).reshape(-1, self.d).copy()
        ev = _l()
        E = self.lib.ccref_minimize(self.h, len(x), _p(x), emin, maxeval, history, fast, ctypes.byref(ev))
        return E, x, ev.value


VARBOX_KINDS = ["K2Potential", "KM3Potential", "K2K2Potential", "K2K2Potential_noV0", "KM3K2Potential_noV0",
                "KM2K2Potential", "KM3K2Potential", "KM4K2Potential", "KM3KM2Potential", "KM3KMLogPotential",
                "KM2KnPotential", "KM3KnPotential", "KM4KnPotential", "KM2KlcPotential", "KM3KlcPotential",
                "KM4KlcPotential"]


class RefVarBox(Ref):
    """One of the reference's named variable-cell potentials (potential/CCPotential_Kernels.h) at a fixed cell; its
    constraints and shift are generated by its own SetConfiguration when positions are set. eval() is for the plain
    kinds only: the S2 kinds leave S0 empty (state() reports its length), so their Energy would read past it."""

    def __init__(self, name, d, basis, rK=1.0, n=0.0, nthreads=None):
        self.lib = ref_lib()
        self.d = d
        self.basis = np.ascontiguousarray(basis, np.float64).reshape(d, d)
        nt = nthreads or os.cpu_count() or 1
        self.h = self.lib.ccref_create_varbox(VARBOX_KINDS.index(name), d, _p(self.basis), rK, n, nt)
        if not self.h:
            raise ValueError("ccref_create_varbox failed")
        self.M = 0
        self.N = 0

    def set_positions(self, frac):
        super().set_positions(frac)
        self.M = self.state()[0]

    def state(self):
        M, shift, nS0 = _l(), _d(), _l()
        self.lib.ccref_varbox_state(self.h, ctypes.byref(M), ctypes.byref(shift), ctypes.byref(nS0))
        return M.value, shift.value, nS0.value

    def constraints(self):
        M = self.state()[0]
        k = np.zeros((max(M, 1), self.d))
        V = np.zeros(max(M, 1))
        self.lib.ccref_constraints(self.h, _p(k), _p(V))
        return k[:M], V[:M]

    def weights(self, kcart):
        """The class's own tildeV(k) and S0(k) (NaN for the plain kinds) at Cartesian wavevectors."""
        kcart = np.ascontiguousarray(kcart, np.float64).reshape(-1, self.d)
        V = np.zeros(max(len(kcart), 1))
        S0 = np.zeros(max(len(kcart), 1))
        self.lib.ccref_varbox_weights(self.h, len(kcart), _p(kcart), _p(V), _p(S0))
        return V[:len(kcart)], S0[:len(kcart)]


def ref_kset(d, basis, N, chi, type_=0, cap=400000):
    lib = ref_lib()
    basis = np.ascontiguousarray(basis, np.float64).reshape(d, d)
    modes = np.zeros((cap, d), np.int32)
    V = np.zeros(cap)
    M = lib.ccref_kset_cli(d, _p(basis), N, chi, type_, cap, _p(modes), _p(V))
    if M < 0:
        raise ValueError("cap too small")
    return modes[:M].copy(), V[:M].copy()


def port_eval(d, basis, frac, kcart, V, shift=0.0):
    """The C restatement: (E, F, re, im)."""
    lib = port_lib()
    basis = np.ascontiguousarray(basis, np.float64).reshape(d, d)
    frac = np.ascontiguousarray(frac, np.float64).reshape(-1, d)
    kcart = np.ascontiguousarray(kcart, np.float64).reshape(-1, d)
    V = np.ascontiguousarray(V, np.float64)
    N, M = len(frac), len(V)
    F = np.zeros((max(N, 1), d))
    re = np.zeros(max(M, 1))
    im = np.zeros(max(M, 1))
    E = lib.cco_eval(d, _p(basis), N, _p(frac), M, _p(kcart), _p(V), shift, _p(F), _p(re), _p(im))
    return E, F[:N], re[:M], im[:M]


def port_sk(d, basis, frac, kcart):
    lib = port_lib()
    basis = np.ascontiguousarray(basis, np.float64).reshape(d, d)
    frac = np.ascontiguousarray(frac, np.float64).reshape(-1, d)
    kcart = np.ascontiguousarray(kcart, np.float64).reshape(-1, d)
    S = np.zeros(max(len(kcart), 1))
    lib.cco_sk(d, _p(basis), len(frac), _p(frac), len(kcart), _p(kcart), _p(S))
    return S[: len(kcart)]


def ref_getks(d, basis, circ, lin, p=1.0, kmin=0.0, cap=2000000):
    """GetKs of the reference (restated in oracle/sk_oracle.cpp): Cartesian wavevectors (K x d)."""
    basis = np.ascontiguousarray(basis, np.float64).reshape(d, d)
    out = np.zeros((cap, d))
    K = ref_lib().ccref_getks(d, _p(basis), circ, lin, p, kmin, cap, _p(out))
    if K < 0:
        raise ValueError("cap too small")
    return out[:K]


def ref_isotropic_sk(d, bases, fracs, circ, lin, kprec=0.01, p=1.0, option=0, kmin=0.0, cap=200000):
    """The reference's own IsotropicStructureFactor (pairstat/StructureFactor.cpp): rows (k, S, dk, dS)."""
    n = len(fracs)
    B = np.ascontiguousarray(np.asarray(bases, np.float64).reshape(n, d, d))
    arrs = [np.ascontiguousarray(f, np.float64).reshape(-1, d) for f in fracs]
    N = np.array([len(a) for a in arrs], dtype=np.int64)
    ptrs = (_vp * n)(*[a.ctypes.data_as(_vp) for a in arrs])
    out = np.zeros((cap, 4))
    R = ref_lib().ccref_isotropic_sk(d, n, _p(B), _p(N), ptrs, circ, lin, kprec, p, option, kmin, cap, _p(out))
    if R < 0:
        raise ValueError("cap too small")
    return out[:R]


def ref_multi_eval(d, basis, kcarts, Vs, u0, e0, frac, species, radii=None):
    """The reference's own MultiStealthyPotential: (E, F) with F Cartesian (N x d)."""
    basis = np.ascontiguousarray(basis, np.float64).reshape(d, d)
    S = len(Vs)
    M = np.array([len(v) for v in Vs], dtype=np.int64)
    ks = [np.ascontiguousarray(k, np.float64).reshape(-1, d) for k in kcarts]
    vs = [np.ascontiguousarray(v, np.float64) for v in Vs]
    kp = (_vp * S)(*[k.ctypes.data_as(_vp) for k in ks])
    vp = (_vp * S)(*[v.ctypes.data_as(_vp) for v in vs])
    frac = np.ascontiguousarray(frac, np.float64).reshape(-1, d)
    sp = np.ascontiguousarray(species, np.int32)
    rad = None if radii is None else np.ascontiguousarray(radii, np.float64)
    E = _d()
    F = np.zeros((max(len(frac), 1), d))
    rc = ref_lib().ccref_multi_eval(d, _p(basis), S, _p(M), kp, vp, u0, e0, len(frac), _p(frac), _p(sp),
                                    None if rad is None else _p(rad), ctypes.byref(E), _p(F))
    if rc != 0:
        raise ValueError("the reference's MultiStealthyPotential threw")
    return E.value, F[:len(frac)]


def ref_repulsive_eval(d, basis, kcart, V, e0, sigma, frac, S0=None, nthreads=None):
    """The reference's own RepulsiveCCPotential (plain, or S2 with targets S0): (E, F) with F Cartesian (N x d)."""
    lib = ref_lib()
    lib.ccref_repulsive_eval.argtypes = [ctypes.c_int, _vp, _l, _vp, _vp, _vp, _d, _d, _l, _vp, ctypes.c_int, _vp,
                                         _vp]
    basis = np.ascontiguousarray(basis, np.float64).reshape(d, d)
    kcart = np.ascontiguousarray(kcart, np.float64).reshape(-1, d)
    V = np.ascontiguousarray(V, np.float64)
    S0 = None if S0 is None else np.ascontiguousarray(S0, np.float64)
    frac = np.ascontiguousarray(frac, np.float64).reshape(-1, d)
    E = _d()
    F = np.zeros((max(len(frac), 1), d))
    rc = lib.ccref_repulsive_eval(d, _p(basis), len(V), _p(kcart), _p(V), _p(S0), e0, sigma, len(frac), _p(frac),
                                  nthreads or os.cpu_count() or 1, ctypes.byref(E), _p(F))
    if rc != 0:
        raise ValueError("the reference's RepulsiveCCPotential threw")
    return E.value, F[:len(frac)]


def _mspb_lib():
    lib = ref_lib()
    if not getattr(lib, "_mspb_set", False):
        c = ctypes.c_char_p
        lib.ccref_mspb_write.argtypes = [c, ctypes.c_int, _l, ctypes.c_ulonglong, _vp, _vp, _vp, _vp, _vp, _vp,
                                         ctypes.c_int]
        lib.ccref_mspb_read.argtypes = [c, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(_l),
                                        ctypes.POINTER(ctypes.c_ulonglong), _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int]
        lib.ccref_mspbpack_import.argtypes = [c, c, _vp, ctypes.c_int]
        lib.ccref_mspbpack_count.argtypes = [c, ctypes.POINTER(_l), _vp, ctypes.c_int]
        lib.ccref_mspbpack_export.argtypes = [c, _l, c, _vp, ctypes.c_int]
        lib._mspb_set = True
    return lib


class RefMSPBError(ValueError):
    """The reference's MSPB code threw (its message)."""


def _mspb_call(fn, *args):
    err = ctypes.create_string_buffer(512)
    if fn(*args, err, 512) != 0:
        raise RefMSPBError(err.value.decode())


def ref_mspb_write(path, basis, ids, species, rel, radii, species_count):
    """The reference's MSPBSnapshot::Write of one snapshot to `path`."""
    basis = np.ascontiguousarray(basis, np.float64)
    d = basis.shape[0]
    rel = np.ascontiguousarray(rel, np.float64).reshape(-1, d)
    ids = np.ascontiguousarray(ids, np.uint64)
    species = np.ascontiguousarray(species, np.uint32)
    radii = np.ascontiguousarray(radii, np.float64)
    _mspb_call(_mspb_lib().ccref_mspb_write, str(path).encode(), d, len(rel), int(species_count), _p(basis),
               _p(ids), _p(species), _p(rel), _p(radii))


def ref_mspb_read(path):
    """The reference's MSPBSnapshot::Read of one file: dict(basis, ids, species, rel, radii, species_count)."""
    lib = _mspb_lib()
    d, n, ns = ctypes.c_int(), _l(), ctypes.c_ulonglong()
    _mspb_call(lib.ccref_mspb_read, str(path).encode(), ctypes.byref(d), ctypes.byref(n), ctypes.byref(ns),
               None, None, None, None, None)
    D, N = d.value, n.value
    basis, ids = np.zeros((D, D)), np.zeros(N, np.uint64)
    species, rel, radii = np.zeros(N, np.uint32), np.zeros((N, D)), np.zeros(N)
    _mspb_call(lib.ccref_mspb_read, str(path).encode(), ctypes.byref(d), ctypes.byref(n), ctypes.byref(ns),
               _p(basis), _p(ids), _p(species), _p(rel), _p(radii))
    return dict(basis=basis, ids=ids, species=species, rel=rel, radii=radii, species_count=ns.value)


def ref_mspbpack_import(prefix, path):
    """MSPB_Pack(prefix).ImportFile(path) of the reference."""
    _mspb_call(_mspb_lib().ccref_mspbpack_import, str(prefix).encode(), str(path).encode())


def ref_mspbpack_count(prefix):
    """MSPB_Pack(prefix).NumConfig() of the reference."""
    n = _l()
    _mspb_call(_mspb_lib().ccref_mspbpack_count, str(prefix).encode(), ctypes.byref(n))
    return n.value


def ref_mspbpack_export(prefix, index, path):
    """MSPB_Pack(prefix).ExportFile(index, path) of the reference."""
    _mspb_call(_mspb_lib().ccref_mspbpack_export, str(prefix).encode(), int(index), str(path).encode())
