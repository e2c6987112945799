"""The C ABI library loads, exports every symbol include/cc_gpu.h declares, and fails loudly without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "cc_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cc_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(ccgpu):
    lib = ctypes.CDLL(ccgpu.library_path())
    names = _declared()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n


def test_no_cpu_path(ccgpu):
    if ccgpu.device_available():
        pytest.skip("a GPU is present")
    with pytest.raises(ccgpu.CCError) as e:
        ccgpu.CCPotential(2, np.eye(2), np.array([[1, 0]]), np.array([1.0]))
    assert e.value.code == -7


def test_argument_errors(ccgpu):
    lib = ccgpu.load_library()
    h = ctypes.c_void_p()
    b = np.eye(4)
    assert lib.cc_create(4, b.ctypes.data_as(ctypes.c_void_p), 0, None, None, 0.0, ctypes.byref(h)) == -1
    assert lib.cc_create(0, b.ctypes.data_as(ctypes.c_void_p), 0, None, None, 0.0, ctypes.byref(h)) == -1
    assert lib.cc_create(2, None, 0, None, None, 0.0, ctypes.byref(h)) == -1
    assert lib.cc_destroy(None) == 0
    E = ctypes.c_double()
    assert lib.cc_energy_grad(None, ctypes.byref(E), None, 0) == -1
    assert "null" in lib.cc_last_error().decode()
    assert lib.cc_set_independent_positions(None, 1) == -1
    assert lib.cc_energy_grad_many(None, 1, 1, None, ctypes.byref(E), None, 0) == -1


def test_nonlattice_k_rejected(ccgpu):
    lib = ccgpu.load_library()
    h = ctypes.c_void_p()
    b = np.array([[1.3, 0.0], [0.45, 0.9]])
    k = np.array([[1.37 * 2 * np.pi / 1.3, 0.0]])
    V = np.ones(1)
    rc = lib.cc_create_cartesian(2, b.ctypes.data_as(ctypes.c_void_p), 1, k.ctypes.data_as(ctypes.c_void_p),
                                 V.ctypes.data_as(ctypes.c_void_p), 0.0, ctypes.byref(h))
    assert rc == -5
