"""cc_energy_noalloc, the allocation-free entry point, against the regular entry points.

It exists for callers that cannot allocate GPU memory: processes whose memory manager owns all device memory, and
loops that must not pay for cudaMalloc, which can synchronise the device. The test calls it through the C ABI with
caller-owned device buffers (torch tensors) twice in a row (the second call must not see stale scratch contents)
and compares E and rho with cc_energy_grad / cc_rho on the same inputs, at the FP64 path's tolerance: 1e-10 of the
reference tests' scales. This file sorts last so a stop-at-first-failure run has run every other test first.
"""
import ctypes

import numpy as np
import pytest

from conftest import load_golden, scales

pytestmark = pytest.mark.gpu

_vp = ctypes.c_void_p


@pytest.mark.parametrize("name", ["stealthy_3d_n2000", "lattice_2d_skew", "lattice_1d", "empty_constraints"])
def test_noalloc_matches_handle_path(gpu, name):
    torch = pytest.importorskip("torch")
    r = load_golden(name)
    d = int(r["d"])
    p = gpu.CCPotential(d, r["basis"], r["modes"], r["V"], float(r["shift"]))
    p.set_configuration(r["frac"])
    E_ref = p.energy()
    re_ref, im_ref = p.rho()
    lib = gpu.load_library()
    dev = torch.device("cuda")
    frac = torch.tensor(np.mod(r["frac"], 1.0), dtype=torch.float64, device=dev)
    modes = torch.tensor(r["modes"].reshape(-1, d), dtype=torch.int32, device=dev)
    V = torch.tensor(r["V"], dtype=torch.float64, device=dev)
    M = len(r["V"])
    basis = np.ascontiguousarray(r["basis"], dtype=np.float64)
    s = scales(r)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        E = torch.full((1,), np.nan, dtype=torch.float64, device=dev)
        rho = torch.full((max(M, 1), 2), np.nan, dtype=torch.float64, device=dev)
        rc = lib.cc_energy_noalloc(d, basis.ctypes.data_as(_vp), M, _vp(modes.data_ptr()), _vp(V.data_ptr()),
                                   float(r["shift"]), len(r["frac"]), _vp(frac.data_ptr()), _vp(E.data_ptr()),
                                   _vp(rho.data_ptr()), _vp(stream))
        assert rc == 0, lib.cc_noalloc_last_error()
        torch.cuda.synchronize()
        e = E.item()
        assert abs(e - E_ref) <= 1e-10 * abs(E_ref) + 1e-13 * max(s["energy"], 1.0), (call, e, E_ref)
        if M:
            got = rho.cpu().numpy()[:M]
            assert np.abs(got[:, 0] - re_ref).max() <= 1e-10 * s["rho"], call
            assert np.abs(got[:, 1] - im_ref).max() <= 1e-10 * s["rho"], call


def test_noalloc_rejects_oversize(gpu):
    lib = gpu.load_library()
    basis = np.eye(2)
    E = ctypes.c_double()
    rc = lib.cc_energy_noalloc(2, basis.ctypes.data_as(_vp), 262145, _vp(8), _vp(8), 0.0, 10, _vp(8),
                               ctypes.cast(ctypes.byref(E), _vp), None, None)
    assert rc == -1
    assert b"CC_NOALLOC_MAX_MODES" in lib.cc_noalloc_last_error()
