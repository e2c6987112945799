"""The large 2D workload (N = 100000, chi = 0.20, M = 40002 wavevectors, v = 1: about 4e9 particle-k pairs) against
the reference's own FP64 Energy, AllForce and GetRho on the same positions (tests/golden/large_2d_n100000.npz, made by
tests/golden/make_golden_large.py running potential/CollectiveCoordinatePotential.h:1255-1394 through oracle/_ref).

Tolerances: FP64 paths (direct kernels and non-uniform FFTs) within 1e-10 of the reference tests' scales
(test_finufft_type1.cpp MakeScales :197-208: rho ~ N, energy ~ sum|V| N^2 / vol, force ~ 4 sum|V| N kmax / vol) and
the energy within 1e-10 of itself. The mixed path (FP32 phases from exactly reduced FP64 arguments, FP64 sums) is
held to the bounds stated below and its errors against the reference are printed.
"""
import numpy as np
import pytest

from conftest import load_golden

RTOL = 1e-10
# mixed precision against the reference's FP64: energy relative, forces / rho against the scales
MIXED_E_REL = 1e-7
MIXED_SCALE_REL = 1e-6


def large_scales(r):
    n = len(r["frac"])
    side = float(r["basis"][0, 0])
    kmax = 2 * np.pi * float(np.sqrt((r["modes"].astype(np.float64) ** 2).sum(1).max())) / side
    sumV = float(np.abs(r["V"]).sum())
    vol = float(r["volume"])
    return dict(rho=float(n), energy=sumV * n * n / vol, force=4 * sumV * n * kmax / vol)


@pytest.fixture(scope="module")
def large():
    return load_golden("large_2d_n100000")


def test_golden_is_self_consistent(large):
    """CPU: the stored reference energy is sum V |rho|^2 / vol of the stored rho, the forces sum to zero, and the
    k-set is the CLI's set recorded in ksets.npz."""
    r = large
    E = float((r["V"] * (r["rho_re"] ** 2 + r["rho_im"] ** 2)).sum() / r["volume"])
    assert abs(E - float(r["E"])) <= 1e-12 * abs(E)
    s = large_scales(r)
    assert np.abs(r["F"].sum(0)).max() <= 1e-9 * s["force"]
    ks = load_golden("ksets")
    assert int(ks["ks_2d_n100000_chi020__M"]) == len(r["V"]) == 40002
    import hashlib
    key = np.ascontiguousarray(r["modes"][np.lexsort(r["modes"].T[::-1])])
    assert hashlib.sha256(key.tobytes()).hexdigest() == str(ks["ks_2d_n100000_chi020__sha"])


def _eval(gpu, r, path, prec):
    p = gpu.CCPotential(2, r["basis"], r["modes"], r["V"])
    p.set_path(path)
    p.set_configuration(r["frac"])
    E, F = p.energy_and_forces(precision=prec)
    re, im = p.rho(prec)
    return E, F, re, im


def _errors(r, E, F, re, im):
    s = large_scales(r)
    return dict(E_rel=abs(E - float(r["E"])) / abs(float(r["E"])),
                F_scale=float(np.abs(F - r["F"]).max() / s["force"]),
                F_maxF=float(np.abs(F - r["F"]).max() / np.abs(r["F"]).max()),
                rho_scale=float(max(np.abs(re - r["rho_re"]).max(), np.abs(im - r["rho_im"]).max()) / s["rho"]))


@pytest.mark.gpu
@pytest.mark.parametrize("path", ["split", "nufft"])
def test_fp64_matches_reference_large(gpu, large, path):
    r = large
    E, F, re, im = _eval(gpu, r, {"split": gpu.PATH_SPLIT, "nufft": gpu.PATH_NUFFT}[path], gpu.PREC_FP64)
    err = _errors(r, E, F, re, im)
    print(f"2D N=1e5 {path} FP64 vs reference: {err}")
    assert err["E_rel"] <= RTOL
    assert err["F_scale"] <= RTOL and err["rho_scale"] <= RTOL


@pytest.mark.gpu
def test_mixed_error_against_reference_large(gpu, large):
    r = large
    E, F, re, im = _eval(gpu, r, gpu.PATH_SPLIT, gpu.PREC_MIXED)
    err = _errors(r, E, F, re, im)
    print(f"2D N=1e5 mixed vs reference: {err}")
    assert err["E_rel"] <= MIXED_E_REL
    assert err["F_scale"] <= MIXED_SCALE_REL and err["rho_scale"] <= MIXED_SCALE_REL
