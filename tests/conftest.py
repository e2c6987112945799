import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels through the C ABI")


def load_golden(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def golden_eval_cases():
    skip = {"ksets", "min_2d_n100", "sk_3d_n2000", "isotropic_sk", "multi_stealthy", "large_2d_n100000"}
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if os.path.basename(p)[:-4] not in skip)


def scales(rec):
    """Tolerance scales of the reference's tests (test_finufft_type1.cpp MakeScales :197-208):
    rho ~ N, energy ~ sum|V| N^2 / vol, force ~ 4 sum|V| N kmax / vol."""
    n = max(len(rec["frac"]), 1)
    sumV = float(np.abs(rec["V"]).sum())
    kmax = float(np.sqrt((rec["kcart"] ** 2).sum(1)).max()) if len(rec["V"]) else 0.0
    vol = float(rec["volume"])
    return dict(rho=float(n), energy=sumV * n * n / vol, force=4 * sumV * n * kmax / vol)


@pytest.fixture(scope="session")
def ccgpu():
    import modules_b200
    lib = modules_b200.load_library()
    return modules_b200


@pytest.fixture(scope="session")
def gpu(ccgpu):
    if not ccgpu.device_available():
        pytest.skip("no CUDA device")
    return ccgpu
