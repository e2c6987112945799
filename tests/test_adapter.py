"""The C++ drop-in adapter (include/GpuCCPotential.h) against the reference's own class and optimiser."""
import os
import subprocess

import pytest

import oracle
from adapter_build import EXE, build


@pytest.mark.skipif(not (oracle.REFERENCE_TREE and os.path.isdir(oracle.REFERENCE_TREE)),
                    reason="needs the reference tree (CC_REFERENCE_TREE) to compile")
def test_adapter_compiles_against_reference_headers(ccgpu):
    if not oracle.ref_available():
        oracle.build(ref=True)
    assert build() == EXE and os.path.exists(EXE)


@pytest.mark.gpu
def test_adapter_matches_reference_and_minimises(gpu):
    if not os.path.exists(EXE):
        pytest.skip("adapter_check was not built (needs the reference tree at build time)")
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0 and "ADAPTER OK" in r.stdout, r.stdout + r.stderr
