"""CPU check of the host planner's index arithmetic (tests/plan_check.cpp) on the workload k-sets and on adversarial
ones: scrambled modes with repeats, zero and negative modes, very wide index ranges, 1D/2D/3D."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden

EXE = os.path.join(ROOT, "tests", "_build", "plan_check")


@pytest.fixture(scope="module")
def plan_check():
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    src = os.path.join(ROOT, "tests", "plan_check.cpp")
    plan = os.path.join(ROOT, "modules_b200", "csrc", "cc_plan.cpp")
    subprocess.run(["g++", "-std=c++17", "-O1", "-o", EXE, src, plan], check=True)
    return EXE


def _run(exe, ksets):
    text = []
    for modes, V in ksets:
        modes = np.asarray(modes, np.int64).reshape(len(V), -1)
        d = modes.shape[1] if len(V) else 1
        text.append(f"{d} {len(V)}")
        for m, v in zip(modes, V):
            text.append(" ".join(str(int(x)) for x in m) + f" {float(v)!r}")
    r = subprocess.run([exe], input="\n".join(text) + "\n", capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_plan_workload_ksets(ccgpu, plan_check):
    ks = []
    for d, N, chi, side in [(2, 100, 0.30, 1.0), (3, 2000, 0.45, 2000 ** (1 / 3)), (2, 100000, 0.20, np.sqrt(1e5)),
                            (3, 5000, 0.49, 5000 ** (1 / 3)), (1, 500, 0.4, 500.0)]:
        ks.append(ccgpu.stealthy_kset(d, np.eye(d) * side, N, chi))
    out = _run(plan_check, ks)
    print(out)


def test_plan_adversarial(plan_check):
    rng = np.random.default_rng(3)
    ks = []
    for name in ["lattice_1d", "lattice_2d_skew", "lattice_3d_skew", "fd_2d_skew", "empty_particles"]:
        r = load_golden(name)
        ks.append((r["modes"], r["V"]))
    for d in (1, 2, 3):
        m = rng.integers(-1000000, 1000000, size=(300, d))
        ks.append((m, rng.uniform(-1, 1, 300)))
        m = rng.integers(-3, 4, size=(2000, d))          # many repeats
        ks.append((m, rng.uniform(0, 1, 2000)))
        line = np.zeros((5000, d), np.int64)
        line[:, d - 1] = np.arange(-2500, 2500)          # one very long line
        ks.append((line, np.ones(5000)))
        sparse = np.zeros((64, d), np.int64)
        sparse[:, 0] = np.arange(64) * 997               # far-apart prefixes
        ks.append((sparse, np.ones(64)))
    _run(plan_check, ks)
