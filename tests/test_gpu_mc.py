"""Monte Carlo trial moves (ShiftedCCPotential_ForMC::TryMove / AcceptMove) against the reference's ForMC class."""
import numpy as np
import pytest

import oracle
from conftest import load_golden, scales

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built")
@pytest.mark.parametrize("name", ["lattice_3d_skew", "stealthy_2d_n100"])
def test_mc_moves_match_reference(gpu, name):
    r = load_golden(name)
    d = int(r["d"])
    p = gpu.CCPotential(d, r["basis"], r["modes"], r["V"], float(r["shift"]))
    frac = np.mod(r["frac"], 1.0).copy()
    p.set_configuration(frac)
    ref = oracle.Ref(d, r["basis"], r["V"], modes=r["modes"], shift=float(r["shift"]))
    ref.set_positions(frac)
    s = scales(r)
    rng = np.random.default_rng(4)
    for step in range(40):
        i = int(rng.integers(len(frac)))
        after = np.mod(frac[i] + rng.normal(0, 0.05, d), 1.0)
        accept = bool(rng.random() < 0.5)
        dE_ref = ref.mc_try_move(frac[i], after, accept)
        dE = p.try_move(frac[i], after)
        assert abs(dE - dE_ref) <= 1e-9 * max(abs(dE_ref), 1.0) + 1e-12 * s["energy"], (step, dE, dE_ref)
        if accept:
            p.accept_move()
            frac[i] = after
    # accepting twice: the second call has no pending trial
    i = 0
    after = np.mod(frac[i] + 0.01, 1.0)
    assert abs(p.try_move(frac[i], after) - ref.mc_try_move(frac[i], after, True)) <= 1e-9 * max(s["energy"], 1.0)
    p.accept_move()
    with pytest.raises(gpu.CCError):
        p.accept_move()
