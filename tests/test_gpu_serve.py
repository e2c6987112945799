"""The continuous-batching server: every request reaches its ground state, and a request's result is the same
(bitwise) served alone and in a mix of requests that arrive while it runs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests(seed=5):
    rng = np.random.default_rng(seed)
    specs = [(2, 150, 0.2, 0), (3, 200, 0.35, 3), (2, 400, 0.1, 3), (3, 120, 0.25, 0), (2, 250, 0.4, 3),
             (3, 300, 0.15, 0)]
    reqs = []
    for k, (d, N, chi, vt) in enumerate(specs):
        reqs.append(dict(d=d, N=N, chi=chi, vtype=vt, frac0=rng.random((N, d)), arrival_s=0.004 * k))
    return reqs


def test_serve_reaches_ground_states(gpu):
    reqs = _requests()
    res, wall = gpu.serve(reqs, iters_per_round=8)
    lat = [r["t_done"] - q["arrival_s"] for r, q in zip(res, reqs)]
    print(f"served {len(reqs)} in {wall:.3f}s, latencies {np.round(lat, 4).tolist()}")
    for r, q in zip(res, reqs):
        assert r["status"] == 1 and r["E"] / q["N"] < 1e-20
        assert r["t_done"] >= r["t_admit"] >= 0


def test_serve_same_alone_and_in_mix(gpu):
    reqs = _requests()
    mix, _ = gpu.serve(reqs, iters_per_round=8)
    for k in (1, 4):
        one = dict(reqs[k], arrival_s=0.0)
        alone, _ = gpu.serve([one], iters_per_round=8)
        assert alone[0]["E"] == mix[k]["E"] and alone[0]["evals"] == mix[k]["evals"]
