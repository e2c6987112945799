"""The seeded request stream shared by the benchmark's served leg and `evalcase --serve` (host only)."""
import numpy as np

from modules_b200.workloads import served_stream


def test_served_stream_is_seeded_and_in_range():
    a, b = served_stream(200), served_stream(200)
    for x, y in zip(a, b):
        assert (x["d"], x["N"], x["chi"], x["vtype"], x["arrival_s"]) == (y["d"], y["N"], y["chi"], y["vtype"],
                                                                           y["arrival_s"])
        assert np.array_equal(x["frac0"], y["frac0"])
    t = np.array([r["arrival_s"] for r in a])
    assert np.all(np.diff(t) > 0)
    assert all(r["d"] in (2, 3) and 100 <= r["N"] <= 4000 and 0.05 <= r["chi"] <= 0.40 and r["vtype"] in (0, 3)
               for r in a)
    assert all(r["frac0"].shape == (r["N"], r["d"]) and r["frac0"].min() >= 0 and r["frac0"].max() < 1 for r in a)
    full = served_stream(200, rate=30.0, nmax=20000, chimax=0.49)
    assert max(r["N"] for r in full) <= 20000 and max(r["chi"] for r in full) <= 0.49
