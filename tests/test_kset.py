"""The product's host k-set generator (cc_kset_stealthy, C++) against the reference's CLI k-set."""
import hashlib

import numpy as np
import pytest

import oracle
from conftest import load_golden


def _sorted_key(modes):
    order = np.lexsort(modes.T[::-1])
    return np.ascontiguousarray(modes[order])


@pytest.mark.parametrize("name", ["ks_2d_n100_chi030", "ks_3d_n2000_chi045", "ks_3d_n300_chi030_t3",
                                  "ks_2d_n100000_chi020"])
def test_kset_matches_reference_golden(ccgpu, name):
    g = load_golden("ksets")
    d, N, chi, side, typ = (int(g[name + "__d"]), int(g[name + "__N"]), float(g[name + "__chi"]),
                            float(g[name + "__side"]), int(g[name + "__type"]))
    modes, V = ccgpu.stealthy_kset(d, np.eye(d) * side, N, chi, typ)
    assert len(V) == int(g[name + "__M"])
    key = _sorted_key(modes)
    assert hashlib.sha256(key.tobytes()).hexdigest() == str(g[name + "__sha"])
    # first nonzero index positive: one k of each +-k pair
    first = np.array([m[np.nonzero(m)[0][0]] for m in modes])
    assert np.all(first > 0)
    gm = g[name + "__modes"]
    if len(gm):
        o1, o2 = np.lexsort(gm.T[::-1]), np.lexsort(modes.T[::-1])
        assert np.allclose(g[name + "__V"][o1], V[o2], rtol=1e-12, atol=1e-15)


def test_kset_sizes_of_workloads(ccgpu):
    """M for the named workloads: 2D N=100 chi .30 -> 60; 3D N=2000 chi .45 -> 2724; 2D N=1e5 chi .20 -> 40002."""
    assert len(ccgpu.stealthy_kset(2, np.eye(2), 100, 0.30)[1]) == 60
    assert len(ccgpu.stealthy_kset(3, np.eye(3) * 2000 ** (1 / 3), 2000, 0.45)[1]) == 2724
    assert len(ccgpu.stealthy_kset(2, np.eye(2) * np.sqrt(1e5), 100000, 0.20)[1]) == 40002


@pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built")
@pytest.mark.parametrize("d,basis,N,chi,typ", [
    (2, [[1.3, 0.0], [0.45, 0.9]], 300, 0.35, 0),
    (3, [[1.1, 0.0, 0.0], [0.3, 0.95, 0.1], [0.2, -0.25, 1.2]], 200, 0.25, 3),
    (1, [[5.0]], 50, 0.37, 0),   # 1D: the CLI radius admits < want modes; Types 1-3 then read past its list
    (2, [[1.0, 0.3], [-0.4, 1.1]], 120, 0.49, 1),
    (3, np.eye(3) * 7.0, 400, 0.05, 0),
])
def test_kset_matches_reference_skew(ccgpu, d, basis, N, chi, typ):
    basis = np.array(basis, np.float64)
    rm, rv = oracle.ref_kset(d, basis, N, chi, typ)
    gm, gv = ccgpu.stealthy_kset(d, basis, N, chi, typ)
    assert len(rv) == len(gv)
    o1, o2 = np.lexsort(rm.T[::-1]), np.lexsort(gm.T[::-1])
    assert np.array_equal(rm[o1], gm[o2])
    assert np.allclose(rv[o1], gv[o2], rtol=1e-12, atol=1e-15)


def test_kset_zero_chi(ccgpu):
    modes, V = ccgpu.stealthy_kset(2, np.eye(2), 100, 0.0)
    assert len(V) == 0
