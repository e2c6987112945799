"""Parity of the sm_100a path (through the C ABI) with the reference's own FP64 results.

Tolerances: the FP64 path must agree with the reference to 1e-10 relative, measured against the reference tests'
scales (test_finufft_type1.cpp MakeScales :197-208; rho ~ N, energy ~ sum|V| N^2/vol, force ~ 4 sum|V| N kmax/vol),
and the energy also to 1e-10 of its own magnitude.
"""
import numpy as np
import pytest

import oracle
from conftest import golden_eval_cases, load_golden, scales

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def make_pot(gpu, r):
    return gpu.CCPotential(int(r["d"]), r["basis"], r["modes"], r["V"], float(r["shift"]))


def assert_energy(E, Eref, s):
    assert abs(E - Eref) <= RTOL * abs(Eref) + 1e-13 * max(s["energy"], 1.0), (E, Eref)


@pytest.mark.parametrize("name", golden_eval_cases())
def test_fp64_matches_reference(gpu, name):
    r = load_golden(name)
    s = scales(r)
    p = make_pot(gpu, r)
    p.set_configuration(r["frac"])
    E, F = p.energy_and_forces()
    assert_energy(E, float(r["E"]), s)
    if len(r["frac"]):
        assert F.shape == r["F"].shape
        assert np.abs(F - r["F"]).max() <= RTOL * s["force"]
    re, im = p.rho()
    if len(r["V"]):
        assert np.abs(re - r["rho_re"]).max() <= RTOL * s["rho"]
        assert np.abs(im - r["rho_im"]).max() <= RTOL * s["rho"]


def test_sign_kats(gpu):
    """TestSign: rho(k) = sum_j exp(+i k.r_j) on the analytic 1D and skew 2D cases."""
    r = load_golden("sign_1d")
    p = make_pot(gpu, r)
    p.set_configuration(r["frac"])
    re, im = p.rho()
    assert np.allclose([re[0], im[0], im[1], re[2]], [0.0, 1.0, -1.0, 1.0], atol=1e-12)
    r = load_golden("sign_2d_skew")
    p = make_pot(gpu, r)
    p.set_configuration(r["frac"])
    re, im = p.rho()
    p0, p1 = 2 * np.pi * (0.25 + 0.125), 2 * np.pi * (-2 * 0.25 + 3 * 0.125)
    assert np.allclose([re[0], im[0], re[1], im[1]], [np.cos(p0), np.sin(p0), np.cos(p1), np.sin(p1)], atol=1e-12)


def test_empty_lists(gpu):
    r = load_golden("empty_constraints")
    p = make_pot(gpu, r)
    p.set_configuration(r["frac"])
    E, F = p.energy_and_forces()
    assert E == 0.7 and F.shape == (12, 2) and np.all(F == 0)
    r = load_golden("empty_particles")
    p = make_pot(gpu, r)
    p.set_configuration(r["frac"])
    E, F = p.energy_and_forces()
    re, im = p.rho()
    assert E == 0.0 and F.shape == (0, 3) and np.all(re == 0) and np.all(im == 0)


def test_force_one_and_repeatability(gpu):
    r = load_golden("lattice_3d_skew")
    p = make_pot(gpu, r)
    p.set_configuration(r["frac"])
    E1, F1 = p.energy_and_forces()
    E2, F2 = p.energy_and_forces()
    assert E1 == E2 and np.array_equal(F1, F2)   # fixed summation order: bitwise repeatable
    for i in (0, 30, 59):
        assert np.array_equal(p.force(i), F1[i])


def test_graph_path_tracks_positions(gpu):
    """From its second identical call on, cc_energy_grad replays a captured graph that reads the staged positions
    itself; every visit of each of several configurations must give the first visit's energy, forces and rho
    (bitwise), rho being computed afterwards from the device copy of the positions that the graph leaves."""
    r = load_golden("lattice_3d_skew")
    p = make_pot(gpu, r)
    rng = np.random.default_rng(4)
    confs = [r["frac"]] + [rng.random(r["frac"].shape) for _ in range(3)]
    first = []
    for c in confs:
        p.set_configuration(c)
        E, F = p.energy_and_forces()
        first.append((E, F.copy(), p.rho()))
    for _ in range(3):
        for c, (E0, F0, (re0, im0)) in zip(confs, first):
            for _k in range(2):   # consecutive identical calls: the second at the latest runs the graph
                p.set_configuration(c)
                E, F = p.energy_and_forces()
                assert E == E0 and np.array_equal(F, F0)
            re, im = p.rho()
            assert np.array_equal(re, re0) and np.array_equal(im, im0)


def test_finite_difference(gpu):
    """TestFiniteDifference: central differences of the energy (h = 5e-5, rtol 1e-5, atol 1e-8)."""
    r = load_golden("fd_2d_skew")
    s = scales(r)
    p = make_pot(gpu, r)
    A = r["basis"]
    frac = r["frac"].copy()
    p.set_configuration(frac)
    _, F = p.energy_and_forces()
    h = 5e-5
    for i in (0, 17):
        cart = frac[i] @ A
        for dim in range(2):
            E = []
            for sgn in (1, -1):
                c = cart.copy()
                c[dim] += sgn * h
                f2 = frac.copy()
                f2[i] = np.linalg.solve(A.T, c)
                p.set_configuration(f2)
                E.append(p.energy())
            fd = -(E[0] - E[1]) / (2 * h)
            assert abs(F[i, dim] - fd) <= 1e-8 + 1e-5 * s["force"]


def test_objective_gradient(gpu):
    """The structure optimiser's Switch-0 objective: grad[i*d+j] = -F_i . a_j / rescale."""
    r = load_golden("lattice_2d_skew")
    p = make_pot(gpu, r)
    rescale = 10000.0
    x = (r["frac"] * rescale).reshape(-1)
    f, g = p.objective(x, rescale)
    s = scales(r)
    assert_energy(f, float(r["E"]), s)
    gref = -(r["F"] @ r["basis"].T).reshape(-1) / rescale
    assert np.abs(g - gref).max() <= RTOL * s["force"] * np.abs(r["basis"]).max() / rescale * 4


def test_cartesian_constructor_and_duplicates(gpu):
    r = load_golden("lattice_2d_rotated_skew")
    p = gpu.CCPotential(2, r["basis"], V=r["V"], shift=float(r["shift"]), kcart=r["kcart"])
    p.set_configuration(r["frac"])
    E, F = p.energy_and_forces()
    s = scales(r)
    assert_energy(E, float(r["E"]), s)
    assert np.abs(F - r["F"]).max() <= RTOL * s["force"]
    modes, _ = p.info()
    assert np.array_equal(modes, r["modes"])


def test_fixed_particle_offset(gpu):
    """HAVETWOFIXEDPARTICLES adds 2 to Re rho (GetRho_Direct :1268-1270); the energy and forces follow from rho."""
    r = load_golden("lattice_2d_skew")
    p = make_pot(gpu, r)
    p.set_configuration(r["frac"])
    p.set_rho_offset(2.0)
    E, F = p.energy_and_forces()
    re, im = r["rho_re"] + 2.0, r["rho_im"]
    vol = float(r["volume"])
    Eexp = float((r["V"] * (re * re + im * im)).sum() / vol + r["shift"])
    cart = oracle.port_eval  # noqa: F841  (the Cartesian positions below mirror the reference's)
    pos = r["frac"] @ r["basis"]
    ph = pos @ r["kcart"].T
    t = (r["V"][None, :] * (im[None, :] * np.cos(ph) - re[None, :] * np.sin(ph)))
    Fexp = -(2.0 / vol) * t @ r["kcart"]
    s = scales(r)
    assert abs(E - Eexp) <= 1e-10 * abs(Eexp)
    assert np.abs(F - Fexp).max() <= 1e-9 * s["force"]


def test_structure_factor_matches_reference(gpu):
    r = load_golden("stealthy_3d_n2000")
    sk = load_golden("sk_3d_n2000")
    p = make_pot(gpu, r)
    p.set_configuration(r["frac"])
    S = p.structure_factor(sk["sk_modes"])
    assert np.abs(S - sk["S"]).max() <= 1e-10 * max(1.0, sk["S"].max())


def test_device_path_matches_host(gpu):
    torch = pytest.importorskip("torch")
    r = load_golden("stealthy_3d_n2000")
    p = make_pot(gpu, r)
    p.set_configuration(r["frac"])
    E, F = p.energy_and_forces()
    d_frac = torch.tensor(r["frac"], dtype=torch.float64, device="cuda")
    d_E = torch.zeros(1, dtype=torch.float64, device="cuda")
    d_F = torch.zeros_like(d_frac)
    d_g = torch.zeros_like(d_frac)
    st = torch.cuda.current_stream().cuda_stream
    p.energy_grad_device(len(r["frac"]), d_frac.data_ptr(), d_E.data_ptr(), d_F.data_ptr(), d_g.data_ptr(), stream=st)
    torch.cuda.synchronize()
    assert d_E.item() == E
    assert np.array_equal(d_F.cpu().numpy(), F)
    gref = -(F @ r["basis"].T)
    assert np.abs(d_g.cpu().numpy() - gref).max() <= 1e-12 * np.abs(gref).max()


def test_independent_positions_bitwise(gpu):
    """A pool of resident configurations evaluated back to back with cc_set_independent_positions (the rho kernel
    runs its phase sums before waiting for the previous kernel on the stream), eagerly and replayed from a CUDA
    graph, gives bitwise the energies and forces of one synchronised evaluation at a time without it."""
    torch = pytest.importorskip("torch")
    r = load_golden("stealthy_3d_n2000")
    p = make_pot(gpu, r)
    n, d = r["frac"].shape
    rng = np.random.default_rng(5)
    pool_h = [np.mod(r["frac"] + rng.normal(0.0, 0.02, r["frac"].shape), 1.0) for _ in range(6)]
    pool = [torch.tensor(x, dtype=torch.float64, device="cuda") for x in pool_h]
    P = len(pool)
    E = torch.zeros(3, P, dtype=torch.float64, device="cuda")
    F = torch.zeros(3, P, n, d, dtype=torch.float64, device="cuda")
    st = torch.cuda.Stream()

    def run(rnd, i):
        p.energy_grad_device(n, pool[i].data_ptr(), E[rnd, i:i + 1].data_ptr(), F[rnd, i].data_ptr(),
                             stream=torch.cuda.current_stream().cuda_stream)

    with torch.cuda.stream(st):
        for i in range(P):   # one at a time, default ordering
            run(0, i)
            torch.cuda.synchronize()
        p.set_independent_positions(True)
        for i in range(P):   # back to back, early rho
            run(1, i)
        for i in range(P):
            run(1, i)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=st):
        for i in range(P):
            run(2, i)
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    del g
    p.set_independent_positions(False)
    assert torch.equal(E[1], E[0]) and torch.equal(F[1], F[0])
    assert torch.equal(E[2], E[0]) and torch.equal(F[2], F[0])
    p.set_configuration(pool_h[0])
    E0, F0 = p.energy_and_forces()
    assert E[1, 0].item() == E0 and np.array_equal(F[1, 0].cpu().numpy(), F0)


def test_energy_grad_many_matches_single(gpu):
    """cc_energy_grad_many over 70 configurations (two copy chunks), from pageable and from pinned host memory, with
    coordinates outside [0, 1) in some of them, equals bitwise one set_configuration + energy_and_forces call per
    configuration; a non-finite coordinate fails the call with CC_ERR_ARG and leaves the handle usable."""
    torch = pytest.importorskip("torch")
    r = load_golden("stealthy_3d_n2000")
    p = make_pot(gpu, r)
    n, d = r["frac"].shape
    rng = np.random.default_rng(11)
    pool = np.stack([np.mod(r["frac"] + rng.normal(0.0, 0.05, r["frac"].shape), 1.0) for _ in range(70)])
    pool[3] += 1.0
    pool[5, :40] -= 1.25
    pool[7, 0, 0] = 1.0
    E, F = p.energy_grad_many(pool)
    pin_in = torch.empty(pool.shape, dtype=torch.float64, pin_memory=True).numpy()
    pin_in[:] = pool
    pin_E = torch.empty(len(pool), dtype=torch.float64, pin_memory=True).numpy()
    pin_F = torch.empty(pool.shape, dtype=torch.float64, pin_memory=True).numpy()
    p.energy_grad_many(pin_in, pin_E, pin_F)
    E2, _ = p.energy_grad_many(pool, forces=False)
    for i in range(len(pool)):
        p.set_configuration(pool[i])
        Ei, Fi = p.energy_and_forces()
        assert E[i] == Ei and pin_E[i] == Ei and E2[i] == Ei, i
        assert np.array_equal(F[i], Fi) and np.array_equal(pin_F[i], Fi), i
    bad = pool[:3].copy()
    bad[1, 5, 0] = np.nan
    with pytest.raises(gpu.CCError) as e:
        p.energy_grad_many(bad)
    assert e.value.code == -1
    E3, F3 = p.energy_grad_many(pool[:3])
    assert np.array_equal(E3, E[:3]) and np.array_equal(F3, F[:3])


def test_mixed_precision_error(gpu):
    """Mixed path (FP32 seeds and recurrences, FP64 partials) against the FP64 path: report and bound the error."""
    r = load_golden("stealthy_3d_n2000")
    p = make_pot(gpu, r)
    p.set_configuration(r["frac"])
    E64, F64 = p.energy_and_forces()
    E32, F32 = p.energy_and_forces(precision=gpu.PREC_MIXED)
    rel_E = abs(E32 - E64) / abs(E64)
    rel_F = np.abs(F32 - F64).max() / np.abs(F64).max()
    print(f"mixed vs fp64: rel dE={rel_E:.2e} rel dF={rel_F:.2e}")
    assert rel_E < 1e-5 and rel_F < 1e-4


@pytest.mark.parametrize("path", ["split", "auto"])
def test_large_size_properties(gpu, path):
    """2D N=1e5 chi=0.20 (M=40002, 4e9 pairs): properties that hold at any size: total force zero,
    translation invariance of E and F, and (direct path) mixed precision close to FP64. The default path takes the
    NUFFT route at this size."""
    N = 100000
    side = np.sqrt(N)
    modes, V = gpu.stealthy_kset(2, np.eye(2) * side, N, 0.20)
    assert len(V) == 40002
    rng = np.random.default_rng(5)
    frac = rng.random((N, 2))
    p = gpu.CCPotential(2, np.eye(2) * side, modes, V)
    p.set_path(gpu.PATH_SPLIT if path == "split" else gpu.PATH_AUTO)
    p.set_configuration(frac)
    E, F = p.energy_and_forces()
    assert np.abs(F.sum(0)).max() <= 1e-9 * np.abs(F).sum(0).max()
    p.set_configuration(frac + np.array([0.123456789, -0.3]))
    E2, F2 = p.energy_and_forces()
    assert abs(E2 - E) <= 1e-10 * E
    assert np.abs(F2 - F).max() <= 1e-9 * np.abs(F).max()
    if path != "split":
        return
    p.set_configuration(frac)
    E3, F3 = p.energy_and_forces(precision=gpu.PREC_MIXED)
    print(f"N=1e5 mixed vs fp64: rel dE={abs(E3 - E) / E:.2e} rel dF={np.abs(F3 - F).max() / np.abs(F).max():.2e}")
    assert abs(E3 - E) <= 1e-4 * E
