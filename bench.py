"""Benchmark of the collective-coordinate energy+gradient hot path on B200.

Workload: 3D stealthy CC configuration, N = 2000 points uniform in a periodic cube of side N^(1/3) (unit density),
chi = 0.45, the CLI's Type 0 k-set (M = 2724 half-space k-vectors, v(k) = 1): one STEP is one FP64 energy + Cartesian
forces evaluation of one configuration. Synthetic seeded inputs (no dataset exists for this workload).

  value : evaluations/s with positions resident in HBM. The evaluations run round-robin over a pool of distinct
          configurations larger than L2 (so no step re-reads cached inputs), replayed from CUDA graphs of the
          evaluations' kernels, timed with CUDA events on the launching stream. The pool is resident and never
          written during the run, so the handle is told so (cc_set_independent_positions): each evaluation's rho
          kernel computes while the previous evaluation's force kernel drains.
  e2e   : the same metric through the C ABI with host buffers, wall clock: one cc_energy_grad_many call per step (the
          step's positions from pinned host memory to the device and E and F back, inside the timed region, the
          copies overlapped with the evaluations); `e2e.per_call` is one cc_set_positions + cc_energy_grad call per
          configuration (the reference's interface), each waiting for its result.
  roofline: the dominant kernel's algorithmic FLOPs ((17 + 2d) per particle-k pair and evaluation: 8 in the rho
          kernel, 9 + 2d in the force kernel) / its CUDA-event duration, against the FP64 FMA peak measured in the
          same run by an FMA-chain probe kernel (MEASURED_PEAKS.json has no FP64 figure).
  cpu_baseline: the reference's own ShiftedCCPotential (Energy + AllForce, oracle/_ref) on the host cores.

--impl reference times that reference CPU path alone on the same workload and prints its line.
Multi-GPU: replicas only (independent configurations per rank, no collective on the data path).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

D, N, CHI = 3, 2000, 0.45
SIDE = N ** (1.0 / 3.0)
METRIC = "CC energy+grad evals/s"
UNIT = "evals/s"
# DRAM bytes (read + write) per launch of the kernels on this workload, from one ncu capture
# (profiles/cc_kernels_3d_n2000_ncu.md: dram__bytes_read.sum + dram__bytes_write.sum)
# DRAM bytes (read + write) per launch at this workload from ncu captures with ncu's default cache flush before each
# pass (cold); with warm caches (--cache-control none) each of the three kernels reads about 256 bytes of DRAM
NCU_TRAFFIC_BYTES = {"cc_force_kernel": 0.149e6, "cc_rho_kernel": 0.028e6, "cc_reduce_kernel": 1.418e6}
NCU_L2_BYTES_WARM = {"cc_force_kernel": 5.45e6, "cc_rho_kernel": 3.24e6, "cc_reduce_kernel": 2.23e6}
WORKLOAD = "3D stealthy CC ground-state evaluation: N=2000 uniform in a periodic cube (unit density), chi=0.45, " \
           "M=2724 half-space k (v=1), FP64 energy + Cartesian forces"
DATA = "synthetic (seeded uniform positions; k-set of the reference CLI's Type 0 rule)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--path", default="auto", choices=["auto", "split"],
                    help="evaluation path of the headline (auto: the library's own choice for this size)")
    ap.add_argument("--pool", type=int, default=4096,
                    help="configurations per step: each step evaluates every one once (their positions exceed L2)")
    ap.add_argument("--ref-seconds", type=float, default=120.0,
                    help="reference arm: about this many seconds of evaluations over warm-up and timed steps")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample length")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the batched / ground-state / served measurements")
    ap.add_argument("--batch", type=int, default=512, help="instances of the batched uneven workload")
    ap.add_argument("--gs-instances", type=int, default=48, help="instances of the ground-states/s comparison")
    ap.add_argument("--served", type=int, default=600, help="requests of the served sample (Poisson arrivals)")
    ap.add_argument("--served-rate", type=float, default=20.0, help="Poisson arrival rate of the served stream (1/s)")
    ap.add_argument("--served-capacity", type=int, default=300, help="requests of the capacity run (all at t = 0)")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(x, device):
    """The largest of every rank's x (a time): replicas are timed by the slowest one. Identity for one process."""
    import torch

    if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank, seconds, world):
    """Whole-job throughput of `world` replicas that each processed units_per_rank in at most `seconds`."""
    return world * units_per_rank / seconds


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons while running."""

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "samples": len(rows), "reasons": sorted(reasons)}


POOL_SEED = 1234


def pool_positions(P, rank=0):
    """The P distinct configurations of one step (seeded uniform fractional positions, P x N x D)."""
    return np.random.default_rng(POOL_SEED + rank).random((P, N, D))


def workload_config(M, P):
    """The workload as both arms print it (same keys, same values)."""
    return {"workload": WORKLOAD, "N": N, "d": D, "chi": CHI, "M": M, "pairs_per_eval": N * M,
            "configs_per_step": P, "positions_seed": POOL_SEED,
            "l2": f"inputs larger than L2: each step evaluates {P} distinct configurations "
                  f"({P * N * D * 8 / 1e6:.0f} MB of positions)"}


def reference_potential(cores):
    """The reference's own ShiftedCCPotential (Direct path, oracle/_ref) on this workload's k-set, built by the
    reference's own CLI rule (GeneratePotential Type 0)."""
    import oracle
    if not oracle.ref_available():
        raise RuntimeError("oracle/_ref/libccref.so is not built")
    basis = np.eye(D) * SIDE
    modes, V = oracle.ref_kset(D, basis, N, CHI, 0)
    return oracle.Ref(D, basis, V, modes=modes, nthreads=cores), len(V)


def cpu_reference_rate(seconds, pool):
    """The reference's Direct path on all host cores: SetConfiguration + Energy + AllForce per configuration of the
    pool, in order, for about `seconds`. Returns (evals/s, cores, evals, seconds)."""
    cores = os.cpu_count() or 1
    ref, _M = reference_potential(cores)
    ref.set_positions(pool[0])
    ref.eval()
    n = 0
    t0 = time.perf_counter()
    while True:
        ref.set_positions(pool[n % len(pool)])
        ref.eval()
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds and n >= 3:
            break
    return n / el, cores, n, el


def run_reference(args):
    """The reference arm: the reference's own CPU path on this workload. A step of the workload is one evaluation of
    each of the step's P configurations; the reference evaluates a bounded sample of each step (the first S of its
    configurations, S fixed so that warm-up and timed steps take about --ref-seconds in all)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    ref, M = reference_potential(cores)
    P = args.pool
    pool = pool_positions(P)
    t0 = time.perf_counter()
    for i in range(2):
        ref.set_positions(pool[i])
        ref.eval()
    t_eval = (time.perf_counter() - t0) / 2
    steps, warm = args.steps, args.warmup
    S = int(max(1, min(P, args.ref_seconds / max(1, steps + warm) / t_eval)))

    def one_step():
        for i in range(S):
            ref.set_positions(pool[i])
            ref.eval()

    for _ in range(warm):
        one_step()
    t0 = time.perf_counter()
    for _ in range(steps):
        one_step()
    el = time.perf_counter() - t0
    rate = steps * S / el
    sample = (f"each step: the first {S} of its {P} configurations (SetConfiguration+Energy+AllForce, reference "
              f"Direct path, OpenMP over {cores} threads); {steps} steps, {steps * S} evaluations in {el:.1f} s")
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
            "steps": steps, "warmup": warm, "ms_per_step": 1e3 * el / steps * (P / S), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA, "config": workload_config(M, P),
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def half_space_modes(d, nmax_f):
    """Integer modes n with |n| <= nmax_f and first nonzero component > 0 (the half space of the k-set rule)."""
    m = int(np.floor(nmax_f))
    axes = [np.arange(-m, m + 1)] * d
    n = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, d)
    n = n[(n * n).sum(1) <= nmax_f * nmax_f + 1e-9]
    first = np.array([row[np.nonzero(row)[0][0]] if row.any() else 0 for row in n])
    return np.ascontiguousarray(n[first > 0], dtype=np.int32)


def device_eval_ms(torch, pot, n, d, frac_dev, prec, reps=5):
    """Median CUDA-event time of energy+forces on resident positions, L2 flushed (256 MB write) before each eval."""
    E = torch.zeros(1, dtype=torch.float64, device="cuda")
    F = torch.zeros((n, d), dtype=torch.float64, device="cuda")
    flush = torch.empty(32 << 20, dtype=torch.float64, device="cuda")
    st = torch.cuda.Stream()
    evs = []
    with torch.cuda.stream(st):
        for i in range(2 + reps):
            flush.fill_(float(i))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            pot.energy_grad_device(n, frac_dev.data_ptr(), E.data_ptr(), F.data_ptr(), precision=prec,
                                   stream=st.cuda_stream)
            b.record(st)
            evs.append((a, b))
    torch.cuda.synchronize()
    ms = float(np.median([a.elapsed_time(b) for a, b in evs[2:]]))
    return ms, float(E.item()), F.cpu().numpy()


def run_single_legs(cc, torch):
    """The other single-configuration workloads of the path: the 2D N=100 ground state, the 3D N=2000 full
    minimisation with S(k) on |k| <= 1.5 K, and 2D N=1e5 in FP64 against mixed precision (errors reported)."""
    out = {}
    # 2D N=100 chi=0.30 (M=60): FP64 device L-BFGS to Phi/N < 1e-20 from five seeded starts
    d, n, chi = 2, 100, 0.30
    basis = np.eye(d) * n ** (1.0 / d)
    modes, V = cc.stealthy_kset(d, basis, n, chi)
    pot = cc.CCPotential(d, basis, modes, V)
    ts, evs, epp = [], [], []
    for seed in range(5):
        f0 = np.random.default_rng(100 + seed).random((n, d))
        t0 = time.perf_counter()
        _x, E, ev, _it, _st = pot.minimize(f0, stopval=1e-20 * n)
        ts.append(time.perf_counter() - t0)
        evs.append(ev)
        epp.append(E / n)
    out["ground_state_2d_n100"] = {"workload": "2D N=100 chi=0.30 M=60 v=1, FP64 L-BFGS (history 40) to Phi/N < 1e-20, "
                                               "5 seeded starts", "median_s": float(np.median(ts)),
                                   "median_evals": float(np.median(evs)), "max_E_per_particle": float(max(epp))}
    # 3D N=2000 chi=0.45 (M=2724): full minimisation (FP64, and mixed then FP64), then S(k) on |k| <= 1.5 K
    d, n, chi = 3, 2000, 0.45
    side = n ** (1.0 / d)
    basis = np.eye(d) * side
    modes, V = cc.stealthy_kset(d, basis, n, chi)
    pot = cc.CCPotential(d, basis, modes, V)
    f0 = np.random.default_rng(7).random((n, d))
    # one untimed minimisation per precision from another start: the handle's first call allocates its L-BFGS state
    fw = np.random.default_rng(8).random((n, d))
    pot.minimize(fw, stopval=1e-20 * n, max_evals=50)
    pot.minimize(fw, stopval=1e-20 * n, max_evals=50, precision=cc.PREC_SCHEDULE, switch_energy_per_particle=1e-10)
    t0 = time.perf_counter()
    x, E, ev, _it, _st = pot.minimize(f0, stopval=1e-20 * n)
    t_fp64 = time.perf_counter() - t0
    t0 = time.perf_counter()
    _x2, E2, ev2, _it2, _st2 = pot.minimize(f0, stopval=1e-20 * n, precision=cc.PREC_SCHEDULE,
                                            switch_energy_per_particle=1e-10)
    t_sched = time.perf_counter() - t0
    nmax = float(np.sqrt((np.asarray(modes, np.float64) ** 2).sum(1).max()))
    kq = half_space_modes(d, 1.5 * nmax)
    inside = (kq.astype(np.float64) ** 2).sum(1) <= nmax * nmax + 1e-9
    pot.set_configuration(x)
    S = pot.structure_factor(kq)
    reps = 20
    t0 = time.perf_counter()
    for _ in range(reps):
        S = pot.structure_factor(kq)
    t_sk = (time.perf_counter() - t0) / reps
    out["minimise_3d_n2000"] = {
        "workload": "3D N=2000 chi=0.45 M=2724 v=1 from a seeded uniform start, to Phi/N < 1e-20 (after an untimed "
                    "50-evaluation minimisation on the same handle)",
        "fp64_s": t_fp64, "fp64_evals": int(ev), "fp64_E_per_particle": E / n,
        "schedule_s": t_sched, "schedule_evals": int(ev2), "schedule_E_per_particle": E2 / n,
        "sk_modes": int(len(kq)), "sk_ms_per_call": t_sk * 1e3, "max_S_constrained": float(S[inside].max()),
        "mean_S_beyond": float(S[~inside].mean())}
    # 2D N=1e5 chi=0.20 (M=40002): the configuration of tests/golden/large_2d_n100000.npz, whose E, F and rho are the
    # reference's own FP64 results (made by tests/golden/make_golden_large.py); every path's error is against them
    with np.load(os.path.join(ROOT, "tests", "golden", "large_2d_n100000.npz")) as z:
        g = {k: z[k] for k in z.files}
    d, n = 2, len(g["frac"])
    modes, V, frac = g["modes"], g["V"], g["frac"]
    pot = cc.CCPotential(d, g["basis"], modes, V)
    fdev = torch.tensor(frac, dtype=torch.float64, device="cuda")
    kmax = 2 * np.pi * float(np.sqrt((modes.astype(np.float64) ** 2).sum(1).max())) / float(g["basis"][0, 0])
    sF = 4 * float(np.abs(V).sum()) * n * kmax / float(g["volume"])   # the reference tests' force scale

    def errs(E, F, prec):
        pot.set_configuration(frac)
        re, im = pot.rho(prec)
        return {"rel_err_E": abs(E - float(g["E"])) / abs(float(g["E"])),
                "max_err_F_over_max_F": float(np.abs(F - g["F"]).max() / np.abs(g["F"]).max()),
                "max_err_F_over_scale": float(np.abs(F - g["F"]).max() / sF),
                "max_err_rho_over_N": float(max(np.abs(re - g["rho_re"]).max(), np.abs(im - g["rho_im"]).max()) / n)}

    pot.set_path(cc.PATH_NUFFT)
    msnu, Enu, Fnu = device_eval_ms(torch, pot, n, d, fdev, cc.PREC_FP64)
    e_nu = errs(Enu, Fnu, cc.PREC_FP64)
    pot.set_path(cc.PATH_SPLIT)   # the direct kernels, FP64 and mixed
    ms64, E64, F64 = device_eval_ms(torch, pot, n, d, fdev, cc.PREC_FP64)
    e_64 = errs(E64, F64, cc.PREC_FP64)
    msmx, Emx, Fmx = device_eval_ms(torch, pot, n, d, fdev, cc.PREC_MIXED)
    e_mx = errs(Emx, Fmx, cc.PREC_MIXED)
    pairs = n * len(V)
    out["large_2d_n100000"] = {
        "workload": "2D N=100000 chi=0.20 M=40002 v=1, energy + forces, L2 flushed before each evaluation; errors "
                    "against the reference's own FP64 results on the same positions (tests/golden/large_2d_n100000)",
        "nufft_ms": msnu, "nufft_pairs_per_s_equivalent": pairs / (msnu / 1e3),
        "fp64_ms": ms64, "mixed_ms": msmx, "mixed_speedup": ms64 / msmx,
        "fp64_pairs_per_s": pairs / (ms64 / 1e3), "mixed_pairs_per_s": pairs / (msmx / 1e3),
        "nufft_vs_reference": e_nu, "fp64_vs_reference": e_64, "mixed_vs_reference": e_mx}
    return out


def run_extras(args, cc, torch):
    out = run_single_legs(cc, torch)
    # batched uneven instances: one batched energy+gradient step, CUDA-event timed, inputs resident
    from modules_b200.workloads import batched_workload
    pots, Ns, fracs, pairs = batched_workload(cc, args.batch)
    batch = cc.CCBatch(pots, Ns)
    batch.set_positions(fracs)
    tile = batch.autotune(reps=2)   # tile shapes chosen by timing the candidates on this batch
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        for _ in range(3):
            batch.eval_device(stream=st.cuda_stream)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 10
    with torch.cuda.stream(st):
        a.record(st)
        for _ in range(reps):
            batch.eval_device(stream=st.cuda_stream)
        b.record(st)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    out["batched"] = {"workload": f"{args.batch} instances, d in {{2,3}}, N log-uniform [200,5000], chi U[0.10,0.49], "
                                  "v=(1-|k|/K)^2, FP64", "ms_per_step": ms, "instance_evals_per_s": args.batch / (ms / 1e3),
                      "pairs_per_s": pairs / (ms / 1e3), "launches_per_step": 1,
                      "autotuned_tile": {"particles_per_rho_block": tile[0], "segments_per_force_block": tile[1]}}
    del batch
    # the headline configuration (3D N=2000, chi=0.45) through the same fused batch launch: 128 distinct
    # configurations of the step's pool per launch (an ensemble evaluated together: independent minimisations or
    # Monte Carlo chains), positions resident; the headline itself evaluates one configuration after another
    hbasis = np.eye(D) * SIDE
    hmodes, hV = cc.stealthy_kset(D, hbasis, N, CHI)
    HB = 128
    hb = cc.CCBatch([cc.CCPotential(D, hbasis, hmodes, hV) for _ in range(HB)], [N] * HB)
    hb.set_positions(list(pool_positions(HB)))
    htile = hb.autotune(reps=2)
    with torch.cuda.stream(st):
        for _ in range(3):
            hb.eval_device(stream=st.cuda_stream)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(st):
        a.record(st)
        for _ in range(reps):
            hb.eval_device(stream=st.cuda_stream)
        b.record(st)
    torch.cuda.synchronize()
    hms = a.elapsed_time(b) / reps
    out["batched_headline_config"] = {
        "workload": f"{HB} configurations of the headline workload (3D N={N} chi={CHI} M={len(hV)}) per fused batch "
                    "launch, positions resident, FP64",
        "ms_per_launch": hms, "evals_per_s": HB / (hms / 1e3), "pairs_per_s": HB * N * len(hV) / (hms / 1e3),
        "autotuned_tile": {"particles_per_rho_block": htile[0], "segments_per_force_block": htile[1]}}
    del hb
    # ground states per second: the plain single-configuration FP64 path, one instance after another, against the
    # batched minimisation of the same instances (mixed precision until E/N <= 1e-10, then FP64)
    rng = np.random.default_rng(77)
    gpots, gN, gfr = [], [], []
    for _ in range(args.gs_instances):
        d = int(rng.choice([2, 3]))
        n = int(round(np.exp(rng.uniform(np.log(200), np.log(1000)))))
        chi = float(rng.uniform(0.10, 0.40))
        basis = np.eye(d) * n ** (1.0 / d)
        modes, V = cc.stealthy_kset(d, basis, n, chi, 3)
        gpots.append(cc.CCPotential(d, basis, modes, V))
        gN.append(n)
        gfr.append(rng.random((n, d)))
    # untimed short runs first on both sides: each handle's and the batch's first minimisation allocates its L-BFGS
    # state, and a single allocation call on these hosts can take a large fraction of a second
    for p, f, n in zip(gpots, gfr, gN):
        p.minimize(f, stopval=1e-20 * n, max_evals=20)
    t0 = time.perf_counter()
    plain_E = []
    for p, f, n in zip(gpots, gfr, gN):
        x, E, ev, it, stt = p.minimize(f, stopval=1e-20 * n)
        plain_E.append(E / n)
    t_plain = time.perf_counter() - t0
    gb = cc.CCBatch(gpots, gN)
    gb.set_positions(gfr)
    gb.autotune(reps=2)
    gb.minimize(gfr, precision=cc.PREC_SCHEDULE, switch_energy_per_particle=1e-10, max_evals=20)
    t0 = time.perf_counter()
    xs, E, ev, it, stt = gb.minimize(gfr, precision=cc.PREC_SCHEDULE, switch_energy_per_particle=1e-10)
    t_batch = time.perf_counter() - t0
    epp = E / np.array(gN)
    out["ground_states"] = {
        "workload": f"{args.gs_instances} instances, d in {{2,3}}, N log-uniform [200,1000], chi U[0.10,0.40], "
                    "v=(1-|k|/K)^2, to Phi/N < 1e-20",
        "plain_fp64_per_s": args.gs_instances / t_plain, "batched_schedule_per_s": args.gs_instances / t_batch,
        "speedup": t_plain / t_batch, "reached": int((epp < 1e-20).sum()),
        "max_E_per_particle_batched": float(epp.max()), "max_E_per_particle_plain": float(max(plain_E))}
    del gb
    # served stream: config 5's distribution (N log-normal, median 1000, clipped to [100, 20000]; chi U[0.05, 0.49])
    # on a bounded sample of its 10000 requests, first with Poisson arrivals, then with every request at t = 0
    # (the server's capacity)
    from modules_b200.workloads import served_stream
    out["served"] = served_leg(cc, served_stream(args.served, args.served_rate, 20000, 0.49),
                               f"{args.served} requests, Poisson arrivals at {args.served_rate:g}/s")
    cap = served_stream(args.served_capacity, args.served_rate, 20000, 0.49, seed=100)
    for q in cap:
        q["arrival_s"] = 0.0
    out["served_capacity"] = served_leg(cc, cap, f"{args.served_capacity} requests, all arriving at t = 0")
    return out


def served_leg(cc, reqs, what):
    """Serve `reqs` and report throughput, time-to-ground-state percentiles and their split into admission wait
    (arrival to admission) and run time (admission to completion)."""
    res, wall = cc.serve(reqs, iters_per_round=16)
    arr = np.array([q["arrival_s"] for q in reqs])
    adm = np.array([r["t_admit"] for r in res])
    fin = np.array([r["t_done"] for r in res])
    lat, wait, run = fin - arr, adm - arr, fin - adm
    ok = np.array([r["status"] >= 0 and r["E"] / q["N"] < 1e-20 for r, q in zip(res, reqs)])
    slow = np.argsort(lat)[-max(1, len(lat) // 100):]   # the slowest 1 %
    pct = lambda x, p: float(np.percentile(x, p) * 1e3)   # noqa: E731
    return {"workload": what + ", d in {2,3}, N log-normal (median 1000, clipped to [100,20000]), chi U[0.05,0.49], "
                               "v in {1,(1-|k|/K)^2}, each to Phi/N < 1e-20",
            "requests": len(reqs), "ground_states_per_s": float(ok.sum()) / wall, "wall_s": wall,
            "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99),
            "admission_wait_p50_ms": pct(wait, 50), "admission_wait_p99_ms": pct(wait, 99),
            "run_p50_ms": pct(run, 50), "run_p99_ms": pct(run, 99),
            "slowest_1pct": {"admission_wait_ms": float(wait[slow].mean() * 1e3),
                             "run_ms": float(run[slow].mean() * 1e3),
                             "N_mean": float(np.mean([reqs[i]["N"] for i in slow])),
                             "evals_mean": float(np.mean([res[i]["evals"] for i in slow]))},
            "reached": int(ok.sum()), "not_reached": [
                {"N": int(reqs[i]["N"]), "d": int(reqs[i]["d"]), "chi": float(reqs[i]["chi"]),
                 "status": int(res[i]["status"]), "E_per_N": float(res[i]["E"] / reqs[i]["N"]),
                 "evals": int(res[i]["evals"])} for i in np.nonzero(~ok)[0][:20]]}


def run_ours(args):
    import torch

    import modules_b200 as cc

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    prec = cc.PREC_FP64 if args.precision == "fp64" else cc.PREC_MIXED
    basis = np.eye(D) * SIDE
    modes, V = cc.stealthy_kset(D, basis, N, CHI)
    M = len(V)
    pot = cc.CCPotential(D, basis, modes, V)
    path = {"auto": cc.PATH_AUTO, "split": cc.PATH_SPLIT}[args.path]
    pot.set_path(path)
    P = args.pool
    host_pool = pool_positions(P, rank)
    dev = torch.device("cuda", local)
    pool = torch.tensor(host_pool, dtype=torch.float64, device=dev)
    E = torch.zeros(P, dtype=torch.float64, device=dev)
    F = torch.zeros_like(pool)
    side = torch.cuda.Stream(device=dev)
    # the pool is written once, here, and never during the run: each evaluation's rho kernel may overlap the
    # previous evaluation's force kernel (results bitwise those of the default ordering)
    torch.cuda.synchronize()
    pot.set_independent_positions(True)

    def evaluate(i, stream):
        pot.energy_grad_device(N, pool[i].data_ptr(), E[i:i + 1].data_ptr(), F[i].data_ptr(), precision=prec,
                               stream=stream)

    # first evaluations allocate the library's work buffers (before any capture)
    with torch.cuda.stream(side):
        for i in range(3):
            evaluate(i, side.cuda_stream)
    torch.cuda.synchronize()

    # one step = one evaluation of each of the P configurations: CUDA graphs of G consecutive evaluations
    G = 128
    graphs = []
    for g0 in range(0, P, G):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            cs = torch.cuda.current_stream().cuda_stream
            for i in range(g0, min(P, g0 + G)):
                evaluate(i, cs)
        graphs.append(g)
    torch.cuda.synchronize()

    def run_step():
        for g in graphs:
            g.replay()

    with torch.cuda.stream(side):
        for _ in range(max(args.warmup, 3)):
            run_step()
    torch.cuda.synchronize()

    K = args.steps
    clocks = Clocks(local)
    time.sleep(0.3)   # the sampler is running before the timed region starts
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(side):
        t_start.record(side)
        for _ in range(K):
            run_step()
        t_end.record(side)
    torch.cuda.synchronize()
    ms = t_start.elapsed_time(t_end)
    clk = clocks.stop()
    ms = max_over_ranks(ms, dev)
    value = replica_rate(K * P, ms / 1e3, world)
    pot.check_device_error()

    # per-kernel CUDA-event timing: events recorded around each kernel INSIDE a replayed CUDA graph of G evaluations
    # (no host launch gap falls between an event and its kernel); the events are created before the capture
    pot.set_timing(True)
    with torch.cuda.stream(side):
        for i in range(G):
            evaluate(i, side.cuda_stream)
    pot.get_timing()
    pot.set_timing(True)
    tg = torch.cuda.CUDAGraph()
    with torch.cuda.graph(tg, stream=side):
        cs = torch.cuda.current_stream().cuda_stream
        for i in range(G):
            evaluate(i, cs)
    pot.set_timing(False)
    torch.cuda.synchronize()
    with torch.cuda.stream(side):
        tg.replay()
    torch.cuda.synchronize()
    rho_ms, red_ms, force_ms, nt = pot.get_timing()
    del tg
    info = pot.plan_info(N)
    info["path"] = pot.eval_path(N, prec)
    pairs = N * M
    t_rho, t_red, t_force = rho_ms / nt, red_ms / nt, force_ms / nt
    peak = cc.probe_fma_peak(cc.PREC_FP64 if prec == cc.PREC_FP64 else cc.PREC_MIXED)
    rho_flops, force_flops = 8.0 * pairs, (9.0 + 2 * D) * pairs
    # the dominant kernel is the force kernel: the largest share of the evaluation's device time in the ncu launch
    # list (42.8 % against rho 41.9 %) and of its FLOPs; their CUDA-event intervals are within a few percent of
    # each other and either can come out longer in a given run, so both are reported
    dom, fl, tk = "cc_force_kernel", force_flops, t_force
    kernel_ms = {"cc_rho_kernel": t_rho, "cc_reduce_kernel": t_red, "cc_force_kernel": t_force}
    launches_per_eval = 3
    achieved = fl / (tk * 1e-3) / 1e12

    # end to end through the C ABI with host buffers, the same K steps of P configurations. Headline: one
    # cc_energy_grad_many call per step (the step's positions from pinned host memory in, E and F out to pinned host
    # memory, copies overlapped with the evaluations). Beside it: one cc_set_positions + cc_energy_grad call per
    # configuration, each waiting for its result (the reference's one-configuration-per-call interface).
    h_in = torch.empty((P, N, D), dtype=torch.float64, pin_memory=True).numpy()
    h_in[:] = host_pool
    h_E = torch.empty(P, dtype=torch.float64, pin_memory=True).numpy()
    h_F = torch.empty((P, N, D), dtype=torch.float64, pin_memory=True).numpy()
    pot.energy_grad_many(h_in, h_E, h_F, precision=prec)   # untimed: the first call allocates the device buffers
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(K):
        pot.energy_grad_many(h_in, h_E, h_F, precision=prec)
    e2e_s = max_over_ranks(time.perf_counter() - t0, dev)
    e2e = replica_rate(K * P, e2e_s, world)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(K):
        for i in range(P):
            pot.set_configuration(host_pool[i])
            pot.energy_and_forces(precision=prec)
    e2e_call_s = max_over_ranks(time.perf_counter() - t0, dev)
    e2e_call = replica_rate(K * P, e2e_call_s, world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            rate, cores, n, el = cpu_reference_rate(args.cpu_seconds, host_pool)
            cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference",
                   "sample": f"{n} evaluations of the step's configurations in order (SetConfiguration+Energy+"
                             f"AllForce, reference Direct path, OpenMP over {cores} threads), {el:.1f} s"}
        except Exception as exc:  # the baseline is a report, never a reason to drop the GPU line
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"unavailable: {exc}"}

    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        try:
            extras = run_extras(args, cc, torch)
        except Exception as exc:   # extras are reports; never drop the headline line
            extras = {"extras_error": str(exc)[:300]}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
                "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if prec == cc.PREC_FP64 else "f32-recurrence/f64-accumulate",
                "data": DATA, "config": workload_config(M, P),
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                "method": {"path": info["path"], "graphs": f"CUDA graphs of {G} evaluations, {len(graphs)} per step",
                           "segment_len": info["L"], "segments": info["nseg"], "rho_splits": info["nsplit"],
                           "force_splits": info["nksplit"]},
                "pairs_per_s": value * pairs,
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": P * N * D * 8,
                        "d2h_bytes_per_step": P * (N * D * 8 + 8),
                        "api": "cc_energy_grad_many: one call per step, pinned host buffers, wall clock",
                        "per_call": {"value": e2e_call, "unit": UNIT,
                                     "api": "cc_set_positions + cc_energy_grad per configuration, wall clock"}},
                "gpu_launches": launches_per_eval * K * P,
                "roofline": {"bound": "fp64_fma" if prec == cc.PREC_FP64 else "fp32_fma", "kernel": dom,
                             "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                             "peak_source": "measured in this run: FMA-chain probe kernel (cc_probe_fma_peak); "
                                            "MEASURED_PEAKS.json has no FP64 figure",
                             "flops_per_launch": fl, "launch_ms": tk, "traffic": NCU_TRAFFIC_BYTES.get(dom),
                             "traffic_unit": "DRAM bytes per launch (ncu capture, cold caches; warm: ~256 B)",
                             "l2_bytes_warm": NCU_L2_BYTES_WARM.get(dom), "kernel_ms": kernel_ms,
                             "rho_kernel": {"flops_per_launch": rho_flops, "launch_ms": t_rho,
                                            "achieved": rho_flops / (t_rho * 1e-3) / 1e12,
                                            "frac": rho_flops / (t_rho * 1e-3) / 1e12 / peak},
                             "timing": "CUDA events around each kernel inside a replayed graph; under programmatic "
                                       "dependent launch consecutive kernels overlap, so the intervals overlap and "
                                       "sum to more than the evaluation",
                             "eval_us": 1e3 * ms / (K * P)},
                "clocks": clk, "cpu_baseline": cpu}
        line.update(extras)
        print(json.dumps(line), flush=True)
    del graphs
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
