#!/usr/bin/env python
"""Benchmark: converged eigenpairs per second at FP64 residual <= 1e-10.

Workload (the Quantum Sun configuration the headline metric is quoted on):
spin-1/2 Quantum Sun, a grain of N=3 spins with a seeded GOE 8x8 block scaled
by gamma=1, L_loc=13 outer spins (full dimension 2^16 = 65536), couplings
alpha^{u_j} with alpha=0.75, u_j = (j-1) + U[-0.2, 0.2], fields U[0.5, 1.5],
g0=1; block Lanczos with block size s=8, nev=200 at rescaled energy 0.5,
FP64 throughout; KPM DoS with the reference defaults (N=250, R=300, Jackson).

One step = a batch of complete POLFED solves of fresh disorder realisations
(16 by default, ``--batch``) in flight together on a request pool's worker
streams; each solve runs the Emin/Emax Lanczos probes, KPM, interval and
order, the Chebyshev-filtered block Lanczos, Ritz extraction, FP64 Rayleigh
quotients and residuals.  An
eigenpair counts iff its FP64 residual ||H psi - E psi|| <= 1e-10 (eigentol).

* ``value``  -- whole-job eigenpairs/s with x0 and the outputs resident in HBM;
  timed with CUDA events on the library's stream, max over ranks.
* ``e2e``    -- the same metric through the public Python API with host x0 and
  host eigenvectors (H2D / D2H inside the timed region).
* ``roofline`` -- the dominant kernel (the Clenshaw recurrence step):
  algorithmic bytes per launch 4*D*s*8 (read b_{k+1}, b_{k+2}, X; write b_k)
  over its average duration inside the timed solves (CUDA events in the library).
* ``cpu_baseline`` -- one complete solve with the CPU port of the reference
  algorithm (oracle/) on this host's cores, measured.

N > 1 (torchrun): every rank solves its own realisations (replicas, no data
path collective); ``scaling`` is weak.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = {
    "workload": "qsun_Lloc13_Lgrain3_D65536_s8_nev200_eps0.5_fp64",
    "model": "Quantum Sun (S=1/2, full space)", "L_loc": 13, "L_grain": 3, "D": 65536, "g0": 1.0,
    "alpha": 0.75, "zeta": 0.2, "hz": 1.0, "w": 0.5, "gamma": 1.0, "blocksize": 8, "nev": 200,
    "target": "(:rescaled, 0.5)", "dos_N": 250, "dos_R": 300, "kernel": "Jackson", "eigentol": 1e-10,
}
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2
PROFILE_SUMMARY = os.path.join(ROOT, "profiles", "k_step_qsun_fp64_D65536_s8.md")


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


# --------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------- ranks
def rank_seed0(rank: int) -> int:
    """First realisation seed of a rank: ranks solve disjoint realisations."""
    return 1000 + 7919 * rank


def aggregate(nconv: float, seconds: float, world: int, device="cpu"):
    """Whole-job throughput over ranks: every rank's converged pairs divided
    by the slowest rank's device time.  Returns (value, total, max_seconds);
    collectives run on ``device`` (cuda with NCCL, cpu with gloo)."""
    if world == 1:
        return nconv / seconds, float(nconv), float(seconds)
    import torch
    import torch.distributed as dist
    tot = torch.tensor([float(nconv)], dtype=torch.float64, device=device)
    mx = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    return float(tot.item()) / float(mx.item()), float(tot.item()), float(mx.item())


# ----------------------------------------------------------- the workload
def make_realisations(pkg, n, seed0, device=0):
    import numpy as np
    ops, x0s = [], []
    for i in range(n):
        rng = np.random.default_rng(seed0 + i)
        op = pkg.qsun_hamiltonian(WORKLOAD["L_loc"], WORKLOAD["L_grain"], WORKLOAD["g0"], WORKLOAD["alpha"],
                                  gamma=WORKLOAD["gamma"], w=WORKLOAD["w"], hz=WORKLOAD["hz"],
                                  zeta=WORKLOAD["zeta"], rng=rng, device=device)
        D = 2 ** (WORKLOAD["L_loc"] + WORKLOAD["L_grain"])
        q, _ = np.linalg.qr(rng.standard_normal((D, WORKLOAD["blocksize"])))
        ops.append(op)
        x0s.append(np.asfortranarray(q))
    return ops, x0s


def solve(pkg, op, x0, seed):
    return pkg.polfed(op, x0, WORKLOAD["nev"], ("rescaled", 0.5), produce_report=True,
                      dos=pkg.DoSConfig(N=WORKLOAD["dos_N"], R=WORKLOAD["dos_R"], seed=seed),
                      fact=pkg.FactorizationConfig(eigentol=WORKLOAD["eigentol"]))


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def read_traffic():
    """DRAM bytes per launch of the step kernel from the committed ncu summary."""
    try:
        text = open(PROFILE_SUMMARY).read()
    except OSError:
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", text)
    return float(m.group(1)) if m else None


# ------------------------------------------------------- CPU baseline
def _cpu_realisation(seed, L_loc=None):
    """One seeded realisation of the workload for the CPU port: the FP64 CSR
    matrix (the operator of the reference's default CPU path, polfed(mat, ...)
    with optimize_mapping = false: mul!(Y, mat, X), PolfedCore.jl:172), x0 and
    the KPM probes."""
    import numpy as np
    from oracle import oracle as orc
    import __graft_entry__ as ge
    pkg = ge.load_package()
    L_loc = WORKLOAD["L_loc"] if L_loc is None else L_loc
    rng = np.random.default_rng(seed)
    f, n, c, g = pkg.qsun_parameters(L_loc, WORKLOAD["L_grain"], WORKLOAD["alpha"], gamma=WORKLOAD["gamma"],
                                     w=WORKLOAD["w"], hz=WORKLOAD["hz"], zeta=WORKLOAD["zeta"], rng=rng)
    H = orc.qsun_matrix(L_loc, WORKLOAD["L_grain"], WORKLOAD["g0"], c, n, f, g)
    D = H.shape[0]
    x0, _ = np.linalg.qr(rng.standard_normal((D, WORKLOAD["blocksize"])))
    probes = orc.normalized_gaussian_probes(D, WORKLOAD["dos_R"], rng)
    return orc.CSROperator(H), x0, probes


def cpu_solve(seed, L_loc=None, nev=None):
    """One complete POLFED solve of a fresh realisation on the host cores with
    the CPU port of the reference path (oracle/: C/OpenMP CSR kernels for the
    operator, Clenshaw filter and threaded KPM, numpy/OpenBLAS for Lanczos and
    the projected eigenproblem).  Returns (converged pairs at FP64 residual
    <= 1e-10, seconds)."""
    from oracle import oracle as orc
    op, x0, probes = _cpu_realisation(seed, L_loc)
    t0 = time.perf_counter()
    res = orc.polfed(op, x0, WORKLOAD["nev"] if nev is None else nev, ("rescaled", 0.5), N=WORKLOAD["dos_N"],
                     R=WORKLOAD["dos_R"], probes=probes, eigentol=WORKLOAD["eigentol"])
    return len(res.vals), time.perf_counter() - t0


def cpu_baseline_sample(seed=4242):
    """The cpu_baseline of our arm: one complete CPU solve of the workload,
    measured (not extrapolated)."""
    from oracle import oracle as orc
    n, sec = cpu_solve(seed)
    return {"value": n / sec, "unit": "eigenpairs/s", "cores": int(orc.lib().orc_num_threads()), "kind": "port",
            "sample": (f"one complete solve of a fresh realisation of the workload (D=65536, s=8, nev=200) with the "
                       f"CPU port of the reference's default path (CSR mul!, Clenshaw filter, threaded KPM with "
                       f"R=300 probes, FP64 block Lanczos): {n} pairs at residual <= 1e-10 in {sec:.1f} s")}


def run_reference(args, rank, world):
    """The reference arm: complete CPU solves with the CPU port of the
    reference's path on this host's cores, one fresh realisation per step.
    Warm-up steps solve a small realisation of the same model (L_loc = 7,
    nev = 20), which loads the kernels and starts the thread pools without the
    cost of a full solve."""
    if rank != 0:
        return 0
    from oracle import oracle as orc
    for i in range(args.warmup):
        cpu_solve(4000 + i, L_loc=7, nev=20)
    pairs, secs = [], []
    for k in range(args.steps):
        n, sec = cpu_solve(4242 + k)
        pairs.append(n)
        secs.append(sec)
    v = sum(pairs) / sum(secs)
    cores = int(orc.lib().orc_num_threads())
    cb = {"value": v, "unit": "eigenpairs/s", "cores": cores, "kind": "port",
          "sample": (f"{args.steps} complete solves of fresh realisations (D=65536, s=8, nev=200) with the CPU "
                     f"port of the reference's default path (CSR mul!, Clenshaw filter, threaded KPM, FP64 block "
                     f"Lanczos); {sum(pairs)} pairs at residual <= 1e-10 in {sum(secs):.1f} s")}
    out = {
        "metric": "converged eigenpairs/s at resid<=1e-10", "value": v, "unit": "eigenpairs/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(secs) / len(secs), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded realisations)",
        "config": dict(WORKLOAD, step="one complete CPU solve of a fresh realisation"),
        "impl": "reference", "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "eigenpairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "converged_per_solve": sum(pairs) / len(pairs),
    }
    print(json.dumps(out))
    return 0


# -------------------------------------------------------------- our arm
def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import torch.distributed as dist
    import __graft_entry__ as ge

    torch.cuda.set_device(local_rank)
    dev = f"cuda:{local_rank}"
    pkg = ge.load_package()
    from polfed_b200 import _lib
    pkg.load_library()
    B = max(1, args.batch)
    nsteps = args.warmup + args.steps
    ops, x0s = make_realisations(pkg, nsteps * B, rank_seed0(rank), device=local_rank)
    handle = _lib.handle(local_rank)
    stream = torch.cuda.ExternalStream(_lib.stream_of(handle), device=dev)
    # set-up outside the timed region: device descriptors, tuned step width, device x0,
    # worker handles (one stream each) for the batched solves
    width, _ = pkg.autotune(ops[0], WORKLOAD["blocksize"], "fp64")
    for o in ops[1:]:
        pkg.autotune(o, WORKLOAD["blocksize"], "fp64")
    x0_dev = []
    for x in x0s:
        t = pkg.col_major(x.shape[0], x.shape[1], device=local_rank)
        t.copy_(torch.from_numpy(np.ascontiguousarray(x)).to(dev))
        x0_dev.append(t)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    pool = pkg.solver_pool(B, local_rank)   # native request pool: B workers, one stream each
    wstreams = [torch.cuda.ExternalStream(st, device=dev) for st in pool.streams()]
    tstream = torch.cuda.Stream(device=dev)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()

    def batch(step, host):
        idx = list(range(step * B, (step + 1) * B))
        xs = [x0s[i] if host else x0_dev[i] for i in idx]
        return pool.solve_batch([ops[i] for i in idx], xs, WORKLOAD["nev"], ("rescaled", 0.5),
                                produce_report=True, dos=pkg.DoSConfig(N=WORKLOAD["dos_N"], R=WORKLOAD["dos_R"],
                                                                       seed=17 + step),
                                fact=pkg.FactorizationConfig(eigentol=WORKLOAD["eigentol"]))

    for k in range(args.warmup):
        batch(k, host=False)
    # the host-array path has its own first-call costs (page-locked staging,
    # result arrays): one more untimed batch of warm-up realisations through it
    batch(0, host=True)
    torch.cuda.synchronize()

    def join(into, streams):
        for ws in streams:
            ev = torch.cuda.Event()
            ev.record(ws)
            into.wait_event(ev)

    def timed(host_inputs):
        """K steps of B concurrent solves; device time from one timing stream
        that every worker stream waits on before a step and joins after it."""
        sampler = ClockSampler(local_rank)
        barrier()
        torch.cuda.synchronize()
        sampler.start()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        nconv, reps = [], []
        w0 = time.perf_counter()
        e0.record(tstream)
        for k in range(args.steps):
            with torch.cuda.stream(tstream):
                flush.fill_(float(k))  # evict the previous step's blocks from L2
            join(stream, [tstream])
            for ws in wstreams:
                join(ws, [tstream])
            for vals, vecs, rep in batch(args.warmup + k, host_inputs):
                nconv.append(len(vals))
                reps.append(rep)
            join(tstream, wstreams)
        e1.record(tstream)
        e1.synchronize()
        wall = time.perf_counter() - w0
        torch.cuda.synchronize()
        barrier()
        clocks = sampler.stop()
        return nconv, e0.elapsed_time(e1) * 1e-3, wall, reps, clocks

    nconv, sec, wall, breps, clocks = timed(host_inputs=False)
    value, _, sec_max = aggregate(sum(nconv), sec, world, device=dev)
    e_nconv, e_sec, e_wall, e_reps, e_clocks = timed(host_inputs=True)
    e_value, _, _ = aggregate(sum(e_nconv), e_sec, world, device=dev)
    # plain single solves (one at a time on one stream): the kernels run alone,
    # so the library's stage timers give the step kernel's own duration
    reps, s_conv = [], 0
    torch.cuda.synchronize()
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for k in range(args.steps):
        i = (args.warmup + k) * B
        vals, vecs, rep = solve(pkg, ops[i], x0_dev[i], seed=17 + k)
        s_conv += len(vals)
        reps.append(rep)
    s1.record(stream)
    s1.synchronize()
    single_value = s_conv / (s0.elapsed_time(s1) * 1e-3)
    D, s = ops[0].dim, WORKLOAD["blocksize"]

    # roofline of the Clenshaw step from the library's CUDA-event stage timers
    step_time, steps_total = 0.0, 0
    for r in reps:
        step_time += r.benchmark.stage_seconds["mapping"]
        steps_total += r.factorization.itersneeded * (r.spectral.order + 1)
    avg_step = step_time / max(steps_total, 1)
    alg_bytes = 4.0 * D * s * 8
    achieved = alg_bytes / avg_step / 1e9
    peak, peak_kind = read_peaks()
    # KPM: ceil((N-1)/2) doubling steps per probe column block, 3 D R_b 8 bytes each
    # (read v_n, read v_{n-1}, write v_{n+1}); all R probes pass through every step
    kpm_steps = (WORKLOAD["dos_N"] - 1 + 1) // 2
    kpm_bytes = 3.0 * D * WORKLOAD["dos_R"] * 8 * kpm_steps
    kpm_sec = statistics.mean(r.benchmark.stage_seconds["dos"] for r in reps)
    # the measured ceiling of an L2-resident step: random 64-byte row gathers
    gather_peak = _lib.gather_peak(local_rank, int(round(math.log2(D)))) / 1e9
    flip_bytes = float(D) * WORKLOAD["L_loc"] * s * 8   # the flipped rows a step gathers
    launches = sum(r.benchmark.kernel_launches for r in breps)
    stages = {k: sum(r.benchmark.stage_seconds[k] for r in reps) / len(reps) for k in reps[0].benchmark.stage_seconds}
    if rank != 0:
        return 0
    served = served_sample(pkg, local_rank) if world == 1 else None
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample()
    out = {
        "metric": "converged eigenpairs/s at resid<=1e-10", "value": value, "unit": "eigenpairs/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sec_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded disorder realisations, a fresh batch per step)",
        "config": dict(WORKLOAD, **{"l2": "256 MB buffer written between steps (inside the timed region)",
                                    "step": f"a batch of {B} full POLFED solves in flight together, "
                                            f"one per worker stream",
                                    "batch": B, "parallelism": f"replicas x{world}", "step_width": width,
                                    "step_profile": pkg.step_profile(ops[0], WORKLOAD["blocksize"])}),
        "e2e": {"value": e_value, "unit": "eigenpairs/s", "h2d_bytes_per_step": B * D * s * 8,
                "d2h_bytes_per_step": int(statistics.mean(e_nconv) * B * (D * 8 + 8)), "wall_seconds": e_wall},
        "single_solve": {"value": single_value, "unit": "eigenpairs/s",
                         "note": "one solve at a time on one stream (the plain single-solve form)"},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "k_step (Clenshaw recurrence)", "achieved": achieved,
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": read_traffic(), "algorithmic_bytes_per_launch": alg_bytes,
                     "avg_launch_us": avg_step * 1e6,
                     "measured_in": "the single-solve runs (library CUDA-event stage timers)",
                     "l2_gather": {"peak_gbs": gather_peak, "achieved_gbs": flip_bytes / avg_step / 1e9,
                                   "frac": flip_bytes / avg_step / 1e9 / gather_peak,
                                   "note": "the step's blocks stay in L2 (3 x 4 MB); its L_loc flipped-row "
                                           "gathers (64 B each) against the measured random-row gather "
                                           "throughput of an L2-resident block (pf_gather_peak)"},
                     "kpm": {"kernel": "k_step (KPM doubling step, fused dots)",
                             "algorithmic_bytes_per_solve": kpm_bytes,
                             "achieved": kpm_bytes / kpm_sec / 1e9, "frac": kpm_bytes / kpm_sec / 1e9 / peak,
                             "seconds_per_solve": kpm_sec,
                             "measured_in": "the single-solve runs (library stage timer 'dos')"}},
        "cpu_baseline": cpu,
        "served": served,
        "clocks": clocks,
        "e2e_clocks": e_clocks,
        "converged_per_solve": statistics.mean(nconv),
        "stage_seconds_per_solve": stages,
    }
    print(json.dumps(out))
    return 0


# ------------------------------------------------ served stream and disorder batch
SERVE = {"workload": "served stream: XXZ L=14..20 (Lup=L//2, W=5) and Quantum Sun L_grain=3, L_loc=10..15, "
                     "eps~U[0.1,0.9], nev in {20,50,100,200}, s in {4,8,16}, Poisson arrivals",
         "seed": 2025, "eigentol": 1e-10, "dos_N": 250, "dos_R": 300}
DISORDER = {"workload": "disorder average: 256 x XXZ L=16 (D=12870) + 32 x XXZ L=18 (D=48620), Sz=0, "
                        "Delta=1, W=3, nev=50, eps in {0.3,0.5,0.7}",
            "seed": 31337, "eigentol": 1e-10, "dos_N": 250, "dos_R": 300, "nev": 50}


def _serve_request(pkg, rng, device, small=False):
    """One request of the mixed served stream (seeded).  small: the bounded
    sample of the main benchmark line (XXZ L 14..16, Quantum Sun L_loc 10..13,
    nev 50..200), whose solves take well under a second each."""
    import numpy as np
    if rng.random() < 0.5:
        L = int(rng.integers(14, 17 if small else 21))
        op = pkg.xxz_hamiltonian(L, L // 2, 1.0, 1.0, 5.0, rng=rng, device=device)
        name = f"xxz_L{L}"
    else:
        L_loc = int(rng.integers(10, 14 if small else 16))
        op = pkg.qsun_hamiltonian(L_loc, 3, 1.0, 0.75, gamma=1.0, w=0.5, hz=1.0, zeta=0.2, rng=rng, device=device)
        name = f"qsun_Lloc{L_loc}"
    eps = float(rng.uniform(0.1, 0.9))
    nev = int(rng.choice([50, 100, 200] if small else [20, 50, 100, 200]))
    s = int(rng.choice([4, 8, 16]))
    x0 = np.asfortranarray(rng.random((op.dim, s)))
    return name, op, x0, eps, nev, s


def served_sample(pkg, local_rank, requests=12, rate=2.0, workers=4):
    """A bounded served stream for the main benchmark line: seeded Poisson
    arrivals submitted at their arrival times to a request pool; returns the
    pool's latency percentiles (submit -> done) and throughput."""
    import numpy as np
    rng = np.random.default_rng(SERVE["seed"] + 1)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=requests))
    arrivals -= arrivals[0]
    pool = pkg.SolverPool(workers=workers, device=local_rank)
    pool.set_admission("shortest")
    wrng = np.random.default_rng(1)
    _, op, x0, eps, nev, s = _serve_request(pkg, wrng, local_rank, small=True)
    pool.result(pool.submit(op, x0, 20, ("rescaled", eps), dos=pkg.DoSConfig(N=64, R=16, seed=1)))
    base = pool.stats()
    ids = []
    t0 = time.perf_counter()
    for i in range(requests):
        delay = t0 + arrivals[i] - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        _, op, x0, eps, nev, s = _serve_request(pkg, rng, local_rank, small=True)
        ids.append(pool.submit(op, x0, nev, ("rescaled", eps), vecs=False,
                               dos=pkg.DoSConfig(N=SERVE["dos_N"], R=SERVE["dos_R"], seed=SERVE["seed"] + i),
                               fact=pkg.FactorizationConfig(eigentol=SERVE["eigentol"])))
    nconv, rejected, failed, errors = 0, 0, 0, []
    for rid in ids:
        try:
            vals, _ = pool.result(rid)
            nconv += len(vals)
        except pkg._lib.PolfedRejected as e:
            rejected += 1
            errors.append(str(e))
        except pkg._lib.PolfedError as e:
            failed += 1
            errors.append(str(e))
    wall = time.perf_counter() - t0
    st = pool.stats()
    pool.close()
    return {"requests": requests, "rate_per_s": rate, "workers": workers, "admission": "shortest", "errors": errors,
            "mix": "XXZ L=14..16 (Sz=0 or -1/2) and Quantum Sun L_loc=10..13, eps~U[0.1,0.9], nev in {50,100,200}, "
                   "s in {4,8,16}, seeded Poisson arrivals",
            "eigenpairs_per_s": nconv / wall, "converged": nconv, "rejected": rejected, "failed": failed,
            "latency_s": {"p50": st.p50_latency, "p99": st.p99_latency, "mean": st.mean_latency,
                          "note": "submit -> done, host clock, queueing included"},
            "completed": st.completed - base.completed, "wall_seconds": wall}


def run_serve(args, local_rank):
    """A seeded Poisson request stream through the native request pool.
    Requests are created and submitted at their arrival times; latency is
    submit -> done (host clock, the pool's own record); throughput is the
    converged pairs of all requests over the first arrival -> last completion."""
    import numpy as np
    import torch
    import __graft_entry__ as ge
    torch.cuda.set_device(local_rank)
    pkg = ge.load_package()
    pkg.load_library()
    rng = np.random.default_rng(SERVE["seed"])
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, size=args.requests))
    arrivals -= arrivals[0]
    pool = pkg.SolverPool(workers=args.workers, device=local_rank)
    pool.set_admission(args.admission)
    # warm-up: one small request of each kind (library set-up, cuBLAS/cuSOLVER handles)
    wrng = np.random.default_rng(1)
    for _ in range(2):
        name, op, x0, eps, nev, s = _serve_request(pkg, wrng, local_rank)
        pool.result(pool.submit(op, x0, 20, ("rescaled", eps), dos=pkg.DoSConfig(N=64, R=16, seed=1)))
    torch.cuda.synchronize()
    base = pool.stats()
    sampler = ClockSampler(local_rank)
    sampler.start()
    ids, meta = [], []
    t0 = time.perf_counter()
    for i in range(args.requests):
        delay = t0 + arrivals[i] - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        name, op, x0, eps, nev, s = _serve_request(pkg, rng, local_rank)
        rid = pool.submit(op, x0, nev, ("rescaled", eps), produce_report=True, vecs=False,
                          dos=pkg.DoSConfig(N=SERVE["dos_N"], R=SERVE["dos_R"], seed=SERVE["seed"] + i),
                          fact=pkg.FactorizationConfig(eigentol=SERVE["eigentol"]))
        ids.append(rid)
        meta.append((name, op, op.dim, nev, s, eps))
    nconv, per = 0, []
    for rid, (name, op, D, nev, s, eps) in zip(ids, meta):
        item = {"model": name, "D": D, "nev": nev, "s": s, "eps": round(eps, 3)}
        try:
            vals, _, rep = pool.result(rid)
        except pkg._lib.PolfedRejected as e:
            # infeasible: fewer than nev states within reach of the target (the
            # reference raises the same bisection error); rejected, not failed
            item["rejected"] = str(e)
            per.append(item)
            continue
        except pkg._lib.PolfedError as e:
            item["error"] = str(e)
            per.append(item)
            continue
        nconv += len(vals)
        item.update({"converged": len(vals), "K": rep.spectral.order,
                     "solve_s": round(rep.benchmark.stage_seconds["total"], 4)})
        per.append(item)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    st = pool.stats()
    pool.close()
    lat = sorted(p["solve_s"] for p in per if "solve_s" in p) or [0.0]
    out = {
        "metric": "converged eigenpairs/s at resid<=1e-10 (served stream)", "value": nconv / wall,
        "unit": "eigenpairs/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f64",
        "data": "synthetic (seeded request stream)",
        "config": dict(SERVE, requests=args.requests, rate_per_s=args.rate, workers=args.workers,
                       admission=args.admission),
        "latency_s": {"p50": st.p50_latency, "p99": st.p99_latency, "mean": st.mean_latency,
                      "note": "submit -> done, host clock, queueing included"},
        "solve_seconds": {"p50": lat[len(lat) // 2], "max": lat[-1]},
        "wall_seconds": wall, "busy_seconds": st.busy_seconds - base.busy_seconds,
        "converged": nconv, "completed": st.completed - base.completed, "failed": st.failed - base.failed,
        "rejected": st.rejected - base.rejected,
        "hbm": {"budget_bytes": st.bytes_budget, "peak_admitted_bytes": st.bytes_peak},
        "clocks": clocks, "requests": per,
    }
    print(json.dumps(out))
    return 0


def _disorder_problems(pkg, device):
    import numpy as np
    probs = []
    for i in range(288):
        L = 16 if i < 256 else 18
        rng = np.random.default_rng(DISORDER["seed"] + i)
        op = pkg.xxz_hamiltonian(L, L // 2, 1.0, 1.0, 3.0, rng=rng, device=device)
        probs.append((op, (0.3, 0.5, 0.7)[i % 3], rng))
    return probs


def run_disorder(args, local_rank):
    """The disorder average: 288 realisations through the request pool, block
    size per L picked by timing s in {4, 8, 16} on one realisation, against
    the same realisations solved one at a time."""
    import numpy as np
    import torch
    import __graft_entry__ as ge
    torch.cuda.set_device(local_rank)
    dev = f"cuda:{local_rank}"
    pkg = ge.load_package()
    pkg.load_library()
    probs = _disorder_problems(pkg, local_rank)
    kw = lambda seed: dict(fact=pkg.FactorizationConfig(eigentol=DISORDER["eigentol"]), vecs=False,
                           dos=pkg.DoSConfig(N=DISORDER["dos_N"], R=DISORDER["dos_R"], seed=seed))
    nev = DISORDER["nev"]
    # block-size tuner (outside the timed region): converged pairs per second of one solve
    best_s, tune = {}, {}
    for L, i in ((16, 0), (18, 256)):
        best_s[L], rates = pkg.tune_block_size(probs[i][0], nev, ("rescaled", 0.5), (4, 8, 16), **kw(1))
        tune[f"L{L}"] = {str(k): round(v, 2) for k, v in rates.items()}
    x0s = []
    for op, eps, rng in probs:
        s = best_s[16 if op.dim == 12870 else 18]
        x0s.append(np.asfortranarray(rng.random((op.dim, s))))
    pool = pkg.SolverPool(workers=args.workers, device=local_rank)
    streams = [torch.cuda.ExternalStream(st, device=dev) for st in pool.streams()]
    tstream = torch.cuda.Stream(device=dev)

    def timed_pool(idx):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(tstream)
        for ws in streams:
            ws.wait_event(e0)
        # every realisation queued at once with its own target, largest D first
        # (longest solves start first, so no worker idles at the end on a
        # batch boundary)
        order = sorted(idx, key=lambda i: -probs[i][0].dim)
        rids = [pool.submit(probs[i][0], x0s[i], nev, ("rescaled", probs[i][1]), **kw(5)) for i in order]
        nconv = sum(len(pool.result(r)[0]) for r in rids)
        for ws in streams:
            ev = torch.cuda.Event()
            ev.record(ws)
            tstream.wait_event(ev)
        e1.record(tstream)
        e1.synchronize()
        return nconv, e0.elapsed_time(e1) * 1e-3

    timed_pool(list(range(0, 288, 24)))   # warm-up
    sampler = ClockSampler(local_rank)
    sampler.start()
    n_pool, t_pool = timed_pool(list(range(288)))
    clocks = sampler.stop()
    # the single-solve form: one at a time on the library's stream, every 4th realisation
    from polfed_b200 import _lib
    st = torch.cuda.ExternalStream(_lib.stream_of(_lib.handle(local_rank)), device=dev)
    sub = list(range(0, 288, 4))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    n_single = 0
    for i in sub:
        vals, _ = pkg.polfed(probs[i][0], x0s[i], nev, ("rescaled", probs[i][1]), **kw(5))
        n_single += len(vals)
    e1.record(st)
    e1.synchronize()
    t_single = e0.elapsed_time(e1) * 1e-3
    pool.close()
    out = {
        "metric": "converged eigenpairs/s at resid<=1e-10 (disorder batch)", "value": n_pool / t_pool,
        "unit": "eigenpairs/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f64",
        "data": "synthetic (seeded realisations)",
        "config": dict(DISORDER, workers=args.workers, blocksize={f"L{k}": v for k, v in best_s.items()}),
        "blocksize_tuning_pairs_per_s": tune,
        "seconds": t_pool, "converged": n_pool,
        "single_solve": {"value": n_single / t_single, "unit": "eigenpairs/s", "realisations": len(sub),
                         "converged": n_single, "seconds": t_single},
        "clocks": clocks,
    }
    print(json.dumps(out))
    return 0


C3 = {"workload": "j1j2_L24_Sz0_D2704156_s16_nev100_eps0.5_fp64",
      "model": "J1-J2 Heisenberg chain, PBC, J1=1, J2=0.5, Delta=1, h_i~U[-1,1], Sz=0", "L": 24, "D": 2704156,
      "blocksize": 16, "nev": 100, "target": "(:rescaled, 0.5)", "dos_N": 512, "dos_R": 64,
      "probes": "Rademacher +-1/sqrt(D)", "eigentol": 1e-10, "seed": 2424}


def run_c3(args, local_rank):
    """One complete FP64 solve at the J1-J2 L = 24 configuration, with every
    returned pair's residual checked again against the FP64 CSR matrix of the
    oracle (a different code path: scipy sparse products on the host) for a
    sample of the returned vectors."""
    import numpy as np
    import torch
    import __graft_entry__ as ge
    from oracle import oracle as orc
    torch.cuda.set_device(local_rank)
    pkg = ge.load_package()
    pkg.load_library()
    rng = np.random.default_rng(C3["seed"])
    op = pkg.j1j2_hamiltonian(24, 12, 1.0, 0.5, 1.0, 1.0, 1.0, rng=rng, device=local_rank)
    D, s, nev = op.dim, C3["blocksize"], C3["nev"]
    x0 = np.asfortranarray(rng.random((D, s)))
    pkg.autotune(op, s, "fp64")
    sampler = ClockSampler(local_rank)
    sampler.start()
    t0 = time.perf_counter()
    vals, vecs, rep = pkg.polfed(op, x0, nev, ("rescaled", 0.5), produce_report=True,
                                 dos=pkg.DoSConfig(N=C3["dos_N"], R=C3["dos_R"], probe_kind="rademacher", seed=11),
                                 fact=pkg.FactorizationConfig(eigentol=C3["eigentol"]))
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    t1 = time.perf_counter()
    H = orc.j1j2_matrix(24, 12, 1.0, 0.5, 1.0, 1.0, op.fields)
    sample = list(range(0, len(vals), max(1, len(vals) // 8)))[:8]
    res = [float(np.linalg.norm(H @ vecs[:, j] - vals[j] * vecs[:, j])) for j in sample]
    check_s = time.perf_counter() - t1
    b = rep.benchmark
    steps = rep.factorization.itersneeded * (rep.spectral.order + 1)
    out = {"metric": "converged eigenpairs/s at resid<=1e-10 (J1-J2 L=24 solve)",
           "value": len(vals) / b.stage_seconds["total"], "unit": "eigenpairs/s", "n_gpus": 1, "dtype": "f64",
           "data": "synthetic (seeded realisation)", "config": C3, "converged": len(vals),
           "solve_seconds": b.stage_seconds["total"], "wall_seconds": wall, "order": rep.spectral.order,
           "iters": rep.factorization.itersneeded, "krylovdim": rep.factorization.krylovdim,
           "eigenresidual_max": rep.factorization.eigenresidual,
           "step_us": 1e6 * b.stage_seconds["mapping"] / max(steps, 1),
           "step_frac_of_hbm": (4.0 * D * s * 8) / (b.stage_seconds["mapping"] / max(steps, 1)) / 1e9 /
                               read_peaks()[0],
           "csr_check": {"vectors": sample, "residuals": res, "max": max(res) if res else None,
                         "seconds": check_s},
           "stage_seconds": b.stage_seconds, "clocks": clocks}
    print(json.dumps(out))
    return 0


def profile_step(width=None, profile=0):
    """Two order-30 Chebyshev filters on one realisation of the workload's
    operator (s = 8, FP64) with the autotuned step, or with the given step
    width and profile (the autotuner's timings are not those of a run under
    ncu, which serialises every launch): a small, bounded case for ncu
    captures of the step kernel."""
    import numpy as np
    import torch
    import __graft_entry__ as ge
    pkg = ge.load_package()
    ops, x0s = make_realisations(pkg, 1, 1000)
    op = ops[0]
    if width is None:
        width, _ = pkg.autotune(op, WORKLOAD["blocksize"], "fp64")
    else:
        pkg.set_step_width(op, WORKLOAD["blocksize"], width, "fp64", profile)
    D, s = op.dim, WORKLOAD["blocksize"]
    X = pkg.col_major(D, s)
    X.copy_(torch.from_numpy(np.ascontiguousarray(x0s[0])).cuda())
    Y = pkg.col_major(D, s)
    c = np.cos(np.arange(31) * 1.0) * 0.05
    torch.cuda.synchronize()
    # the filters run inside an NVTX range "filters", so a capture can leave
    # out the autotuner's timing launches (ncu --nvtx --nvtx-include filters/)
    torch.cuda.nvtx.range_push("filters")
    for _ in range(2):
        pkg.chebyshev_filter(op, Y, X, c, a=8.0, b=0.0)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    print(json.dumps({"profile_step": True, "D": D, "s": s, "width": width,
                      "profile": pkg.step_profile(op, s), "norm": float(Y.norm())}))
    return 0


# The reference's published single-vector XXZ H-apply times, FP64, Delta = 0.55,
# PBC, Sz = 0 (docs/src/tutorials/advanced/custom-mapping/index.md:92-115; CPU,
# hardware not stated): generic sparse mul! and its bucketed custom mapping, us.
PUBLISHED_APPLY = {18: (856.653, 579.533), 20: (5402.0, 2340.0), 22: (25727.0, 10202.0), 24: (109943.0, 41825.0)}


def apply_sweep():
    """The reference's only published timings on this path, re-measured here:
    one H-apply of a single vector (s = 1) of the XXZ chain at L = 18..24,
    Delta = 0.55, PBC, Sz = 0, FP64, through pf_apply (graph-free, one launch
    per apply).  CUDA events on the library stream around 200 applies issued
    back to back through the C entry point after 20 warm-up applies (at small
    L the host's issue rate can bound it); inputs larger than L2 at L >= 22,
    L2-resident below."""
    import torch
    import __graft_entry__ as ge
    pkg = ge.load_package()
    from polfed_b200 import _lib
    st = torch.cuda.ExternalStream(_lib.stream_of(_lib.handle(0)), device="cuda:0")
    for L, (generic, custom) in PUBLISHED_APPLY.items():
        op = pkg.xxz_hamiltonian(L, L // 2, 1.0, 0.55, 0.0, fields=[0.0] * L)
        D = op.dim
        X = pkg.col_major(D, 1)
        X.copy_(torch.rand(D, 1, dtype=torch.float64, device="cuda:0"))
        Y = pkg.col_major(D, 1)
        pkg.apply(op, Y, X)   # creates the operator and joins the streams once
        torch.cuda.synchronize()
        lib, h = _lib.load(), op.op
        args = (h, _lib.PF_F64, 1.0, 0.0, 1, X.data_ptr(), D, Y.data_ptr(), D)
        for _ in range(20):
            _lib.check(lib.pf_apply(*args))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n = 200
        e0.record(st)
        for _ in range(n):
            _lib.check(lib.pf_apply(*args))
        e1.record(st)
        e1.synchronize()
        us = e0.elapsed_time(e1) * 1e3 / n
        print(json.dumps({"apply_sweep": True, "model": "xxz", "L": L, "D": D, "s": 1, "dtype": "f64",
                          "us_per_apply": us, "rows_per_s": D / us * 1e6,
                          "published_us": {"generic_mul": generic, "custom_mapping": custom},
                          "speedup_vs_custom": custom / us}), flush=True)
    return 0


def profile_solve():
    """Two complete solves of the workload (two fresh realisations) through
    pkg.polfed, no pool: a bounded case for an ncu launch list of solves."""
    import __graft_entry__ as ge
    pkg = ge.load_package()
    ops, x0s = make_realisations(pkg, 2, 1000)
    for i in range(2):
        vals, _, rep = solve(pkg, ops[i], x0s[i], seed=17 + i)
    print(json.dumps({"profile_solve": True, "pairs": len(vals), "order": rep.spectral.order,
                      "launches": int(rep.benchmark.kernel_launches)}))
    return 0


def profile_kpm():
    """KPM on the workload's operator at its block width: one 64-probe block of
    normalised Gaussian probes, 40 moments (20 doubling steps with fused
    dots), FP64 -- a bounded case for ncu captures of the KPM step."""
    import numpy as np
    import __graft_entry__ as ge
    pkg = ge.load_package()
    ops, _ = make_realisations(pkg, 1, 1000)
    op = ops[0]
    mu = pkg.kpm_moments(op, 40, 64, a=8.0, b=0.0)
    print(json.dumps({"profile_kpm": True, "D": op.dim, "R": 64, "N": 40, "mu0": float(np.asarray(mu)[0])}))
    return 0


def profile_gram():
    """The split-BF16 tensor-core Gram product G = B^T r at the workload's
    final Krylov size (D = 65536, 624 basis columns, s = 8), twice -- a
    bounded case for ncu captures of k_gram_bf16x3."""
    import torch
    import __graft_entry__ as ge
    ge.load_package()
    from polfed_b200 import _lib
    D, nB, s = 65536, 624, WORKLOAD["blocksize"]
    g = torch.Generator(device="cuda:0").manual_seed(5)
    B = torch.randn(D, nB, dtype=torch.float64, device="cuda:0", generator=g)
    r = torch.randn(D, s, dtype=torch.float64, device="cuda:0", generator=g)
    G = torch.empty(s, nB, dtype=torch.float64, device="cuda:0")
    for _ in range(2):
        _lib.check(_lib.load().pf_gram_bf16x3(_lib.handle(0), D, nB, B.data_ptr(), nB, r.data_ptr(), s,
                                              G.data_ptr()))
    torch.cuda.synchronize()
    ref = (B.t() @ r).t()
    err = float((G - ref).abs().max() / (B.norm(dim=0).max() * r.norm(dim=0).max()))
    print(json.dumps({"profile_gram": True, "D": D, "nB": nB, "s": s, "max_err_rel": err}))
    return 0


STEP_CASES = [
    # (name, constructor, s)
    ("qsun_Lloc13_D65536", lambda pkg, rng: pkg.qsun_hamiltonian(13, 3, 1.0, 0.75, rng=rng), 8),
    ("xxz_L16_D12870", lambda pkg, rng: pkg.xxz_hamiltonian(16, 8, 1.0, 1.0, 3.0, rng=rng), 16),
    ("xxz_L20_D184756", lambda pkg, rng: pkg.xxz_hamiltonian(20, 10, 1.0, 1.0, 5.0, rng=rng), 16),
    ("j1j2_L24_D2704156", lambda pkg, rng: pkg.j1j2_hamiltonian(24, 12, 1.0, 0.5, 1.0, 1.0, 1.0, rng=rng), 16),
]


def step_sweep(large_only=False):
    """Per-step time of the Clenshaw recurrence step across sizes and
    precisions: (t(K=40) - t(K=20)) / 20 from CUDA events on the library's
    stream around pf_filter, so the layout copies and set-up cancel.
    Algorithmic bytes per step 4 * D * s * w; fraction of the measured HBM
    copy peak."""
    import numpy as np
    import torch
    import __graft_entry__ as ge
    pkg = ge.load_package()
    from polfed_b200 import _lib
    pkg.load_library()
    peak, peak_kind = read_peaks()
    st = torch.cuda.ExternalStream(_lib.stream_of(_lib.handle(0)), device="cuda:0")
    cases = STEP_CASES[-1:] if large_only else STEP_CASES
    for name, make, s in cases:
        op = make(pkg, np.random.default_rng(3))
        D = op.dim
        for dt, tdt, w in (("fp64", torch.float64, 8), ("fp32", torch.float32, 4)):
            width, tune = pkg.autotune(op, s, dt)
            X = pkg.col_major(D, s, dtype=tdt)
            X.copy_(torch.rand(D, s, dtype=tdt, device="cuda:0"))
            Y = pkg.col_major(D, s, dtype=tdt)

            def t_filter(K, reps=3):
                c = np.cos(np.arange(K + 1) * 0.7) * 0.05
                pkg.chebyshev_filter(op, Y, X, c, a=2.0 * s, b=0.0)   # warm-up
                best = None
                for _ in range(reps):
                    torch.cuda.synchronize()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(st)
                    pkg.chebyshev_filter(op, Y, X, c, a=2.0 * s, b=0.0)
                    e1.record(st)
                    e1.synchronize()
                    t = e0.elapsed_time(e1) * 1e-3
                    best = t if best is None else min(best, t)
                return best

            per = (t_filter(40) - t_filter(20)) / 20
            alg = 4.0 * D * s * w
            print(json.dumps({"case": name, "D": D, "s": s, "dtype": dt, "width": width,
                              "profile": pkg.step_profile(op, s, dt),
                              "tune_us": {str(k): round(v * 1e3, 2) for k, v in tune.items()},
                              "us_per_step": per * 1e6, "alg_bytes": alg, "achieved_gbs": alg / per / 1e9,
                              "frac": alg / per / 1e9 / peak, "peak": peak, "peak_kind": peak_kind}), flush=True)
            del X, Y
    return 0


def profile_step_large(dtype="fp64", width=None, profile=0):
    """Two order-2 Chebyshev filters on the J1-J2 L=24 Sz=0 operator
    (D = 2,704,156, s = 16) with the autotuned step or the given width and
    profile, inside an NVTX range "filters": a bounded large-D case for ncu
    captures."""
    import numpy as np
    import torch
    import __graft_entry__ as ge
    pkg = ge.load_package()
    name, make, s = STEP_CASES[-1]
    op = make(pkg, np.random.default_rng(3))
    tdt = torch.float64 if dtype == "fp64" else torch.float32
    if width is None:
        width, _ = pkg.autotune(op, s, dtype)
    else:
        pkg.set_step_width(op, s, width, dtype, profile)
    X = pkg.col_major(op.dim, s, dtype=tdt)
    X.copy_(torch.rand(op.dim, s, dtype=tdt, device="cuda:0"))
    Y = pkg.col_major(op.dim, s, dtype=tdt)
    c = np.array([0.1, 0.2, 0.3])
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("filters")
    for _ in range(2):
        pkg.chebyshev_filter(op, Y, X, c, a=2.0 * s, b=0.0)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    print(json.dumps({"profile_step_large": True, "D": op.dim, "s": s, "dtype": dtype, "width": width,
                      "profile": pkg.step_profile(op, s, dtype)}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch", type=int, default=16, help="solves in flight together per step")
    ap.add_argument("--serve", action="store_true", help="run the seeded Poisson request stream instead")
    ap.add_argument("--disorder", action="store_true", help="run the 288-realisation disorder batch instead")
    ap.add_argument("--requests", type=int, default=24)
    ap.add_argument("--rate", type=float, default=0.5, help="served stream arrivals per second")
    ap.add_argument("--workers", type=int, default=4)
    ap.add_argument("--admission", choices=["fifo", "shortest"], default="fifo",
                    help="served stream admission order")
    ap.add_argument("--c3", action="store_true", help="one FP64 solve at the J1-J2 L=24 configuration")
    ap.add_argument("--step-sweep", action="store_true", help="time the Clenshaw step across sizes and precisions")
    ap.add_argument("--large-only", action="store_true", help="with --step-sweep: only the J1-J2 L=24 case")
    ap.add_argument("--profile-step-large", choices=["fp64", "fp32"], default=None,
                    help="two order-2 filters on J1-J2 L=24 (a bounded large-D case for ncu)")
    ap.add_argument("--profile-step", action="store_true",
                    help="only run two short Chebyshev filters on one realisation (a bounded case for ncu)")
    ap.add_argument("--step-width", type=int, default=None,
                    help="with --profile-step / --profile-step-large: this step width (columns per thread) "
                         "instead of the autotuner's")
    ap.add_argument("--step-profile", type=int, default=0, help="with --step-width: the step profile")
    ap.add_argument("--apply-sweep", action="store_true",
                    help="single-vector XXZ H-apply at L=18..24 (the reference's published timings)")
    ap.add_argument("--profile-solve", action="store_true",
                    help="only run two complete solves of the workload, no pool (a bounded case for ncu)")
    ap.add_argument("--profile-kpm", action="store_true",
                    help="only run 40 KPM moments of one 64-probe block (a bounded case for ncu)")
    ap.add_argument("--profile-gram", action="store_true",
                    help="only run the tensor-core Gram product at the final Krylov size (a bounded case for ncu)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local_rank = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.profile_step:
        return profile_step(args.step_width, args.step_profile)
    if args.apply_sweep:
        return apply_sweep()
    if args.profile_solve:
        return profile_solve()
    if args.profile_kpm:
        return profile_kpm()
    if args.profile_gram:
        return profile_gram()
    if args.step_sweep:
        return step_sweep(args.large_only)
    if args.profile_step_large:
        return profile_step_large(args.profile_step_large, args.step_width, args.step_profile)
    if args.c3:
        return run_c3(args, local_rank)
    if args.serve:
        return run_serve(args, local_rank)
    if args.disorder:
        return run_disorder(args, local_rank)
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        return run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
