"""Benchmark: mean-field ADP residual evaluations per second.

One step = one residual evaluation (rho-bar, V0, S0, R_q, R_sigma, R_x and the
FP64 totals) of the plain drop-in workload: periodic hcp Mg 20x15x15
hexagonal cells (9000 Mg) with H on all 18000 tetrahedral sites
(x ~ U[0, 0.3]), positions jittered N(0, 0.02 A), sigma ~ U[0.08, 0.15] A,
T = 400 K; synthetic, seeded.  Neighbour lists are built once before timing
(the reference also builds them once, main-BT-AM.cpp:100-104).

Default arm (--impl btam): the headline `value` is the FP64 drop-in (the
reference's arithmetic type, autotuned kernels); `e2e` times the same FP64
evaluation through the C ABI with host buffers (pinned), including the
host->device state copy and the device->host residual read.  The
FP32-compensated form is reported in its own `fp32c` record (value, e2e,
error against the FP64 form, ratios), beside the plain two-pass FP64 kernel
pair.  Reference arm (--impl reference): the reference's own CPU arithmetic
(oracle/_ref, -Ofast, all host threads) on a bounded sample of the same
workload, extrapolated to one full evaluation and labelled as such.

Multi-GPU (torchrun): every rank evaluates its own replica (independent
systems, no data-path collective); value = evaluations of all ranks / max
rank time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "bt-am_b200"), os.path.join(ROOT, "oracle")]

METRIC = "mean-field ADP residual evals/s & DMD jobs/s, p50/p99, vs plain FP64 on GPU"
WORKLOAD = ("plain drop-in: periodic hcp Mg 20x15x15 hexagonal cells, 9000 Mg + 18000 "
            "tetrahedral H sites (x~U[0,0.3]), jitter N(0,0.02 A), sigma~U[0.08,0.15] A, "
            "T=400 K, seed 2")
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FLOP_PASS1, FLOP_PASS2 = 1000.0, 2000.0  # algorithmic flops per directed active pair
# spline lookups per directed pair: 48 at the 12 pair-rule points (rho, phi,
# u, w), 26 at the 13 triplet points (u, w); the algorithmic flops of each
# pass are attributed to kernels by these lookups
LOOK_PR, LOOK_TRIP = 48.0, 26.0
# Per launch of the FP32C kernels on this workload, from one ncu capture
# (--set full) of the undirected variants (28, 26): DRAM bytes (read +
# write), and L1 global-load sectors (32 bytes each) with the L1 LSU
# data-pipe utilisation
NCU_DRAM_BYTES = {"pass1 pair-rule kernel": 113.1e6, "pass1 site kernel": 65.4e6,
                  "pass2 pair kernel": 253.2e6, "pass2 site kernel": 75.4e6, "totals": 1.5e6}
NCU_L1_SECTORS = {"pass1 pair-rule kernel": 51.73e6, "pass1 site kernel": 54.59e6,
                  "pass2 pair kernel": 28.55e6, "pass2 site kernel": 2.56e6}
NCU_L1_PIPE = {"pass1 pair-rule kernel": 0.91, "pass1 site kernel": 0.71,
               "pass2 pair kernel": 0.69, "pass2 site kernel": 0.31}
# DRAM bytes (read + write) per launch of the FP64 kernels on this workload
# (autotuned variants (26, 30)), from one ncu capture
NCU_DRAM_BYTES_FP64 = {"pass1 pair-rule kernel": 264.1e6, "pass1 site kernel": 107.8e6,
                       "pass2 pair kernel": 486.3e6}
# L1 data-pipe wavefront utilisation of the same FP64 launches (ncu
# l1tex__data_pipe_lsu_wavefronts, share of peak): the binding unit
NCU_L1_PIPE_FP64 = {"pass1 pair-rule kernel": 0.902, "pass1 site kernel": 0.769,
                    "pass2 pair kernel": 0.711}
# shared-memory wavefronts per launch: the pass-2 pair kernel reads its u/w
# spline records from shared memory (its global sectors are the moment and
# pair records only)
NCU_SHARED_WAVEFRONTS = {"pass1 pair-rule kernel": 0.45e6, "pass1 site kernel": 3.35e6,
                         "pass2 pair kernel": 15.30e6, "pass2 site kernel": 1.37e6}


def kernel_flops(undirected):
    """Algorithmic flops per directed active pair of the five kernels of one
    evaluation (pass-1 pair-rule, pass-1 site, pass-2 pair, pass-2 site,
    totals).  Undirected variants: the pair-rule kernel evaluates the pair
    rule of both passes (value and derivative) once per pair for both
    directions, the pass-1 site kernel the triplet points of pass 1, the
    pass-2 pair kernel the triplet points of pass 2; directed variants have
    no pair kernels."""
    tot = LOOK_PR + LOOK_TRIP
    if undirected:
        return [(FLOP_PASS1 + FLOP_PASS2) * LOOK_PR / tot, FLOP_PASS1 * LOOK_TRIP / tot,
                FLOP_PASS2 * LOOK_TRIP / tot, 0.0, 0.0]
    return [0.0, FLOP_PASS1, 0.0, FLOP_PASS2, 0.0]


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, streamed every 50 ms by one
    `nvidia-smi -lms` process from before the warm-up; the summary keeps the
    samples read between begin() and end() (the timed region) and falls back
    to all samples when the region was shorter than the sampling period."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []  # (host time, fields)
        self.t0 = self.t1 = None
        self._proc = None
        self._t = None

    def _read(self):
        for line in self._proc.stdout:
            f = [v.strip() for v in line.strip().split(",")]
            if len(f) == 6:
                self.samples.append((time.perf_counter(), f))

    def start(self):
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self._proc = None
            return self
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()
        return self

    def begin(self):
        self.t0 = time.perf_counter()

    def end(self):
        self.t1 = time.perf_counter()

    def stop(self):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=10)
            except subprocess.TimeoutExpired:
                self._proc.kill()
        if self._t is not None:
            self._t.join(timeout=10)

    def __enter__(self):
        return self.start()

    def __exit__(self, *a):
        self.stop()

    def summary(self):
        inside = [f for t, f in self.samples
                  if self.t0 is not None and self.t1 is not None and self.t0 <= t <= self.t1]
        window = "timed region"
        if not inside:
            inside, window = [f for _, f in self.samples], "whole run (timed region too short)"
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in inside if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in inside if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in inside for k in range(4)
                          if s[2 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(inside), "window": window}


def reduce_max(v, dist, device):
    """v on this rank -> the maximum over ranks (v itself without a process
    group); device: where the reduction tensor lives ("cuda" for NCCL)."""
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(ws, step_ms):
    """Whole-job evaluations per second: every rank evaluates its own replica
    once per step, and a step lasts as long as the slowest rank's."""
    return ws * 1e3 / step_ms


def time_replicas(timed_steps, warmup, steps, barrier, max_over_ranks, ws, sampler=None):
    """The timed region of one form on every rank: `warmup` untimed steps, a
    barrier, `steps` timed steps (timed_steps returns their device times in
    ms) closed by a barrier, then the mean step time's maximum over ranks
    and the whole-job value.  sampler: the clock sampler, started before the
    warm-up and told where the timed region begins and ends."""
    if sampler is not None:
        sampler.start()
    try:
        timed_steps(warmup)
        barrier()
        if sampler is not None:
            sampler.begin()
        ms = timed_steps(steps)
        barrier()
        if sampler is not None:
            sampler.end()
    finally:
        if sampler is not None:
            sampler.stop()
    step_ms = max_over_ranks(float(np.mean(ms)))
    return step_ms, replica_value(ws, step_ms)


def launches_per_eval(shape):
    """Kernel launches of one evaluation with launch variants (v1, v2): pass 1
    (plus the pair-rule kernel when either pass is undirected), pass 2 (pair
    and site kernels when undirected), two totals launches."""
    v1, v2 = shape
    und = bool((v1 | v2) & 16)
    return (2 if und else 1) + (2 if v2 & 16 else 1) + 2


def active_pairs(sys_, offs, idx, owner):
    x = sys_["x"]
    n = len(x)
    xa = x[owner]
    act_i = np.repeat(x >= 5e-4, np.diff(offs[:n + 1]))
    return int(np.sum(act_i & (xa[idx] >= 5e-4)))


def cpu_reference_sample(sys_, threads, budget_s=12.0, seed=0, scale=1, multipole=False,
                         info=None):
    """Times the reference's own arithmetic (oracle/_ref, -Ofast build, on
    `threads` host threads) on a bounded sample of one evaluation (divided
    by `scale`) and extrapolates.  With `multipole`, the -O2 build with
    MULTIPOLE_INTEGRAL and the reference's own -DNUMERICAL_DERIVATIVES=0
    (the oracle's rule 1 when that build is absent).  Returns
    (evals_per_s, description, kind, seconds per evaluation); `info`, when
    given, receives the sample sizes and the wall time the sample took."""
    t_start = time.perf_counter()
    import pyoracle
    ref = pyoracle.reference_multipole() if multipole else pyoracle.reference(fast=True)
    kind = "reference"
    orc = pyoracle.Oracle()
    if ref is None:
        ref, kind = orc, "port"
        if multipole:
            orc.set_rule(1)
    os.environ["BTAM_REF_THREADS"] = str(threads)
    os.environ["BTAM_ORACLE_THREADS"] = str(threads)
    rng = np.random.default_rng(seed)
    n = len(sys_["x"])
    full, nr, owner, image = pyoracle.expand(sys_, orc)
    # neighbour lists of the sampled sites and of their neighbours' owners
    sample_rho = np.sort(rng.choice(n, 1200 // scale, replace=False)).astype(np.int32)
    sample_v0 = sample_rho[::12]
    sample_res = sample_rho[::100]
    need = set(map(int, sample_rho))
    o1, i1 = orc.neighbors(full["q"], query=sample_res)
    for j in i1:
        need.add(int(owner[j]))
    query = np.array(sorted(need), np.int32)
    oq, iq = orc.neighbors(full["q"], query=query)
    counts = np.zeros(len(full["x"]), np.int64)
    counts[query] = np.diff(oq)
    offs = np.zeros(len(full["x"]) + 1, np.int32)
    offs[1:] = np.cumsum(counts)
    idx = np.zeros(offs[-1], np.int32)
    for k, qi in enumerate(query):
        idx[offs[qi]:offs[qi + 1]] = iq[oq[k]:oq[k + 1]]
    t0 = time.perf_counter()
    rho_q = ref.mf_rho(full, offs, idx, query)
    t_rho = (time.perf_counter() - t0) / len(query)
    rho_real = np.zeros(nr)
    rho_real[query] = rho_q
    rho = rho_real[owner]
    t0 = time.perf_counter()
    ref.V0(full, rho, offs, idx, sample_v0)
    t_v0 = (time.perf_counter() - t0) / len(sample_v0)
    # residual of a site: dV0_i/d(q,sigma) and dV0_i/dx over i in {u} U N(u)
    us, is_ = [], []
    for u in sample_res:
        for i in [u, *idx[offs[u]:offs[u + 1]]]:
            us.append(int(u))
            is_.append(int(owner[i]) if int(owner[i]) == int(i) else int(owner[i]))
    t0 = time.perf_counter()
    ref.DV0_pairs(full, rho, offs, idx, us, is_)
    t_res = (time.perf_counter() - t0) / len(sample_res)
    t_full = n * (t_rho + t_v0 + t_res)
    if info is not None:
        info.update({"rho_sites": len(query), "V0_sites": len(sample_v0),
                     "residual_sites": len(sample_res), "total_sites": n,
                     "sample_wall_s": time.perf_counter() - t_start})
    desc = (f"{kind} arithmetic on {threads} threads: rho-bar of {len(query)} sites, V0 of "
            f"{len(sample_v0)} sites, residual assembly (dV0_i/d(q,sigma,x) over i in "
            f"{{u}}+N(u)) of {len(sample_res)} sites, each scaled to all {n} sites")
    return 1.0 / t_full, desc, kind, t_full


def run_reference(args, ws, rank):
    """The reference's own CPU arithmetic on the plain drop-in workload.  A
    full evaluation would take about 25 minutes on 16 host threads (the
    reference's residual assembly is O(N_nb^3) per site), so each step times
    a bounded, seeded sample of sites and extrapolates it to all sites; the
    line says so ("extrapolated", the sample sizes, and the wall time each
    sampled step really took)."""
    if rank != 0:
        return
    from btam import lattice
    sys_ = lattice.config2()
    threads = os.cpu_count() or 1
    vals, walls, info = [], [], {}
    for k in range(args.warmup + args.steps):
        v, desc, kind, _ = cpu_reference_sample(sys_, threads, seed=k, info=info)
        if k >= args.warmup:
            vals.append(v)
            walls.append(info["sample_wall_s"])
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "evals/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 / value, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sites": len(sys_["x"])},
            "extrapolated": True,
            "steps_meaning": ("each step is one seeded site sample of a full evaluation, timed "
                              "and scaled to all sites; ms_per_step is that extrapolated full "
                              "evaluation, sample_wall_ms_per_step the time a step really took"),
            "sample_wall_ms_per_step": 1e3 * float(np.mean(walls)),
            "sampled_sites": {k: info[k] for k in ("rho_sites", "V0_sites", "residual_sites",
                                                   "total_sites")},
            "cpu_baseline": {"value": value, "unit": "evals/s", "cores": threads,
                             "kind": kind, "sample": desc},
            "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def bench_batched(args, tables, flush, max_over_ranks, barrier):
    """The batched workload: 128 hcp Mg-H spheres (radii log-uniform on
    [8, 25] A, T ~ U[300, 600] K, H fraction ~ U[0, 0.5]).  One evaluation of
    all 128 systems as one graph launch (persistent autotuned kernels,
    FP32C), against the plain drop-in: 128 per-system evaluations, each on
    its system's own stream so that they may overlap, in FP32C and FP64."""
    import torch
    import btam
    from btam import lattice

    dicts = lattice.config4()
    systems = []
    for d in dicts:
        S = btam.System(tables, d)
        S.build_neighbors()
        systems.append(S)
    B = btam.Batch(systems)
    info = B.info()
    shapes = B.autotune(btam.FP32C)
    bstream = torch.cuda.ExternalStream(B.stream())

    def graph_steps(k):
        evs = []
        for _ in range(k):
            with torch.cuda.stream(bstream):
                flush.add_(1.0)
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(bstream)
                B.evaluate_async(btam.FP32C)
                b.record(bstream)
            evs.append((a, b))
        B.sync()
        return [a.elapsed_time(b) for a, b in evs]

    def plain_steps(prec, k):
        # device-bracketed host clock: the 128 evaluations run on 128 streams
        ts = []
        for _ in range(k):
            flush.add_(1.0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for S in systems:
                S.evaluate_async(prec)
            for S in systems:
                S.sync()
            torch.cuda.synchronize()
            ts.append((time.perf_counter() - t0) * 1e3)
        return ts

    graph_steps(args.warmup)
    barrier()
    g_ms = max_over_ranks(float(np.mean(graph_steps(min(args.steps, 200)))))
    # wall clock of back-to-back graph launches (launch overhead included)
    barrier()
    t0 = time.perf_counter()
    for _ in range(min(args.steps, 200)):
        B.evaluate_async(btam.FP32C)
    B.sync()
    g_wall = max_over_ranks((time.perf_counter() - t0) * 1e3 / min(args.steps, 200))
    v32 = [S.autotune(btam.FP32C) for S in systems]
    v64 = [S.autotune(btam.FP64) for S in systems]
    out = {}
    k_plain = min(args.steps, 50)
    for prec, name in ((btam.FP32C, "plain_fp32c"), (btam.FP64, "plain_fp64"),
                       (btam.FP64, "plain_fp64_two_pass")):
        if name == "plain_fp64_two_pass":
            for S in systems:
                S.set_variants(btam.FP64, 0, 0)
        plain_steps(prec, args.warmup)
        barrier()
        out[name] = max_over_ranks(float(np.mean(plain_steps(prec, k_plain))))
    ns = info["n_sys"]
    res = {"workload": "128 hcp Mg-H spheres, R log-uniform [8, 25] A, seed 4",
           "systems": ns, "sites": info["n_real"], "directed_pairs": info["n_pairs"],
           "unit": "system evals/s",
           "graph_fp32c": {"ms_per_batch": g_ms, "value": ns * 1e3 / g_ms,
                           "wall_ms_per_batch": g_wall, "kernel_variants": shapes,
                           "launches_per_batch": launches_per_eval(shapes)},
           "plain_fp32c_128_launches": {"ms_per_batch": out["plain_fp32c"],
                                        "value": ns * 1e3 / out["plain_fp32c"],
                                        "kernels": "each system's autotuned variants",
                                        "launches_per_batch": sum(map(launches_per_eval, v32))},
           "plain_fp64_128_launches": {"ms_per_batch": out["plain_fp64"],
                                       "value": ns * 1e3 / out["plain_fp64"],
                                       "kernels": "each system's autotuned variants",
                                       "launches_per_batch": sum(map(launches_per_eval, v64))},
           "plain_fp64_two_pass_128_launches": {
               "ms_per_batch": out["plain_fp64_two_pass"],
               "value": ns * 1e3 / out["plain_fp64_two_pass"],
               "kernels": "plain two-pass pair (directed, variants (0, 0))",
               "launches_per_batch": ns * launches_per_eval((0, 0))}}
    res["graph_fp32c_over_plain_fp64"] = out["plain_fp64"] / g_ms
    res["graph_fp32c_over_plain_fp64_two_pass"] = out["plain_fp64_two_pass"] / g_ms
    B.close()
    for S in systems:
        S.close()
    return res


def bench_nanowire(args, tables):
    """The precision workload: hcp Mg nanowire of radius 30 A along c, 20
    cells long, periodic along the axis, H occupancy x ~ U[0, 0.5] beyond
    20 A and 0.02 inside (seed 3).  1000 master-equation steps (dt = 1e-3)
    with FP32C residuals and FP64 occupancy updates in integer quanta: total
    hydrogen is checked to the quantum and the trajectory against the same
    run with FP64 residuals."""
    import torch
    import btam
    from btam import lattice

    sys_ = lattice.config3()
    h = sys_["species"] == 1
    steps = args.dmd_steps
    out, xs = {}, {}
    # error of the FP32C residual evaluation against the FP64 one on the
    # wire's initial state
    S = btam.System(tables, sys_)
    S.build_neighbors()
    a, b = S.evaluate(btam.FP64), S.evaluate(btam.FP32C)
    S.close()
    err = {"vs": "FP64 form, initial state",
           "energy_rel": abs(b["totals"][0] - a["totals"][0]) / abs(a["totals"][0]),
           "V0_max_abs": float(np.abs(b["V0"] - a["V0"]).max()),
           "Rq_max_abs": float(np.abs(b["Rq"] - a["Rq"]).max()),
           "Rs_max_abs": float(np.abs(b["Rs"] - a["Rs"]).max()),
           "Rx_max_abs": float(np.abs(b["Rx"] - a["Rx"]).max()),
           "sum_Rq_fp64": float(np.abs(a["Rq"].sum(axis=0)).max()),
           "tolerance": "energy <= 1e-6 relative, residuals <= 1e-5 eV/A"}
    for prec, name in ((btam.FP32C, "fp32c"), (btam.FP64, "fp64")):
        S = btam.System(tables, sys_)
        S.build_neighbors()
        S.autotune(prec)
        S.dmd_setup()
        total0 = S.dmd_step(0, prec, dt=1e-3)
        S.dmd_step(3, prec, dt=0.0)  # warm-up steps that move nothing (dt = 0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        total = S.dmd_step(steps, prec, dt=1e-3)
        t = time.perf_counter() - t0
        x, X, mu = S.dmd_occupancy()
        xs[name] = x
        out[name] = {"steps_per_s": steps / t, "ms_per_step": t * 1e3 / steps,
                     "total_h_conserved": bool(total == total0),
                     "clipped_edge_moves": S.dmd_clip_count(),
                     "x_min": float(x[h].min()), "x_max": float(x[h].max())}
        S.close()
    # the same FP32C run with step control (sub-steps where a move would be
    # cut to its room or a site would change by more than 0.05)
    S = btam.System(tables, sys_)
    S.build_neighbors()
    S.autotune(btam.FP32C)
    S.dmd_setup()
    total0 = S.dmd_step(0, btam.FP32C, dt=1e-3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    total, st = S.dmd_step_ctl(steps, btam.FP32C, dt=1e-3)
    t = time.perf_counter() - t0
    x, X, mu = S.dmd_occupancy()
    out["fp32c_step_control"] = dict(st, steps_per_s=steps / t, ms_per_step=t * 1e3 / steps,
                                     total_h_conserved=bool(total == total0),
                                     max_abs_dx_vs_fixed_steps=float(
                                         np.abs(x - xs["fp32c"]).max()))
    S.close()
    nr = len(sys_["x"])
    return {"workload": "hcp Mg nanowire R = 30 A along c, 20 cells, periodic along the axis, "
                        "x ~ U[0, 0.5] beyond 20 A, 0.02 inside, seed 3",
            "sites": nr, "h_sites": int(h.sum()), "steps": steps, "dt": 1e-3,
            "fp32c_error": err,
            "timing": "host clock around one call of all steps (device-resident loop)",
            **out,
            "fp32c_vs_fp64_max_abs_dx": float(np.abs(xs["fp32c"] - xs["fp64"]).max())}


def bench_bulk_stretch(args, tables, cpu_budget_s=6.0):
    """The reference's one compiled solver, the bulk stretch relaxation
    (mechanical_relaxation_bulk), on the plain drop-in workload: Newton on
    the diagonal stretch F with the non-mean-field stress residual
    Y = sum_u diag(dV_u/dF) / V0 at fixed x and neighbour lists, from F = 1
    to |Y| <= 1e-12.  Each residual is one device evaluation of rho and
    dV_u/dF over all sites.  The reference's arithmetic for one residual
    (evaluate_rho_i and evaluate_DV_i_dF_MgHx, oracle/_ref, all host
    threads) is timed on a sample of sites and scaled to all sites."""
    import torch
    import btam
    import pyoracle
    from btam import lattice

    sys_ = lattice.config2()
    runs = []
    for k in range(2):  # the first run warms up (allocations, module load)
        S = btam.System(tables, sys_)
        S.build_neighbors()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        F, info = S.relax_stretch(atol=1e-12, rtol=1e-10, max_iter=20)
        runs.append((time.perf_counter() - t0, F, info))
        S.close()
    t, F, info = runs[-1]
    out = {"workload": WORKLOAD, "sites": len(sys_["x"]),
           "solver": "Newton, forward-difference Jacobian (3 residuals), backtracking",
           "F": [float(f) for f in F], "iterations": info["iterations"],
           "residual_evaluations": info["evaluations"], "final_norm": info["norm"],
           "status": info["status"], "ms_total": t * 1e3,
           "ms_per_residual": t * 1e3 / max(info["evaluations"], 1),
           "timing": "host clock around the call (each residual ends in a 96-byte read)"}
    # the solver the reference's main program configures for this relaxation:
    # N-GMRES(m = 3) with the critical-point line search
    S = btam.System(tables, sys_)
    S.build_neighbors()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    Fg, ig = S.relax_stretch_ngmres(m=3, atol=1e-12, rtol=1e-10, max_iter=60)
    tg = time.perf_counter() - t0
    S.close()
    out["ngmres_m3_cp"] = {"F": [float(f) for f in Fg], "iterations": ig["iterations"],
                           "residual_evaluations": ig["evaluations"], "final_norm": ig["norm"],
                           "status": ig["status"], "ms_total": tg * 1e3,
                           "max_abs_F_vs_newton": float(np.max(np.abs(Fg - F)))}
    if not args.no_cpu:
        ref = pyoracle.reference(fast=True)
        kind = "reference"
        orc = pyoracle.Oracle()
        if ref is None:
            ref, kind = orc, "port"
        threads = os.cpu_count() or 1
        os.environ["BTAM_REF_THREADS"] = str(threads)
        os.environ["BTAM_ORACLE_THREADS"] = str(threads)
        full, nr, owner, image = pyoracle.expand(sys_, orc)
        rng = np.random.default_rng(7)
        sample = np.sort(rng.choice(nr, 400, replace=False)).astype(np.int32)
        need = np.unique(np.concatenate([sample, owner[orc.neighbors(full["q"],
                                                                     query=sample)[1]]]))
        need = need.astype(np.int32)
        oq, iq = orc.neighbors(full["q"], query=need)
        counts = np.zeros(len(full["x"]), np.int64)
        counts[need] = np.diff(oq)
        offs = np.zeros(len(full["x"]) + 1, np.int32)
        offs[1:] = np.cumsum(counts)
        idx = np.zeros(offs[-1], np.int32)
        for k, qi in enumerate(need):
            idx[offs[qi]:offs[qi + 1]] = iq[oq[k]:oq[k + 1]]
        t0 = time.perf_counter()
        rho_n = ref.rho_nmf(full, offs, idx, need)
        t_rho = (time.perf_counter() - t0) / len(need)
        rho = np.zeros(nr)
        rho[need] = rho_n
        per = []
        for chunk in np.array_split(sample, 8):
            t0 = time.perf_counter()
            ref.pt_DV_dF(full, full["q"], rho[owner], offs, idx, chunk)
            per.append((time.perf_counter() - t0) / len(chunk))
            if sum(per) * len(chunk) > cpu_budget_s:
                break
        t_res = nr * (t_rho + float(np.mean(per)))
        out["cpu_reference"] = {
            "s_per_residual": t_res, "threads": threads, "kind": kind,
            "sample": f"evaluate_rho_i of {len(need)} sites and evaluate_DV_i_dF_MgHx of "
                      f"{len(per) * (len(sample) // 8)} sites, scaled to all {nr} sites"}
        out["gpu_over_cpu_per_residual"] = t_res / (out["ms_per_residual"] * 1e-3)
    return out


def bench_config1(args, tables):
    """The CPU-runnable workload end to end: periodic 5x5x5 hexagonal cells
    (250 Mg, 100 H at x ~ U[0, 0.1]), one relaxation of (q, sigma) to
    |R| <= 1e-8 (the Newton option; L-BFGS and the reference's configured
    N-GMRES(3) with the critical-point line search beside it), then 10
    master-equation steps with dt = 1e-3, all in FP64."""
    import torch
    import btam
    from btam import lattice

    sys_ = lattice.config1()
    out = {"workload": "periodic 5x5x5 hexagonal cells, 250 Mg + 100 H (x ~ U[0, 0.1]), "
                       "relaxation to |R| <= 1e-8 then 10 master-equation steps (dt 1e-3), FP64",
           "sites": len(sys_["x"])}
    for name in ("newton", "lbfgs", "ngmres_m3_cp"):
        S = btam.System(tables, sys_)
        S.build_neighbors()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if name == "newton":
            info = S.relax_newton(tol=1e-8, max_newton=100, max_cg=300)
        elif name == "lbfgs":
            info = S.relax(mode=btam.RELAX_FP64, tol=1e-8, max_iter=2000)
        else:  # the reference's SNES options: N-GMRES(3), critical-point line search
            info = S.relax(mode=btam.RELAX_NGMRES, tol=1e-8, max_iter=20000, m=3)
        t1 = time.perf_counter()
        S.dmd_setup()
        S.dmd_step(10, btam.FP64, dt=1e-3)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        out[name] = {"relax_ms": (t1 - t0) * 1e3, "relax_evaluations": info["evaluations"],
                     "relax_norm": info["norm"], "converged": info["status"] == 1,
                     "objective": info["objective"],
                     "dmd_10_steps_ms": (t2 - t1) * 1e3, "total_ms": (t2 - t0) * 1e3}
        S.close()
    out["timing"] = "host clock around each call (device-resident loops)"
    return out


def bench_multipole(args, tables):
    """The reference's other mean-field rule (MULTIPOLE_INTEGRAL) on the
    plain drop-in workload: rho-bar + V0 and the residuals, FP64, under the
    finite-difference Hessians of the reference's build flags (rule 1) and
    the analytic ones (rule 2); host clock around each call (allocation and
    the result copies included).  Beside it, the reference built with the
    rule, timed on a bounded sample on all host threads."""
    import torch
    import btam
    from btam import lattice

    sys_ = lattice.config2()
    S = btam.System(tables, sys_)
    S.build_neighbors()
    out = {"workload": WORKLOAD + ", multipole rule", "sites": len(sys_["x"])}
    for rule, name in ((btam.MP_FD, "rule_fd_hessians"), (btam.MP_ANALYTIC, "rule_analytic")):
        S.mf_eval_multipole(rule)  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, _, E = S.mf_eval_multipole(rule)
        t1 = time.perf_counter()
        S.mf_residuals_multipole(rule)
        t2 = time.perf_counter()
        out[name] = {"energy": E, "rho_V0_ms": (t1 - t0) * 1e3, "residuals_ms": (t2 - t1) * 1e3,
                     "evaluation_ms": (t2 - t0) * 1e3}
    S.close()
    if not args.no_cpu and int(os.environ.get("RANK", "0")) == 0:
        threads = os.cpu_count() or 1
        _, desc, kind, t_full = cpu_reference_sample(sys_, threads, seed=2, scale=4,
                                                     multipole=True)
        out["cpu_reference"] = {"s_per_evaluation": t_full, "threads": threads, "kind": kind,
                                "build": "-O2 -DMULTIPOLE_INTEGRAL -DNUMERICAL_DERIVATIVES=0",
                                "sample": desc}
        out["gpu_over_cpu_rule_fd"] = t_full / (out["rule_fd_hessians"]["evaluation_ms"] * 1e-3)
    out["timing"] = "host clock around each call"
    return out


def bench_serving(args, tables):
    """The served workload: a seeded Poisson stream of relaxation (L-BFGS to
    |R| <= 1e-5 or 100 iterations) and 100-step master-equation jobs, half
    each, on periodic cubes of 250-60 000 Mg, nanowires and spheres, FP32C,
    served with continuous batching (every running job's evaluations merged
    into one batched launch per round, 32 job slots, memory-budget
    admission).  Two runs of the whole stream (--serve-jobs, 1000 by
    default): at 200 jobs/s (more than the server sustains: its capacity)
    and at 70 % of that capacity (steady state: latency without a growing
    queue).  The plain drop-in baselines, one job at a time in FP64 with the
    plain two-pass kernel pair and with the autotuned undirected kernels,
    run on the stream's first --plain-jobs jobs, and the served form runs on
    the same jobs for a like-for-like ratio.  Latency = completion -
    arrival, queueing included; a residual evaluation is one evaluation of
    one job's system."""
    import threading
    import btam
    from btam import lattice

    jobs = lattice.config5(n_jobs=args.serve_jobs)

    def serve(stream, workers, fp64, plain=False):
        srv = btam.Server(tables, workers=workers)
        srv.wait(srv.submit(lattice.periodic_cube(300, seed=1), kind=btam.JOB_EVAL))  # warm-up
        ids = [None] * len(stream)
        t0 = time.perf_counter()

        def feeder():
            for k, (t, sysd, kind) in enumerate(stream):
                d = t - (time.perf_counter() - t0)
                if d > 0:
                    time.sleep(d)
                if kind == "relax":
                    ids[k] = srv.submit(sysd, kind=btam.JOB_RELAX, tol=1e-5, max_iter=100,
                                        mode=btam.RELAX_FP64 if fp64 else btam.RELAX_FP32C,
                                        plain=plain)
                else:
                    ids[k] = srv.submit(sysd, kind=btam.JOB_DMD, nsteps=100,
                                        precision=btam.FP64 if fp64 else btam.FP32C,
                                        plain=plain)

        th = threading.Thread(target=feeder)
        th.start()
        th.join()
        res = [srv.wait(i) for i in ids]
        bs = srv.batch_stats()
        srv.close()
        lat = np.array([r["t_end"] - r["t_submit"] for r in res])
        span = max(r["t_end"] for r in res) - min(r["t_submit"] for r in res)
        evals = int(sum(r["evaluations"] if r["kind"] == btam.JOB_RELAX else r["iterations"]
                        for r in res))
        out = {"jobs": len(stream), "jobs_per_s": len(stream) / span,
               "residual_evals_per_s": evals / span,
               "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
               "makespan_s": span, "residual_evaluations": evals}
        if not plain and workers > 1:
            out["batching"] = dict(bs, evals_per_round=bs["evaluations"] / max(bs["rounds"], 1))
        return out

    slots = 32
    overload = serve(jobs, slots, False)
    rate = 0.7 * overload["jobs_per_s"]
    steady_stream = [(t * 200.0 / rate, sysd, kind) for t, sysd, kind in jobs]
    steady = serve(steady_stream, slots, False)
    sample = jobs[:args.plain_jobs]
    served_sample = serve(sample, slots, False)
    plain = serve(sample, 1, True, plain=True)
    fp64_one = serve(sample, 1, True)
    sizes = np.array([len(s["x"]) for _, s, _ in jobs])
    res = {"workload": f"{len(jobs)} jobs, Poisson arrivals (seed 5): relaxation (|R| <= 1e-5 or "
                       "100 L-BFGS iterations) and 100-step master equation, half each, on "
                       "periodic cubes 250-60000 Mg, nanowires, spheres",
           "sites_total": int(sizes.sum()), "sites_max": int(sizes.max()),
           "served_fp32c_200_per_s": dict(overload, arrival_rate=200.0, slots=slots),
           "served_fp32c_steady": dict(steady, arrival_rate=rate, slots=slots),
           "baseline_sample": f"the stream's first {len(sample)} jobs",
           "served_fp32c_sample": dict(served_sample, slots=slots),
           "plain_fp64_one_at_a_time": dict(plain, kernels="plain two-pass pair, variants (0, 0)"),
           "fp64_one_at_a_time": dict(fp64_one, kernels="undirected kernels, one job at a time"),
           "served_over_plain_jobs_per_s": served_sample["jobs_per_s"] / plain["jobs_per_s"],
           "served_over_fp64_one_at_a_time":
               served_sample["jobs_per_s"] / fp64_one["jobs_per_s"],
           "served_over_plain_evals_per_s":
               served_sample["residual_evals_per_s"] / plain["residual_evals_per_s"]}
    res["summary"] = {"served_jobs_per_s": overload["jobs_per_s"],
                      "steady_rate": rate, "steady_p50_s": steady["p50_s"],
                      "steady_p99_s": steady["p99_s"],
                      "over_plain_fp64": res["served_over_plain_jobs_per_s"],
                      "over_fp64_one_at_a_time": res["served_over_fp64_one_at_a_time"],
                      "evals_per_round": overload.get("batching", {}).get("evals_per_round")}
    return res


def run_btam(args, ws, rank, local):
    import torch
    import btam
    from btam import lattice

    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    sys_ = lattice.config2()
    n = len(sys_["x"])
    tables = btam.Tables()
    S = btam.System(tables, sys_)
    S.build_neighbors()
    nr, ng, npairs = S.info()
    offs, idx = S.neighbors()
    owner = np.concatenate([np.arange(n), S.ghosts()[1]]).astype(np.int64)
    P = active_pairs(sys_, offs, idx, owner)
    # kernel block shapes picked by the library's autotuner (setup, untimed)
    shapes = {"fp32c": S.autotune(btam.FP32C), "fp64": S.autotune(btam.FP64)}
    stream = torch.cuda.ExternalStream(S.stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed_steps(prec, k):
        evs = []
        for _ in range(k):
            with torch.cuda.stream(stream):
                flush.add_(1.0)  # evict the working set from L2 between steps
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                S.evaluate_async(prec)
                b.record(stream)
            evs.append((a, b))
        S.sync()
        return [a.elapsed_time(b) for a, b in evs]

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v):
        return reduce_max(v, dist, "cuda")

    results = {}
    clocks = None
    # the headline first: the FP64 drop-in (the reference's arithmetic type),
    # then the FP32-compensated form and the plain two-pass FP64 kernel pair
    for prec, name in ((btam.FP64, "fp64"), (btam.FP32C, "fp32c"), (btam.FP64, "fp64_two_pass")):
        if name == "fp64_two_pass":
            # the plain two-pass kernel pair: one warp per site in each pass,
            # every directed pair evaluated by its own site, default shapes
            S.set_variants(btam.FP64, 0, 0)
        cs = ClockSampler(local)
        step_ms, value = time_replicas(lambda k: timed_steps(prec, k), args.warmup, args.steps,
                                       barrier, max_over_ranks, ws, cs)
        if name == "fp64":
            clocks = cs.summary()
        results[name] = dict(ms=step_ms, value=value)
    S.set_variants(btam.FP64, *shapes["fp64"])
    # per-kernel times for the rooflines (median of 7 profiled evaluations)
    prof64 = np.median(np.array([S.profile(btam.FP64) for _ in range(7)]), axis=0)
    prof32 = np.median(np.array([S.profile(btam.FP32C) for _ in range(7)]), axis=0)
    fp32_peak = btam.probe_fma_peak(False, 0.5)
    fp64_peak = btam.probe_fma_peak(True, 0.5)
    gather_peak = btam.probe_gather_peak(tables, 0.5)
    names = ["pass1 pair-rule kernel", "pass1 site kernel", "pass2 pair kernel",
             "pass2 site kernel", "totals"]
    eval_flops = (FLOP_PASS1 + FLOP_PASS2) * P

    def kernel_roofline(prof, shape, peak, form, ncu_bytes):
        und = bool((shape[0] | shape[1]) & 16)
        flops = kernel_flops(und)
        dom = int(np.argmax(prof))
        achieved = flops[dom] * P / (prof[dom] * 1e-3) / 1e12
        return {"bound": form, "kernel": f"{names[dom]} ({'FP64' if form == 'fp64' else 'FP32C'})",
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": ncu_bytes.get(names[dom]) if und else None,
                "traffic_unit": "bytes per launch (ncu dram read + write)",
                "peak_source": f"measured live: btam_probe_fma_peak {form.upper()} FMA loop on "
                               "all SMs (no vector-FMA figure in the measured peaks file)",
                "flops_per_launch": flops[dom] * P,
                "kernel_ms": dict(zip(names, map(float, prof))),
                "kernel_flops_per_directed_pair": dict(zip(names, flops))}, und

    roofline, _ = kernel_roofline(prof64, shapes["fp64"], fp64_peak, "fp64", NCU_DRAM_BYTES_FP64)
    eval64 = eval_flops / (results["fp64"]["ms"] * 1e-3) / 1e12
    roofline["evaluation"] = {"flops": eval_flops, "achieved": eval64, "frac": eval64 / fp64_peak,
                              "dram_bytes_ncu": sum(NCU_DRAM_BYTES_FP64.values()) or None,
                              "dram_bytes_kernels": "pair-rule, pass-1 site and pass-2 pair kernels",
                              "algorithmic_bytes": 81 * n + 4 * P}
    roofline["l1_data_pipe"] = {
        "bound": "L1 data pipe (random 32-byte halves of the 64-byte FP64 spline records)",
        "ncu_wavefront_frac": NCU_L1_PIPE_FP64,
        "source": "one ncu capture of the autotuned FP64 shapes (26, 30) on this workload"}
    roof32, und32 = kernel_roofline(prof32, shapes["fp32c"], fp32_peak, "fp32", NCU_DRAM_BYTES)
    eval32 = eval_flops / (results["fp32c"]["ms"] * 1e-3) / 1e12
    roof32["evaluation"] = {"flops": eval_flops, "achieved": eval32, "frac": eval32 / fp32_peak,
                            "dram_bytes_ncu": sum(NCU_DRAM_BYTES.values()),
                            "algorithmic_bytes": 45 * n + 4 * P}
    roof32["l1_gather"] = {
        "bound": "L1 data pipe (random 32-byte record gathers)",
        "peak_gbs": gather_peak,
        "peak_source": "measured live: btam_probe_gather_peak, random 32-byte "
                       "spline-record gathers on all SMs",
        "kernels": {k: {"sector_gbs": NCU_L1_SECTORS[k] * 32 / (prof32[i] * 1e-3) / 1e9,
                        "frac": NCU_L1_SECTORS[k] * 32 / (prof32[i] * 1e-3) / 1e9 / gather_peak,
                        "ncu_data_pipe_frac": NCU_L1_PIPE[k],
                        "ncu_shared_wavefronts": NCU_SHARED_WAVEFRONTS[k]}
                    for i, k in enumerate(names) if k in NCU_L1_SECTORS} if und32 else None,
        "sectors_source": "L1 global-load sectors per launch from one ncu capture"}
    # e2e through the C ABI with pinned host buffers
    qh = torch.from_numpy(sys_["q"]).pin_memory().numpy()
    sh = torch.from_numpy(sys_["sigma"]).pin_memory().numpy()
    xh = torch.from_numpy(sys_["x"]).pin_memory().numpy()
    outs = {k: torch.zeros(sh_, dtype=torch.float64).pin_memory().numpy()
            for k, sh_ in (("Rq", (n, 3)), ("Rs", (n,)), ("Rx", (n,)), ("totals", (4,)))}
    # a second set of result buffers for the pipelined calls (two in flight)
    outs2 = {k: torch.zeros(v.shape, dtype=torch.float64).pin_memory().numpy()
             for k, v in outs.items()}
    lib = btam.lib()

    def e2e_step(prec):
        # new (q, sigma, x) from host buffers, evaluation, residuals back to
        # host buffers: one C-ABI call
        code = lib.btam_mf_eval_state(S.handle, prec, btam._d(qh), btam._d(sh),
                                      btam._d(xh), None, None, None, btam._d(outs["Rq"]),
                                      btam._d(outs["Rs"]), btam._d(outs["Rx"]),
                                      btam._d(outs["totals"]))
        if code:
            raise btam.BtamError(code, "btam_mf_eval_state")

    def e2e_pipelined(prec, k):
        # the same copies and evaluation through btam_mf_eval_state_async:
        # step k's results go to the host while step k + 1 evaluates; every
        # step is waited for inside the timed region
        tickets = []
        for i in range(k):
            o = outs if i % 2 == 0 else outs2
            tk = ctypes.c_longlong()
            code = lib.btam_mf_eval_state_async(
                S.handle, prec, btam._d(qh), btam._d(sh), btam._d(xh), None, None, None,
                btam._d(o["Rq"]), btam._d(o["Rs"]), btam._d(o["Rx"]), btam._d(o["totals"]),
                ctypes.byref(tk))
            if code:
                raise btam.BtamError(code, "btam_mf_eval_state_async")
            tickets.append(tk.value)
            if i >= 1:
                code = lib.btam_mf_eval_state_wait(S.handle, tickets[i - 1])
                if code:
                    raise btam.BtamError(code, "btam_mf_eval_state_wait")
        if tickets:
            code = lib.btam_mf_eval_state_wait(S.handle, tickets[-1])
            if code:
                raise btam.BtamError(code, "btam_mf_eval_state_wait")

    def e2e_ms(prec, pipelined):
        if pipelined:
            e2e_pipelined(prec, args.warmup)
        else:
            for _ in range(args.warmup):
                e2e_step(prec)
        barrier()
        t0 = time.perf_counter()
        if pipelined:
            e2e_pipelined(prec, args.steps)
        else:
            for _ in range(args.steps):
                e2e_step(prec)
        barrier()
        return max_over_ranks((time.perf_counter() - t0) * 1e3 / args.steps)

    e2e64_one = e2e_ms(btam.FP64, False)
    e2e32_one = e2e_ms(btam.FP32C, False)
    e2e64 = e2e_ms(btam.FP64, True)
    e2e32 = e2e_ms(btam.FP32C, True)
    h2d = n * (24 + 8 + 8)
    d2h = n * (24 + 8 + 8) + 32
    # error of the FP32C form against the FP64 form (the FP64 form agrees with
    # the FP64 oracle to 1e-10 relative on the parity systems)
    S.set_state(q=sys_["q"], sigma=sys_["sigma"], x=sys_["x"])
    o32, o64 = S.evaluate(btam.FP32C), S.evaluate(btam.FP64)
    precision = {"vs": "FP64 form of the same system",
                 "energy_rel": abs(o32["totals"][0] - o64["totals"][0]) / abs(o64["totals"][0]),
                 "V0_max_abs": float(np.abs(o32["V0"] - o64["V0"]).max()),
                 "Rq_max_abs": float(np.abs(o32["Rq"] - o64["Rq"]).max()),
                 "Rs_max_abs": float(np.abs(o32["Rs"] - o64["Rs"]).max()),
                 "Rx_max_abs": float(np.abs(o32["Rx"] - o64["Rx"]).max()),
                 "tolerance": "energy <= 1e-6 relative, residuals <= 1e-5 eV/A"}
    batched = None if args.no_batch else bench_batched(args, tables, flush, max_over_ranks,
                                                        barrier)
    serving = None if args.no_serve else bench_serving(args, tables)
    nanowire = None if args.no_wire else bench_nanowire(args, tables)
    stretch = None if args.no_stretch else bench_bulk_stretch(args, tables)
    config1 = None if args.no_stretch else bench_config1(args, tables)
    multipole = None if args.no_multipole else bench_multipole(args, tables)
    cpu = None
    if rank == 0 and not args.no_cpu:
        v, desc, kind, _ = cpu_reference_sample(sys_, os.cpu_count() or 1)
        cpu = {"value": v, "unit": "evals/s", "cores": os.cpu_count() or 1, "kind": kind,
               "sample": desc, "extrapolated": True}
        # the same arithmetic on one thread, on a quarter of the sample
        v1, desc1, _, _ = cpu_reference_sample(sys_, 1, seed=1, scale=4)
        cpu["single_thread"] = {"value": v1, "unit": "evals/s", "cores": 1, "sample": desc1}
    if rank == 0:
        r64, r32, r2p = results["fp64"], results["fp32c"], results["fp64_two_pass"]
        fp32c = {"value": r32["value"], "unit": "evals/s", "ms_per_step": r32["ms"],
                 "kernels": "autotuned variants " + str(shapes["fp32c"]),
                 "e2e": {"value": ws * 1e3 / e2e32, "unit": "evals/s", "ms_per_step": e2e32,
                         "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                         "one_call": {"value": ws * 1e3 / e2e32_one, "ms_per_step": e2e32_one}},
                 "error_vs_fp64": precision, "roofline": roof32,
                 "over_fp64_drop_in": r32["value"] / r64["value"],
                 "over_fp64_two_pass": r32["value"] / r2p["value"],
                 "e2e_over_fp64_e2e": e2e64 / e2e32}
        summary = {"fp64_evals_per_s": r64["value"], "fp64_e2e_evals_per_s": ws * 1e3 / e2e64,
                   "fp32c_evals_per_s": r32["value"], "fp32c_e2e_evals_per_s": ws * 1e3 / e2e32,
                   "fp32c_energy_rel_err": precision["energy_rel"],
                   "fp32c_max_residual_err": max(precision["Rq_max_abs"], precision["Rs_max_abs"],
                                                 precision["Rx_max_abs"]),
                   "fp32c_over_fp64_drop_in": fp32c["over_fp64_drop_in"],
                   "fp32c_over_fp64_two_pass": fp32c["over_fp64_two_pass"]}
        if batched:
            summary["batched_system_evals_per_s"] = batched["graph_fp32c"]["value"]
            summary["batched_over_fp64_autotuned_launches"] = batched["graph_fp32c_over_plain_fp64"]
            summary["batched_over_fp64_two_pass_launches"] = \
                batched["graph_fp32c_over_plain_fp64_two_pass"]
        if serving:
            summary["serving"] = serving.get("summary")
        line = {"metric": METRIC, "value": r64["value"], "unit": "evals/s",
                "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": r64["ms"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": {"workload": WORKLOAD, "sites": n},
                "setup": {"images": ng, "directed_active_pairs": P, "precision": "fp64",
                          "l2": "flushed between steps (256 MiB write, outside step events)",
                          "parallelism": f"{ws} independent replica(s), no collective",
                          "kernel_shapes": shapes},
                "roofline": roofline, "cpu_baseline": cpu,
                "e2e": {"value": ws * 1e3 / e2e64, "unit": "evals/s",
                        "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "ms_per_step": e2e64,
                        "call": "btam_mf_eval_state_async(BTAM_FP64) + _wait per step, pinned "
                                "host buffers, two calls in flight (each step's inputs copied "
                                "in and results copied out inside the timed region)",
                        "one_call": {"value": ws * 1e3 / e2e64_one, "ms_per_step": e2e64_one,
                                     "call": "btam_mf_eval_state(BTAM_FP64), one wait per step"}},
                "gpu_launches": launches_per_eval(shapes["fp64"]) * args.steps,
                "clocks": clocks,
                "fp64_two_pass": {"value": r2p["value"], "unit": "evals/s",
                                  "ms_per_step": r2p["ms"],
                                  "kernels": "plain two-pass pair (directed, variants (0, 0))"},
                "fp32c": fp32c,
                "batched": batched, "serving": serving,
                "precision_nanowire": nanowire, "bulk_stretch": stretch,
                "config1_workflow": config1, "multipole": multipole,
                # last, so that it is inside any tail of the line
                "summary": summary}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="btam", choices=["btam", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched workload")
    ap.add_argument("--no-serve", action="store_true", help="skip the served workload")
    ap.add_argument("--serve-jobs", type=int, default=1000, help="jobs in the served stream")
    ap.add_argument("--plain-jobs", type=int, default=128,
                    help="jobs of the stream the one-at-a-time baselines run")
    ap.add_argument("--no-wire", action="store_true", help="skip the nanowire DMD workload")
    ap.add_argument("--no-stretch", action="store_true",
                    help="skip the bulk stretch relaxation and config-1 workflow workloads")
    ap.add_argument("--no-multipole", action="store_true",
                    help="skip the multipole-rule workload")
    ap.add_argument("--dmd-steps", type=int, default=1000,
                    help="master-equation steps of the nanowire workload")
    args = ap.parse_args()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, ws, rank)
    else:
        run_btam(args, ws, rank, local)


if __name__ == "__main__":
    main()
