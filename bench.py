#!/usr/bin/env python
"""Benchmark: FP64 Gauss-Radau N-body propagation throughput (object-years/s) on B200.

Workload (default): the batched uneven N-body configuration -- 1,000,000 seeded states
(90% main belt, 10% NEO; 5% carry JPL comet non-gravitational A1/A2) each propagated to its
own target epoch drawn uniform in +-5 years, under the Sun, eight planets and the Moon read
from a seeded synthetic SPK type-2 ephemeris (degree-13 Chebyshev records).  One step = one
propagation of the whole population by the node-parallel persistent kernel (the ordering
kernels and the node kernel replayed from a captured CUDA graph).  ``value`` is
device-resident throughput (inputs already in HBM, CUDA-event timed, L2 flushed between
steps); ``e2e`` is the same through the public C ABI with pinned host buffers
(host->device and device->host copies inside the timed region).  The same line carries the
plain form (one thread per object, one launch per call) timed on the same inputs, the
reverse-mode gradient cost on the differentiation workload, the CPU oracle on a seeded 1%
subsample, and parity against the oracle on that subsample with objects that pass within
0.01 AU of a planet reported separately.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl kete_b200|reference]
                  [--workload nbody_mixed_1m|nbody_mba_10k|...]

With N > 1 (torchrun) every rank propagates its own population (weak scaling, no data
exchange); the time is the maximum over ranks.  ``--impl reference`` times the CPU
restatement of kete's path (the oracle) on all host cores on the same workload.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Radau object-years/s at ≤1e-9 AU vs CPU ref: batched+adjoint vs plain on B200"
UNIT = "object-years/s"
EPOCH = 2460000.5
SPAN = 365.25

# algorithmic FP64 flops (add/sub/mul = 1, fma = 2, div = 1, sqrt = 1) the force model and
# the Radau step need, term by term, for the PLANETS force list with 14-coefficient Chebyshev
# records.  The records of one evaluation time: positions and velocities of the Sun and
# Jupiter (2 x 223: their velocities enter the relativistic and non-gravitational terms),
# positions of the other 9 records (9 x 108), Earth/Moon + barycentre (6) -- 1424 in all.
# The force terms at given body positions: 10 Newtonian terms (10 x 19) with 2 relative
# velocities (6), relativistic terms (2 x 34), solar/Jovian J2 (2 x 42), Earth J2 (30) --
# 378 in all.
FLOPS_RECORDS = 1424
FLOPS_FORCE_TERMS = 378
FLOPS_PER_EVAL = FLOPS_RECORDS + FLOPS_FORCE_TERMS  # 1802: one evaluation from scratch
FLOPS_ITER_ALGEBRA = 1201  # predictors (840), node times (14), g (168), b (168), test (11)
FLOPS_PER_ITER = 7 * FLOPS_PER_EVAL + FLOPS_ITER_ALGEBRA  # reference: records every node eval
FLOPS_PER_STEP = 120       # state update + step-size control


def flop_models(steps, iters, exact):
    """FP64 flops of one propagation from the kernel's own counters (accepted steps,
    corrector iterations, exact evaluations), in two models:
    - "work": what the cached algorithm needs -- the records at the 8 distinct times of a step
      (7 nodes + the step end) and once per object at its start, plus the force terms of
      every node and exact evaluation and the Radau algebra;
    - "reference": kete's own count, which evaluates the records at every node evaluation of
      every corrector iteration (radau.rs:249-291 calls spk_accel per node)."""
    starts = max(exact - steps, 0)
    work = ((8 * steps + starts) * FLOPS_RECORDS +
            iters * (7 * FLOPS_FORCE_TERMS + FLOPS_ITER_ALGEBRA) +
            exact * FLOPS_FORCE_TERMS + steps * FLOPS_PER_STEP)
    reference = iters * FLOPS_PER_ITER + exact * FLOPS_PER_EVAL + steps * FLOPS_PER_STEP
    return work, reference


# DRAM traffic of the node kernel from ncu captures (dram__bytes_read.sum +
# dram__bytes_write.sum, one launch), per object, keyed by workload and launch configuration
NODE_TRAFFIC = {
    ("nbody_mixed_1m", 7, 1): {"bytes_per_object": (13_601_536 + 882_944) / 100_000,
                               "fp64_pipe": 0.217,
                               "captured": "one launch on a 100,000-object sample of the workload"},
    ("nbody_mixed_1m", 10, 1): {"bytes_per_object": (12_881_920 + 127_488) / 100_000,
                                "fp64_pipe": 0.326,
                                "captured": "one launch on a 100,000-object sample of the workload"},
}

CLOSE_AU = 0.01  # objects whose closest planet approach is below this are reported apart


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# differentiation workload: NEOs with JPL comet A1/A2 over two years, 20 observation epochs
ADJ_N, ADJ_EPOCHS, ADJ_SPAN = 4096, 20, 730.5
ADJ_WORKLOAD = (f"differentiation: {ADJ_N} NEO states with JPL comet A1~N(0,1e-8), A2~N(0,1e-9), "
                f"{ADJ_SPAN} d to {ADJ_EPOCHS} uniform epochs; observer on a 1 AU, e=0.0167 orbit; "
                "loss = sum of squared RA/Dec residuals against perturbed truth orbits "
                "(dr~N(0,1e-6 AU), dv~N(0,1e-8 AU/d)); gradient w.r.t. (pos0, vel0, A1, A2)")


WORKLOADS = {
    "nbody_mba_10k": "plain N-body Radau, {n} main-belt states x 365.25 d per GPU, Sun+8 planets"
                     "+Moon from a synthetic SPK type-2 file (14-coef records)",
    "nbody_mixed_1m": "batched uneven N-body, {n} states (90% main belt, 10% NEO, 5% JPL comet "
                      "non-grav A1~N(0,1e-8) A2~N(0,1e-9)), per-object target epochs U(+-5 yr)",
    "kepler_100k": "two-body Kepler, {n} main-belt states, per-object target epochs U(+-1000 d)",
    "survey_10m": "survey chain, {n} states (90% main belt, 10% NEO, 5% comet non-grav), {f} "
                  "rectangular 1.8x1.8 deg fields at ecliptic latitude U(-30,30) deg over one year, "
                  "observer on a 1 AU e=0.0167 orbit; fov_state_check schedule (dt_limit 3 d) then "
                  "H-G V and NEATM NEOS-band magnitudes per detection (H U(12,22), G 0.15, p_V "
                  "lognormal median 0.14 sigma_ln 0.6, beaming 1.0, emissivity 0.9)",
}
WORKLOADS["spk_type21_1m"] = ("SPK state queries, {n} epochs of a type-21 (modified difference "
                              "array) asteroid segment (a 48-record slice of a JPL file), relative "
                              "to the solar-system barycentre through the Sun's type-2 segment")
DEFAULT_N = {"nbody_mba_10k": 10_000, "nbody_mixed_1m": 1_000_000, "kepler_100k": 100_000,
             "survey_10m": 10_000_000, "spk_type21_1m": 1_000_000}
SPK21_SUBSET = os.path.join(ROOT, "tests", "golden", "spk_type21_subset.bsp")
WORKLOADS["nbody_long_10k"] = ("system integration (propagate_n_body_long), {n} main-belt states x "
                               "{years} yr with the Sun, planets and Earth-Moon barycentre "
                               "integrated alongside, batches of 10")
DEFAULT_N["nbody_long_10k"] = 10_000
LONG_YEARS = 10.0
WORKLOADS["thermal_wise_1m"] = ("thermal model, FRM with the four WISE bands and their colour "
                                "corrections at {n} geometries (object at r U(1,4) AU, "
                                "ecliptic latitude N(0,15 deg); observer on a 1 AU orbit; p_V "
                                "lognormal median 0.14 sigma_ln 0.6, H U(8,20), G 0.15, "
                                "emissivity 0.9), 2048-facet sphere")
DEFAULT_N["thermal_wise_1m"] = 1_000_000
# ncu sm__pipe_fp64_cycles_active of the FRM WISE kernel (one capture, 20k geometries)
THERMAL_FP64_PIPE = 0.564
WORKLOADS["stm_cov_1m"] = ("two-body state-transition matrices with covariance propagation, {n} "
                           "main-belt states, per-object spans U(-1000, 1000) d, one 6x6 "
                           "covariance per object (Phi C Phi^T)")
DEFAULT_N["stm_cov_1m"] = 1_000_000
# bytes each object moves: pos, vel, jd0, jd1, covariance in (8 x 44); pos, vel, STM,
# covariance, status out (8 x 78 + 4)
STM_BYTES_PER_OBJECT = 8 * 44 + 8 * 78 + 4
WORKLOADS["adjoint_4k"] = ADJ_WORKLOAD
DEFAULT_N["adjoint_4k"] = ADJ_N
SPK21_ID = 20000042
SURVEY_FIELDS, SURVEY_DT_LIMIT = 2000, 3.0


def workload(n, seed=21, kind="nbody_mba_10k"):
    """Seeded inputs: pos (3,n), vel (3,n), jd0 (n,), jd1 (n,), nongrav (10,n) or None."""
    from kete_b200 import synthetic

    if kind == "nbody_mixed_1m":
        pos, vel, ng = synthetic.mixed(n, seed=seed)
        rng = np.random.default_rng(seed + 100)
        jd0 = np.full(n, EPOCH)
        jd1 = EPOCH + rng.uniform(-5 * 365.25, 5 * 365.25, n)
        return pos, vel, jd0, jd1, ng
    pos, vel = synthetic.main_belt(n, seed=seed)
    jd0 = np.full(n, EPOCH)
    if kind == "kepler_100k":
        rng = np.random.default_rng(seed + 100)
        return pos, vel, jd0, EPOCH + rng.uniform(-1000.0, 1000.0, n), None
    return pos, vel, jd0, np.full(n, EPOCH + SPAN), None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu_index = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi's start-up can hold the driver for seconds; let it finish before
            # the caller records its first event, so the stall stays out of the timing
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 20.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
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
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def reduce_max(x, world):
    """Maximum of a per-rank value over all ranks (the job's time is its slowest rank)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def bench_config(kind, n):
    """The workload description both arms print (identical keys and values)."""
    return {"workload": WORKLOADS[kind].format(n=n), "n_objects": n, "seed": 21,
            "l2": "flushed (256 MB write) between timed GPU steps"}


def cpu_sample(kind, n):
    """Indices of the bounded CPU sample for a workload (the full set when it is small)."""
    if kind == "nbody_mixed_1m":
        return np.arange(0, n, 100)  # seeded 1% subsample, extrapolated per object-year
    return np.arange(n)


def cpu_baseline(kind, pos, vel, jd0, jd1, ng, spk_bytes, threads=0):
    """Time the oracle (CPU restatement of kete's path) on all host cores."""
    from oracle import oracle as O

    cores = threads or os.cpu_count()
    if kind == "kepler_100k":
        t = time.perf_counter()
        op, ov, ojd, st = O.propagate_two_body(pos, vel, jd0, jd1, threads=cores)
        return op, st, time.perf_counter() - t, cores
    O.spk_reset()
    O.spk_load_bytes(spk_bytes)
    t = time.perf_counter()
    op, ov, st, ns, ne = O.propagate_n_body(pos, vel, jd0, jd1, ng=ng, threads=cores)
    return op, st, time.perf_counter() - t, cores


def units_of(kind, jd0, jd1):
    """Work units of a workload: object-years (N-body) or objects (two-body)."""
    if kind == "kepler_100k":
        return float(len(jd0)), "objects/s", "two-body objects/s (propagate_two_body)"
    return float(np.sum(np.abs(jd1 - jd0)) / 365.25), UNIT, METRIC


def run_reference_survey(args):
    """The survey chain on the CPU oracle, on the bounded seeded sample of the population."""
    from kete_b200 import synthetic

    n = args.n or DEFAULT_N["survey_10m"]
    F = args.fields
    pos, vel, ng, h, pv, table = survey_inputs(n, F, seed=41)
    rng = np.random.default_rng(7)
    idx = np.sort(rng.choice(n, size=min(n, args.cpu_sample), replace=False))
    with tempfile.TemporaryDirectory() as td:
        spk = synthetic.write_synthetic_spk(os.path.join(td, "syn.bsp"))
        spk_bytes = open(spk, "rb").read()
    w = idx[: min(200, len(idx))]
    for _ in range(args.warmup):
        survey_oracle(pos[:, w], vel[:, w], ng[:, w], table, spk_bytes, SURVEY_DT_LIMIT)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        survey_oracle(pos[:, idx], vel[:, idx], ng[:, idx], table, spk_bytes, SURVEY_DT_LIMIT)
        times.append(time.perf_counter() - t)
    total = float(np.sum(times))
    value = len(idx) * F * args.steps / total
    line = {
        "impl": "reference", "metric": "survey object-fields/s (fov_state_check + magnitudes)",
        "value": value, "unit": "object-fields/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOADS["survey_10m"].format(n=n, f=F), "n_objects": n},
        "cpu_baseline": {"value": value, "unit": "object-fields/s", "cores": os.cpu_count(),
                         "kind": "port",
                         "sample": f"seeded {len(idx)}-object subsample per step (schedule and "
                                   "field checks; magnitudes not included), oracle on all host "
                                   "cores; the reference Rust/rayon path cannot be built"},
        "e2e": {"value": value, "unit": "object-fields/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_spk(args):
    """SPK type-21 state queries on the CPU oracle, all host cores."""
    from kete_b200 import synthetic
    from oracle import oracle as O

    n = args.n or DEFAULT_N["spk_type21_1m"]
    jd, _ = spk21_queries(n)
    with tempfile.TemporaryDirectory() as td:
        spk = synthetic.write_synthetic_spk(os.path.join(td, "syn.bsp"))
        O.spk_reset()
        for p in (spk, SPK21_SUBSET):
            with open(p, "rb") as f:
                O.spk_load_bytes(f.read())
    for _ in range(args.warmup):
        O.spk_get_states(SPK21_ID, jd[:10000], 0, 1)
    t = time.perf_counter()
    for _ in range(args.steps):
        O.spk_get_states(SPK21_ID, jd, 0, 1)
    total = time.perf_counter() - t
    value = n * args.steps / total
    line = {
        "impl": "reference", "metric": "SPK type-21 states/s", "value": value, "unit": "states/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic planets + type-21 slice",
        "config": {"workload": WORKLOADS["spk_type21_1m"].format(n=n), "n_queries": n},
        "cpu_baseline": {"value": value, "unit": "states/s", "cores": os.cpu_count(),
                         "kind": "port", "sample": "the full workload per step; the reference "
                                                   "Rust path cannot be built"},
        "e2e": {"value": value, "unit": "states/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_long(args):
    """The system integration on the CPU oracle (all host cores), a bounded sample."""
    from kete_b200 import synthetic
    from oracle import oracle as O

    n = args.n or DEFAULT_N["nbody_long_10k"]
    k = min(n, 400)
    pos, vel = synthetic.main_belt(n, seed=71)
    pos, vel = synthetic.ecl_to_eq(pos[:, :k]), synthetic.ecl_to_eq(vel[:, :k])
    jd1 = EPOCH + LONG_YEARS * 365.25
    with tempfile.TemporaryDirectory() as td:
        spk = synthetic.write_synthetic_spk(os.path.join(td, "syn.bsp"))
        O.spk_reset()
        with open(spk, "rb") as f:
            O.spk_load_bytes(f.read())
    for _ in range(args.warmup):
        O.propagate_n_body_vec(pos[:, :10], vel[:, :10], EPOCH, EPOCH + 30.0)
    t = time.perf_counter()
    for _ in range(args.steps):
        O.propagate_n_body_vec(pos, vel, EPOCH, jd1)
    total = time.perf_counter() - t
    value = k * LONG_YEARS * args.steps / total
    line = {
        "impl": "reference", "metric": "system-integration object-years/s", "value": value,
        "unit": "object-years/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS["nbody_long_10k"].format(n=n, years=LONG_YEARS),
                   "n_objects": n},
        "cpu_baseline": {"value": value, "unit": "object-years/s", "cores": os.cpu_count(),
                         "kind": "port", "sample": f"the first {k} objects per step; the "
                                                   "reference Rust path cannot be built"},
        "e2e": {"value": value, "unit": "object-years/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_adjoint(args):
    """The gradient on the CPU oracle as kete offers it: the forward chain over the epochs
    plus central differences in the 8 parameters (16 perturbed chains), on all host cores,
    for a seeded sample of the differentiation workload's objects."""
    from kete_b200 import synthetic
    from oracle import oracle as O

    pos, vel, ng, _, _, epochs, _ = adjoint_population(ADJ_N)
    k = 64
    sp, sv, sg = pos[:, :k].copy(), vel[:, :k].copy(), ng[:, :k].copy()
    with tempfile.TemporaryDirectory() as td:
        spk = synthetic.write_synthetic_spk(os.path.join(td, "syn.bsp"))
        O.spk_reset()
        O.spk_load_bytes(open(spk, "rb").read())

    def chain(p, v, g):
        t, m = EPOCH, p.shape[1]
        for e in epochs:
            p, v, _, _, _ = O.propagate_n_body(p, v, np.full(m, t), np.full(m, e), ng=g)
            t = e
        return p

    steps = [1e-4] * 3 + [1e-6] * 3 + [5e-8, 5e-9]

    def gradient():
        chain(sp, sv, sg)
        for q, d in enumerate(steps):
            for s in (d, -d):
                p, v, g = sp.copy(), sv.copy(), sg.copy()
                if q < 3:
                    p[q] += s
                elif q < 6:
                    v[q - 3] += s
                else:
                    g[q - 5] += s
                chain(p, v, g)

    for _ in range(args.warmup):
        chain(sp[:, :4].copy(), sv[:, :4].copy(), sg[:, :4].copy())
    t = time.perf_counter()
    for _ in range(args.steps):
        gradient()
    total = time.perf_counter() - t
    value = k * ADJ_SPAN / 365.25 * args.steps / total
    line = {
        "impl": "reference",
        "metric": "reverse-mode gradient object-years/s (checkpointed forward + adjoint)",
        "value": value, "unit": "object-years/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": ADJ_WORKLOAD, "n_objects": ADJ_N,
                   "l2": "inputs resident; consecutive passes share the ephemeris in L2"},
        "cpu_baseline": {"value": value, "unit": "object-years/s", "cores": os.cpu_count(),
                         "kind": "port",
                         "sample": f"the first {k} objects per step: the forward chain and 16 "
                                   "perturbed chains (central differences in the 8 "
                                   "parameters), oracle on all host cores"},
        "e2e": {"value": value, "unit": "object-years/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference(args, world, rank):
    if rank != 0:
        return
    from kete_b200 import synthetic

    if args.workload == "survey_10m":
        return run_reference_survey(args)
    if args.workload == "spk_type21_1m":
        return run_reference_spk(args)
    if args.workload == "nbody_long_10k":
        return run_reference_long(args)
    if args.workload == "thermal_wise_1m":
        return run_reference_thermal(args)
    if args.workload == "stm_cov_1m":
        return run_reference_stm(args)
    if args.workload == "adjoint_4k":
        return run_reference_adjoint(args)
    kind = args.workload
    n = args.n or DEFAULT_N[kind]
    pos, vel, jd0, jd1, ng = workload(n, kind=kind)
    idx = cpu_sample(kind, n)
    sp, sv, s0, s1 = pos[:, idx], vel[:, idx], jd0[idx], jd1[idx]
    sng = None if ng is None else ng[:, idx]
    units, unit, metric = units_of(kind, s0, s1)
    with tempfile.TemporaryDirectory() as td:
        spk = synthetic.write_synthetic_spk(os.path.join(td, "syn.bsp"))
        spk_bytes = open(spk, "rb").read()
    for _ in range(args.warmup):
        w = slice(0, min(200, len(idx)))
        cpu_baseline(kind, sp[:, w], sv[:, w], s0[w], s1[w], None if sng is None else sng[:, w],
                     spk_bytes)
    times = []
    cores = os.cpu_count()
    for _ in range(args.steps):
        _, st, dt, cores = cpu_baseline(kind, sp, sv, s0, s1, sng, spk_bytes)
        times.append(dt)
    total = float(np.sum(times))
    value = units * args.steps / total
    sample = ("full workload per step" if len(idx) == n else
              f"seeded 1% subsample ({len(idx)} of {n} objects) per step, rate per object-year")
    line = {
        "impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": bench_config(kind, n),
        "cpu_baseline": {"value": value, "unit": unit, "cores": cores, "kind": "port",
                         "sample": sample + "; the reference Rust/rayon path cannot be built "
                                   "(no Rust toolchain), so the C restatement of kete's FP64 code "
                                   "runs under OpenMP on all host cores"},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_gpu(args, world, rank, local):
    import torch

    import kete_b200
    from kete_b200 import _lib, build, synthetic, tune

    build.build()
    torch.cuda.set_device(local)
    kete_b200.init(local)
    td = tempfile.mkdtemp(prefix="kete_b200_bench_")
    spk = synthetic.write_synthetic_spk(os.path.join(td, "syn.bsp"))
    spk_bytes = open(spk, "rb").read()
    kete_b200.spice.kernel_reload([spk])

    kind = args.workload
    n = args.n or DEFAULT_N[kind]
    nbody = kind != "kepler_100k"
    pos, vel, jd0, jd1, ng = workload(n, seed=21 + rank, kind=kind)
    units, unit, metric = units_of(kind, jd0, jd1)
    dev = torch.device("cuda", local)
    host = dict(pos=pos, vel=vel, jd0=jd0, jd1=jd1)
    if ng is not None:
        host["ng"] = ng
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in host.items()}

    sweep = None
    best = None
    if nbody:
        if args.mode == 0:
            # a large population is tuned on a seeded eighth of it (still several waves of
            # lane groups on 148 SMs), which keeps the sweep of every configuration short
            sub = slice(None) if n <= 200_000 else slice(0, None, 8)
            best, sweep = tune.autotune(d["pos"][:, sub].contiguous(),
                                        d["vel"][:, sub].contiguous(),
                                        d["jd0"][sub].contiguous(), d["jd1"][sub].contiguous(),
                                        nongrav=(d["ng"][:, sub].contiguous() if "ng" in d
                                                 else None),
                                        full=(None if n <= 200_000 else
                                              (d["pos"], d["vel"], d["jd0"], d["jd1"],
                                               d.get("ng"))))
        else:
            best = dict(mode=args.mode, variant=args.variant, refill=args.refill)
            tune.set_config(**best)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step(arrs, out=None):
        if nbody:
            return kete_b200.propagate_n_body_arrays(arrs["pos"], arrs["vel"], arrs["jd0"],
                                                     arrs["jd1"], nongrav=arrs.get("ng"),
                                                     mode=best["mode"], out=out)
        return kete_b200.propagate_two_body_arrays(arrs["pos"], arrs["vel"], arrs["jd0"],
                                                   arrs["jd1"])

    flops = flops_ref = None
    steps_total = iters_total = 0
    min_dist = None
    if nbody:  # counts for the flop model (deterministic: same inputs every step)
        _, _, _, det = kete_b200.propagate_n_body_arrays(d["pos"], d["vel"], d["jd0"], d["jd1"],
                                                         nongrav=d.get("ng"), mode=best["mode"],
                                                         with_details=True)
        cnt = det["counters"].to(torch.int64).sum(dim=1).cpu().numpy()
        steps_total, iters_total, exact_total = (int(x) for x in cnt)
        flops, flops_ref = flop_models(steps_total, iters_total, exact_total)
        min_dist = det["min_dist"].cpu().numpy()
    # the library's own launch counter over one step (the graph replays the same launches)
    count = _lib.lib().kete_b200_kernel_launches
    count.restype = ctypes.c_int64
    c0 = count()
    step(d)
    torch.cuda.synchronize()
    launches_per_step = int(count() - c0)

    for _ in range(args.warmup):
        step(d)
    torch.cuda.synchronize()
    # the timed steps replay a captured CUDA graph of one step (the library allocates nothing
    # once its buffers have grown to the workload, so the step captures as it runs)
    graph = None
    if not args.no_graph:
        try:
            side = torch.cuda.Stream(dev)
            side.wait_stream(torch.cuda.current_stream(dev))
            with torch.cuda.stream(side):
                step(d)
            torch.cuda.current_stream(dev).wait_stream(side)
            torch.cuda.synchronize()
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                step(d)
            torch.cuda.synchronize()
            for _ in range(2):
                graph.replay()
            torch.cuda.synchronize()
        except Exception as e:  # capture refused: time direct launches instead
            log("CUDA graph capture failed, timing direct launches:", repr(e))
            graph = None
    run_step = graph.replay if graph is not None else (lambda: step(d))
    stream = torch.cuda.current_stream(dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()  # write > L2 (126 MB) between steps, outside the timed pair
            evs[k][0].record(stream)
            run_step()
            evs[k][1].record(stream)
        torch.cuda.synchronize()
        barrier(world)
    ms = [a.elapsed_time(b) for a, b in evs]
    t_total = reduce_max(float(np.sum(ms)) * 1e-3, world)
    ms_step = 1e3 * t_total / args.steps
    value = world * units * args.steps / t_total

    # the plain form on the same inputs: one thread per object, one launch per call
    plain = None
    if nbody and best.get("mode") != _lib.MODE_THREAD:
        cur = tune.current()
        tune.set_config(mode=_lib.MODE_THREAD, variant=0, refill=0)
        plain_steps = max(1, min(args.steps, 2))
        kete_b200.propagate_n_body_arrays(d["pos"], d["vel"], d["jd0"], d["jd1"],
                                          nongrav=d.get("ng"), mode=_lib.MODE_THREAD)
        torch.cuda.synchronize()
        pev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(plain_steps)]
        barrier(world)
        for k in range(plain_steps):
            flush.zero_()
            pev[k][0].record(stream)
            kete_b200.propagate_n_body_arrays(d["pos"], d["vel"], d["jd0"], d["jd1"],
                                              nongrav=d.get("ng"), mode=_lib.MODE_THREAD)
            pev[k][1].record(stream)
        torch.cuda.synchronize()
        barrier(world)
        p_total = reduce_max(sum(a.elapsed_time(b) for a, b in pev) * 1e-3, world)
        tune.set_config(**cur)
        plain = {"form": "nbody_thread_kernel: one thread per object, one launch per call",
                 "steps": plain_steps, "ms_per_step": 1e3 * p_total / plain_steps,
                 "value": world * units * plain_steps / p_total, "unit": unit,
                 "batched_over_plain": (p_total / plain_steps) / (t_total / args.steps)}

    # end to end through the C ABI with pinned host buffers: the inputs, and for the N-body
    # call the outputs too (allocated once and passed as out=, as a caller that propagates
    # the same population repeatedly would)
    hp = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in host.items()}
    hnp = {k: v.numpy() for k, v in hp.items()}
    hout = None
    if nbody:
        hout = (torch.empty((3, n), dtype=torch.float64).pin_memory().numpy(),
                torch.empty((3, n), dtype=torch.float64).pin_memory().numpy(),
                torch.empty((n,), dtype=torch.int32).pin_memory().numpy())
    step(hnp, hout)
    e2e_t = []
    out = None
    for _ in range(args.steps):
        t = time.perf_counter()
        out = step(hnp, hout)
        e2e_t.append(time.perf_counter() - t)
    e2e_total = reduce_max(float(np.sum(e2e_t)), world)
    e2e_value = world * units * args.steps / e2e_total
    h2d = sum(int(v.nbytes) for v in hnp.values())
    d2h = 6 * n * 8 + 4 * n + (0 if nbody else 8 * n)

    if rank != 0:
        return
    tflops_probe = ctypes_probe(_lib)
    peaks = measured_peaks()
    hbm_bytes = int(h2d + d2h)
    if nbody:
        achieved = flops / (ms_step * 1e-3) / 1e12
        achieved_ref = flops_ref / (ms_step * 1e-3) / 1e12
        tr = NODE_TRAFFIC.get((kind, best.get("variant"), best.get("refill")))
        traffic = None if tr is None else tr["bytes_per_object"] * n
        roof = {"bound": "fp64", "achieved": achieved, "peak": tflops_probe, "unit": "TFLOP/s",
                "frac": achieved / tflops_probe if tflops_probe else None,
                "flop_model": "work: records at the 8 distinct times of each step, force terms "
                              "at every evaluation, Radau algebra (kernel counters)",
                "flops_per_launch": flops,
                "achieved_reference_model": achieved_ref,
                "frac_reference_model": achieved_ref / tflops_probe if tflops_probe else None,
                "flops_per_launch_reference_model": flops_ref,
                "traffic": traffic,
                "traffic_unit": "bytes per launch (DRAM read + write)",
                "traffic_source": (None if tr is None else
                                   f"ncu dram__bytes_read.sum + dram__bytes_write.sum of "
                                   f"{tr['captured']}, scaled to {n} objects "
                                   f"({tr['bytes_per_object']:.1f} B per object)"),
                "peak_source": "measured DFMA probe (kete_b200_fp64_probe) in this run",
                "hbm_bytes_algorithmic": hbm_bytes}
        if tr is not None and tr.get("fp64_pipe") is not None:
            roof["fp64_pipe_active_ncu"] = tr["fp64_pipe"]
    else:
        gbs = hbm_bytes / (ms_step * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": gbs, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                "frac": gbs / peaks["hbm_gbs"] if peaks.get("hbm_gbs") else None,
                "traffic": None, "peak_source": "MEASURED_PEAKS.json hbm_gbs",
                "note": "the two-body solve is transcendental-bound; HBM is the nominal bound"}

    # CPU baseline (oracle on all host cores) on the bounded sample, and a parity check
    idx = cpu_sample(kind, n)
    op, st_cpu, cpu_dt, cores = cpu_baseline(kind, pos[:, idx], vel[:, idx], jd0[idx], jd1[idx],
                                             None if ng is None else ng[:, idx], spk_bytes)
    cpu_units, _, _ = units_of(kind, jd0[idx], jd1[idx])
    # the same oracle on one thread, over every tenth object of the sample
    i1 = idx[::10]
    _, _, cpu1_dt, _ = cpu_baseline(kind, pos[:, i1], vel[:, i1], jd0[i1], jd1[i1],
                                    None if ng is None else ng[:, i1], spk_bytes, threads=1)
    cpu1_units, _, _ = units_of(kind, jd0[i1], jd1[i1])
    gp = out[0][:, idx]
    gst = (out[2] if nbody else out[3])[idx]
    err = np.linalg.norm(gp - op, axis=0)
    ok = (gst == 0) & (st_cpu == 0)
    tol = 1e-9 if nbody else 1e-12
    parity = {"objects_compared": int(ok.sum()),
              "status_mismatches": int((gst != st_cpu).sum()),
              "gpu_status_counts": np.bincount(gst, minlength=8).tolist(),
              "cpu_status_counts": np.bincount(st_cpu, minlength=8).tolist(),
              "tolerance_au": tol,
              "sample": ("the full workload" if len(idx) == n else
                         f"seeded 1% subsample ({len(idx)} objects, every 100th)")}
    if nbody:
        close = min_dist[idx] < CLOSE_AU
        far = ok & ~close
        near = ok & close
        parity["max_err_au"] = float(err[far].max()) if far.any() else None
        parity["max_err_au_note"] = (f"objects whose closest planet approach stays above "
                                     f"{CLOSE_AU} AU")
        parity["close_approach"] = {
            "threshold_au": CLOSE_AU, "objects": int(close.sum()),
            "max_err_au": float(err[near].max()) if near.any() else None,
            "within_tolerance": int((err[near] <= tol).sum()),
            "listed": [{"object": int(idx[i]), "min_planet_dist_au": float(min_dist[idx[i]]),
                        "err_au": float(err[i]), "gpu_status": int(gst[i]),
                        "cpu_status": int(st_cpu[i])}
                       for i in np.flatnonzero(close)[:25]]}
    else:
        parity["max_err_au"] = float(err[ok].max()) if ok.any() else None
    line = {
        "metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(kind, n),
        "launch": {"config": best, "autotune_sweep_ms": sweep,
                   "autotune_inputs": ("the workload" if n <= 200_000 else
                                       "every 8th object of the workload; the configurations "
                                       "within 5% of its best (at most 3) re-timed on the "
                                       "whole workload (_full)"),
                   "cuda_graph": graph is not None,
                   "parallelism": f"replicas x{world} (objects independent)"},
        "roofline": roof,
        "cpu_baseline": {"value": cpu_units / cpu_dt, "unit": unit, "cores": cores,
                         "kind": "port",
                         "sample": ("the full workload" if len(idx) == n else
                                    f"seeded 1% subsample ({len(idx)} objects, every 100th), "
                                    "rate per object-year") +
                                   ", oracle (C restatement of kete's FP64 path) with OpenMP on "
                                   "all host cores",
                         "one_thread": {"value": cpu1_units / cpu1_dt, "unit": unit, "cores": 1,
                                        "sample": f"every tenth object of that sample "
                                                  f"({len(i1)} objects)"}},
        "e2e": {"value": e2e_value, "unit": unit, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": args.steps * launches_per_step,
        "clocks": clk.summary(),
        "parity": parity,
    }
    if plain is not None:
        line["plain"] = plain
    if nbody:
        line["object_steps_per_s"] = world * steps_total * args.steps / t_total
        line["corrector_iterations_per_step"] = iters_total / max(steps_total, 1)
    if kind in ("nbody_mba_10k", "nbody_mixed_1m") and not args.no_adjoint:
        line["adjoint"] = adjoint_section(dev, max(1, args.warmup), max(1, min(args.steps, 3)))
    print(json.dumps(line), flush=True)


def run_adjoint(args, world, rank, local):
    """The differentiation workload on its own: forward pass, checkpointed forward, adjoint
    and forward sensitivities (the gradient-cost section of the default line)."""
    import torch

    import kete_b200
    from kete_b200 import build, synthetic

    build.build()
    torch.cuda.set_device(local)
    kete_b200.init(local)
    td = tempfile.mkdtemp(prefix="kete_b200_bench_")
    kete_b200.spice.kernel_reload([synthetic.write_synthetic_spk(os.path.join(td, "syn.bsp"))])
    dev = torch.device("cuda", local)
    sec = adjoint_section(dev, max(1, args.warmup), max(1, min(args.steps, 3)))
    if rank != 0:
        return
    years = ADJ_N * ADJ_SPAN / 365.25
    line = {
        "metric": "reverse-mode gradient object-years/s (checkpointed forward + adjoint)",
        "value": world * years / ((sec["checkpointed_forward_ms"] + sec["adjoint_ms"]) * 1e-3),
        "unit": "object-years/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sec["checkpointed_forward_ms"] + sec["adjoint_ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": ADJ_WORKLOAD, "n_objects": ADJ_N,
                   "l2": "inputs resident; consecutive passes share the ephemeris in L2"},
        "adjoint": sec,
    }
    print(json.dumps(line), flush=True)


def adjoint_population(n, seed=33):
    """NEO states with comet A1/A2, their perturbed truth, the epochs and observer positions."""
    from kete_b200 import synthetic

    pos, vel = synthetic.neo(n, seed=seed)
    rng = np.random.default_rng(seed + 1)
    ng = np.repeat(synthetic.comet_nongrav(0.0, 0.0)[:, None], n, axis=1)
    ng[1] = rng.normal(0.0, 1e-8, n)
    ng[2] = rng.normal(0.0, 1e-9, n)
    tpos = pos + rng.normal(0.0, 1e-6, (3, n))
    tvel = vel + rng.normal(0.0, 1e-8, (3, n))
    epochs = EPOCH + np.linspace(ADJ_SPAN / ADJ_EPOCHS, ADJ_SPAN, ADJ_EPOCHS)
    obs, _ = synthetic.kepler_state(1.0, 0.0167, 0.0, 0.0, 1.7967, 0.0, EPOCH, epochs)
    return pos, vel, np.ascontiguousarray(ng), tpos, tvel, epochs, np.ascontiguousarray(obs)


def adjoint_section(dev, warmup, steps):
    """Cost of the reverse-mode gradient beside one forward pass on the differentiation
    workload, and its agreement with the transposed forward sensitivities."""
    import torch

    from kete_b200 import autodiff as A
    from kete_b200 import propagate_n_body_arrays, tune

    pos, vel, ng, tpos, tvel, epochs, obs = adjoint_population(ADJ_N)
    n, K = ADJ_N, ADJ_EPOCHS
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    P, V, G, E = T(pos), T(vel), T(ng), T(epochs)
    O = T(obs.T)[:, :, None]  # observer (K, 3, 1)
    jd0 = torch.full((n,), EPOCH, dtype=torch.float64, device=dev)
    ts, tst, _ = A.propagate_n_body_checkpointed(T(tpos), T(tvel), jd0, E, nongrav=G)
    ra_t, dec_t = A.radec(A.ecliptic_to_equatorial_torch(ts[:, 0:3] - O))

    def seed_of(states):
        s = states.detach().clone().requires_grad_(True)
        ra, dec = A.radec(A.ecliptic_to_equatorial_torch(s[:, 0:3] - O))
        dra = torch.remainder(ra - ra_t + np.pi, 2 * np.pi) - np.pi
        loss = (dra ** 2 + (dec - dec_t) ** 2).sum()
        (g,) = torch.autograd.grad(loss, s)
        return g.contiguous()

    best, _ = tune.autotune(P, V, jd0, torch.full((n,), EPOCH + ADJ_SPAN, dtype=torch.float64,
                                                  device=dev), nongrav=G)
    jds = [torch.full((n,), float(e), dtype=torch.float64, device=dev) for e in epochs]

    def forward():  # the product path: one propagate_n_body call per epoch
        p, v, t0 = P, V, jd0
        for k in range(K):
            p, v, _ = propagate_n_body_arrays(p, v, t0, jds[k], nongrav=G, mode=best["mode"])
            t0 = jds[k]
        return p

    states, st, ck = A.propagate_n_body_checkpointed(P, V, jd0, E, nongrav=G)
    cap = ck.capacity
    seed = seed_of(states)
    g_adj, gst = A.propagate_n_body_adjoint(ck, seed)
    _, stm, sst = A.propagate_n_body_stm_arrays(P, V, jd0, E, nongrav=G)
    g_stm = torch.einsum("kcn,kcpn->pn", seed, stm)
    ok = ((st == 0) & (gst == 0) & (sst == 0)).cpu().numpy()
    rel = {}
    for name, rows in (("pos0", slice(0, 3)), ("vel0", slice(3, 6)), ("A1", slice(6, 7)),
                       ("A2", slice(7, 8))):
        a_, b_ = g_adj[rows].cpu().numpy()[:, ok], g_stm[rows].cpu().numpy()[:, ok]
        rel[name] = float((np.abs(a_ - b_).max(axis=0) / np.abs(b_).max(axis=0)).max())

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    fwd_ms = timed(forward)
    ck_ms = timed(lambda: A.propagate_n_body_checkpointed(P, V, jd0, E, nongrav=G, capacity=cap))
    adj_ms = timed(lambda: A.propagate_n_body_adjoint(ck, seed))
    stm_ms = timed(lambda: A.propagate_n_body_stm_arrays(P, V, jd0, E, nongrav=G))
    return {
        "workload": ADJ_WORKLOAD,
        "forward_ms": fwd_ms, "forward_launch": best,
        "checkpointed_forward_ms": ck_ms, "adjoint_ms": adj_ms,
        "adjoint_over_forward": adj_ms / fwd_ms,
        "adjoint_over_checkpointed_forward": adj_ms / ck_ms,
        "checkpointed_forward_plus_adjoint_over_forward": (ck_ms + adj_ms) / fwd_ms,
        "stm_ms": stm_ms, "stm_over_forward": stm_ms / fwd_ms,
        "checkpoints_per_object": cap, "objects_ok": int(ok.sum()),
        "adjoint_vs_transposed_stm_max_rel_err": rel,
        "note": "forward = one node-kernel propagate_n_body call per epoch (autotuned); "
                "adjoint = kete_b200_propagate_n_body_adjoint given dL/d(states)",
    }


def survey_inputs(n, n_fields, seed=41):
    """Population with H/G/albedo, and the time-sorted field table (20, F)."""
    from kete_b200 import fov as fovmod
    from kete_b200 import synthetic
    from kete_b200.state import Frames, State

    pos, vel, ng = synthetic.mixed(n, seed=seed)
    rng = np.random.default_rng(seed + 1)
    h = rng.uniform(12.0, 22.0, n)
    pv = np.exp(np.log(0.14) + 0.6 * rng.normal(size=n))
    frng = np.random.default_rng(seed + 2)
    jds = np.sort(EPOCH + frng.uniform(0.0, 365.25, n_fields))
    lat = np.radians(frng.uniform(-30.0, 30.0, n_fields))
    lon = frng.uniform(0.0, 2 * np.pi, n_fields)
    op, ov = synthetic.kepler_state(1.0, 0.0167, 0.0, 0.0, 1.7967, 0.0, EPOCH, jds)
    cols = []
    for k in range(n_fields):
        pointing = [np.cos(lat[k]) * np.cos(lon[k]), np.cos(lat[k]) * np.sin(lon[k]), np.sin(lat[k])]
        obs = State("observer", jds[k], op[:, k], ov[:, k], Frames.Ecliptic, 10)
        cols.append(fovmod.RectangleFOV(pointing, 0.0, obs, 1.8, 1.8).ecliptic_column())
    return pos, vel, ng, h, pv, np.ascontiguousarray(np.stack(cols, axis=1))


def survey_magnitudes(ff, oo, ss, table, h, pv):
    """H-G V magnitude and NEATM NEOS-band magnitudes of every detection (GPU kernels)."""
    from kete_b200 import flux

    m = len(oo)
    if m == 0:
        return np.empty(0), np.empty((2, 0))
    sun2obj = np.ascontiguousarray(ss[1:4])
    sun2obs = np.ascontiguousarray(table[1:4, ff])
    hh, alb = h[oo], pv[oo]
    v = flux.hg_apparent_mag_arrays(sun2obj, sun2obs, hh, np.full(m, 0.15))
    diam = flux.C_V / np.sqrt(alb) * 10.0 ** (-0.2 * hh)
    res = flux.neatm_arrays(sun2obj, sun2obs, hh, np.full(m, 0.15), diam, alb, np.ones(m),
                            np.full(m, 0.9), np.array(flux.NEOS_BANDS), np.stack([alb, alb]),
                            zero_mags=np.array(flux.NEOS_ZERO_MAG))
    return v, res["magnitudes"]


def survey_oracle(pos, vel, ng, table, spk_bytes, dt_limit):
    """The fov_state_check schedule on the CPU oracle (all host cores): set of (field, obj)
    and the oracle's state per pair."""
    from kete_b200.fov import chunk_bounds
    from oracle import oracle as O

    O.spk_reset()
    O.spk_load_bytes(spk_bytes)
    n = pos.shape[1]
    jds = table[0]

    def prop(p, target):
        op, ov, st, _, _ = O.propagate_n_body(p[0], p[1], np.full(n, p[3]), np.full(n, target),
                                              ng=ng)
        return [op, ov, p[2] & (st == 0), target]

    cur_jd = big_jd = EPOCH
    cur = [pos.copy(), vel.copy(), np.ones(n, bool), EPOCH]
    big = [pos.copy(), vel.copy(), np.ones(n, bool), EPOCH]
    found = {}
    bounds = chunk_bounds(jds, dt_limit)
    for k0, k1 in zip(bounds[:-1], bounds[1:]):
        jd_mean = (jds[k1 - 1] + jds[k0]) / 2.0
        if abs(jd_mean - big_jd) >= dt_limit * 50:
            big_jd = jd_mean
            big = prop(big, cur_jd)
        if abs(jd_mean - cur_jd) >= dt_limit:
            if abs(cur_jd - big_jd) >= dt_limit * 25:
                cur = [big[0].copy(), big[1].copy(), big[2].copy(), big[3]]
            cur_jd = jd_mean
            cur = prop(cur, cur_jd)
        idx = np.nonzero(cur[2])[0]
        for k in range(k0, k1):
            col = table[:, k]
            flags, out7 = O.fov_check_visible(col[:7], col[7:19].reshape(4, 3), cur[0][:, idx],
                                              cur[1][:, idx], np.full(idx.size, cur[3]), dt_limit)
            for j in np.nonzero(flags)[0]:
                found[(k, int(idx[j]))] = out7[:, j]
    return found


def run_survey(args, world, rank, local):
    import torch

    import kete_b200
    from kete_b200 import build, synthetic
    from kete_b200.fov import fov_state_check_arrays

    build.build()
    torch.cuda.set_device(local)
    kete_b200.init(local)
    td = tempfile.mkdtemp(prefix="kete_b200_bench_")
    spk = synthetic.write_synthetic_spk(os.path.join(td, "syn.bsp"))
    spk_bytes = open(spk, "rb").read()
    kete_b200.spice.kernel_reload([spk])
    n = args.n or DEFAULT_N["survey_10m"]
    F = args.fields
    pos, vel, ng, h, pv, table = survey_inputs(n, F, seed=41 + rank)
    dev = torch.device("cuda", local)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    P, V, G, TB = T(pos), T(vel), T(ng), T(table)
    n_chunks = [0]

    def chain(P_, V_):
        n_chunks[0] = 0
        ff, oo, ss = fov_state_check_arrays(P_, V_, EPOCH, TB, SURVEY_DT_LIMIT, False, G,
                                            on_chunk=lambda a, b: n_chunks.__setitem__(0, n_chunks[0] + 1))
        v, mags = survey_magnitudes(ff, oo, ss, table, h, pv)
        return ff, oo, ss, v, mags

    # launch configuration of the chunk re-propagations, tuned on a 200k-object sample over
    # one chunk's span (2 x dt_limit), the closest configurations re-timed on every object
    from kete_b200 import tune

    m = min(n, 200_000)
    span = lambda k, d: torch.full((k,), EPOCH + d, dtype=torch.float64, device=dev)
    launch, _ = tune.autotune(P[:, :m].contiguous(), V[:, :m].contiguous(), span(m, 0.0),
                              span(m, 2 * SURVEY_DT_LIMIT), nongrav=G[:, :m].contiguous(),
                              full=(None if m == n else
                                    (P, V, span(n, 0.0), span(n, 2 * SURVEY_DT_LIMIT), G)))
    for _ in range(args.warmup):
        chain(P, V)
    torch.cuda.synchronize()
    from kete_b200 import _lib as klib

    count = klib.lib().kete_b200_kernel_launches
    count.restype = ctypes.c_int64
    with ClockSampler(local) as clk:
        barrier(world)
        launches0 = count()
        t = time.perf_counter()
        for _ in range(args.steps):
            ff, oo, ss, vmag, bmag = chain(P, V)
        torch.cuda.synchronize()
        chain_s = reduce_max((time.perf_counter() - t) / args.steps, world)
        launches = int(count() - launches0)
        barrier(world)
    value = world * n * F / chain_s
    # end to end: the population starts in pinned host memory
    hp = {k: torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for k, a in
          (("pos", pos), ("vel", vel), ("ng", ng), ("table", table))}
    t = time.perf_counter()
    P2, V2 = hp["pos"].to(dev, non_blocking=True), hp["vel"].to(dev, non_blocking=True)
    G2, TB2 = hp["ng"].to(dev, non_blocking=True), hp["table"].to(dev, non_blocking=True)
    G, TB = G2, TB2
    chain(P2, V2)
    torch.cuda.synchronize()
    e2e_s = reduce_max(time.perf_counter() - t, world)

    # FOV prefilter roofline on one chunk: algorithmic bytes = the population's states,
    # epochs and flags read once (57 B per object) plus the field columns
    from kete_b200.fov import chunk_bounds, fov_check_visible_arrays
    b = chunk_bounds(table[0], SURVEY_DT_LIMIT)
    sub = TB[:, b[0]:b[1]].contiguous()
    # the schedule checks each chunk with the population at the chunk's mean epoch
    jd_mean = 0.5 * (float(table[0, b[0]]) + float(table[0, b[1] - 1]))
    jdv = torch.full((n,), jd_mean, dtype=torch.float64, device=dev)
    okv = torch.ones(n, dtype=torch.uint8, device=dev)
    fov_check_visible_arrays(P, V, jdv, okv, sub, SURVEY_DT_LIMIT)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    reps = 3
    for _ in range(reps):
        fov_check_visible_arrays(P, V, jdv, okv, sub, SURVEY_DT_LIMIT)
    e1.record()
    torch.cuda.synchronize()
    fov_ms = e0.elapsed_time(e1) / reps
    fov_bytes = n * 57 + sub.numel() * 8
    # one more pass of the chain with its stages timed apart (device synchronized around
    # each stage): the N-body re-propagations, the field checks, the magnitudes
    stages = {}
    ff_s, oo_s, ss_s = fov_state_check_arrays(P, V, EPOCH, TB, SURVEY_DT_LIMIT, False, G,
                                              stage_times=stages)
    torch.cuda.synchronize()
    t = time.perf_counter()
    survey_magnitudes(ff_s, oo_s, ss_s, table, h, pv)
    torch.cuda.synchronize()
    stages["magnitudes"] = time.perf_counter() - t
    peaks = measured_peaks()
    if rank != 0:
        return

    # CPU oracle on a bounded seeded sample: its per-field lists must match the GPU's
    rng = np.random.default_rng(7)
    idx = np.sort(rng.choice(n, size=min(n, args.cpu_sample), replace=False))
    t = time.perf_counter()
    ref = survey_oracle(pos[:, idx], vel[:, idx], ng[:, idx], table, spk_bytes, SURVEY_DT_LIMIT)
    cpu_s = time.perf_counter() - t
    pos_of = {int(o): j for j, o in enumerate(idx)}
    got = {}
    for j in range(len(oo)):
        o = int(oo[j])
        if o in pos_of:
            got[(int(ff[j]), pos_of[o])] = ss[:, j]
    mism, edge_ok, max_err = 0, 0, 0.0
    for key in set(ref) ^ set(got):
        st = ref[key] if key in ref else got[key]
        col = table[:, key[0]]
        rel = st[1:4] - col[1:4]
        rel = rel / np.linalg.norm(rel)
        if np.min(np.abs(col[7:19].reshape(4, 3) @ rel)) < 1e-10:
            edge_ok += 1
        else:
            mism += 1
    for key in set(ref) & set(got):
        max_err = max(max_err, float(np.abs(ref[key][1:4] - got[key][1:4]).max()))
    line = {
        "metric": "survey object-fields/s (fov_state_check + magnitudes)", "value": value,
        "unit": "object-fields/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": chain_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS["survey_10m"].format(n=n, f=F), "n_objects": n,
                   "n_fields": F, "chunks": n_chunks[0], "detections": int(len(oo)),
                   "launch": launch,
                   "l2": "inputs (the population's states) larger than L2",
                   "parallelism": f"replicas x{world} (objects independent)"},
        "stages_s": {"nbody_repropagation": stages.get("propagate"),
                     "field_checks": stages.get("check"), "magnitudes": stages.get("magnitudes"),
                     "note": "one extra pass of the chain with the device synchronized around "
                             "each stage"},
        "roofline": {"bound": "hbm", "kernel": "fov_screen_kernel + fov_pairs_kernel (one chunk)",
                     "achieved": fov_bytes / (fov_ms * 1e-3) / 1e9, "peak": peaks.get("hbm_gbs"),
                     "unit": "GB/s",
                     "frac": (fov_bytes / (fov_ms * 1e-3) / 1e9) / peaks["hbm_gbs"]
                     if peaks.get("hbm_gbs") else None, "traffic": None,
                     "chunk_ms": fov_ms, "bytes_algorithmic": fov_bytes,
                     "note": "time of one chunk's fov_check_visible call (linear screen, "
                             "two-body pass, n-body branch if any, result copy-back); the "
                             "chain's dominant kernel is the node kernel of the chunk "
                             "re-propagations (stages_s), whose roofline the N-body workloads "
                             "report"},
        "cpu_baseline": {"value": len(idx) * F / cpu_s, "unit": "object-fields/s",
                         "cores": os.cpu_count(), "kind": "port",
                         "sample": f"seeded {len(idx)}-object subsample of the population, full "
                                   "field list and schedule, oracle on all host cores"},
        "e2e": {"value": world * n * F / e2e_s, "unit": "object-fields/s",
                "h2d_bytes_per_step": int(pos.nbytes + vel.nbytes + ng.nbytes + table.nbytes),
                "d2h_bytes_per_step": int(len(oo) * (4 + 4 + 56 + 8 + 16))},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "parity": {"sample_objects": int(len(idx)), "oracle_pairs": len(ref),
                   "gpu_pairs_in_sample": len(got), "mismatches_off_edge": mism,
                   "mismatches_within_1e-10_rad_of_edge": edge_ok,
                   "max_state_err_au": max_err},
        "magnitudes": {"v_median": float(np.nanmedian(vmag)) if len(vmag) else None,
                       "neatm_band_mag_median": [float(np.nanmedian(x)) for x in bmag]
                       if len(vmag) else None},
    }
    print(json.dumps(line), flush=True)


def spk21_queries(n, seed=51):
    """Seeded query epochs inside the type-21 slice's coverage, and the FP64 flops each
    needs: the modified-difference interpolation at its record's orders plus the Sun's
    type-2 record (223) and the chain sums (6)."""
    from kete_b200 import synthetic

    (_, _, _, _, s0, s1, data), = synthetic.read_daf_segments(SPK21_SUBSET)
    nr, md = int(data[-1]), int(data[-2])
    rl = 4 * md + 11
    ep = data[nr * rl:nr * rl + nr]
    rng = np.random.default_rng(seed)
    jds = rng.uniform(s0 + 1.0, s1 - 1.0, n)
    rec = np.minimum(np.searchsorted(ep, jds, side="left"), nr - 1)
    m = data[rec * rl + 4 * md + 7]
    kq = sum(data[rec * rl + 4 * md + 8 + c] for c in range(3))
    flops = (3 * (m - 2) + m + 1.5 * (m - 2) * (m - 1) + 3 * (m - 2) + 4 * kq + 27 + 2 + 223 + 6)
    return jds / 86400.0 + 2451545.0, float(flops.sum())


def run_spk(args, world, rank, local):
    import ctypes

    import torch

    import kete_b200
    from kete_b200 import _lib, build, synthetic
    from oracle import oracle as O

    build.build()
    torch.cuda.set_device(local)
    kete_b200.init(local)
    td = tempfile.mkdtemp(prefix="kete_b200_bench_")
    spk = synthetic.write_synthetic_spk(os.path.join(td, "syn.bsp"))
    kete_b200.spice.kernel_reload([spk, SPK21_SUBSET])
    n = args.n or DEFAULT_N["spk_type21_1m"]
    jd, flops = spk21_queries(n, seed=51 + rank)
    dev = torch.device("cuda", local)
    L = _lib.lib()
    d_jd = torch.from_numpy(jd).to(dev)
    d_out = torch.empty((6, n), dtype=torch.float64, device=dev)
    d_st = torch.empty(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        _lib.check(L.kete_b200_spk_get_states(n, SPK21_ID, d_jd.data_ptr(), 0, 1, d_out.data_ptr(),
                                              d_st.data_ptr(), 1, ctypes.c_void_p(stream.cuda_stream)))

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        barrier(world)
        for k in range(args.steps):
            flush.zero_()
            evs[k][0].record(stream)
            step()
            evs[k][1].record(stream)
        torch.cuda.synchronize()
        barrier(world)
    t_total = reduce_max(sum(a.elapsed_time(b) for a, b in evs) * 1e-3, world)
    ms_step = 1e3 * t_total / args.steps
    value = world * n * args.steps / t_total
    # end to end from host arrays (copies inside)
    hj = torch.from_numpy(jd).pin_memory().numpy()
    t = time.perf_counter()
    for _ in range(args.steps):
        out6, st = kete_b200.spice.get_states_arrays(SPK21_ID, hj, 0, 1)
    e2e_s = reduce_max((time.perf_counter() - t) / args.steps, world)
    if rank != 0:
        return
    tflops_probe = ctypes_probe(_lib)
    achieved = flops / (ms_step * 1e-3) / 1e12
    O.spk_reset()
    for p in (spk, SPK21_SUBSET):
        with open(p, "rb") as f:
            O.spk_load_bytes(f.read())
    t = time.perf_counter()
    ref, rst = O.spk_get_states(SPK21_ID, jd, 0, 1)
    cpu_s = time.perf_counter() - t
    ok = (st == 0) & (rst == 0)
    rel = np.abs(out6 - ref).max(axis=0) / np.abs(ref).max(axis=0)
    line = {
        "metric": "SPK type-21 states/s", "value": value, "unit": "states/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic planets + a slice of a JPL type-21 asteroid segment",
        "config": {"workload": WORKLOADS["spk_type21_1m"].format(n=n), "n_queries_per_gpu": n,
                   "l2": "flushed (256 MB write) between timed steps"},
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": tflops_probe,
                     "unit": "TFLOP/s", "frac": achieved / tflops_probe, "traffic": None,
                     "flops_per_launch": flops,
                     "peak_source": "measured DFMA probe (kete_b200_fp64_probe) in this run"},
        "cpu_baseline": {"value": n / cpu_s, "unit": "states/s", "cores": os.cpu_count(),
                         "kind": "port", "sample": "the full workload, oracle on all host cores"},
        "e2e": {"value": world * n / e2e_s, "unit": "states/s", "h2d_bytes_per_step": 8 * n,
                "d2h_bytes_per_step": 52 * n},
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
        "parity": {"max_rel_err": float(rel[ok].max()) if ok.any() else None,
                   "objects_compared": int(ok.sum()),
                   "status_mismatches": int((st != rst).sum()), "tolerance_rel": 5e-14},
    }
    print(json.dumps(line), flush=True)


def run_long(args, world, rank, local):
    """propagate_n_body_long on the device: object-years/s of the test particles."""
    import torch

    import kete_b200
    from kete_b200 import _lib, build, synthetic
    from oracle import oracle as O

    build.build()
    torch.cuda.set_device(local)
    kete_b200.init(local)
    td = tempfile.mkdtemp(prefix="kete_b200_bench_")
    spk = synthetic.write_synthetic_spk(os.path.join(td, "syn.bsp"))
    kete_b200.spice.kernel_reload([spk])
    n = args.n or DEFAULT_N["nbody_long_10k"]
    pos, vel = synthetic.main_belt(n, seed=71 + rank)
    pos, vel = np.ascontiguousarray(synthetic.ecl_to_eq(pos)), np.ascontiguousarray(synthetic.ecl_to_eq(vel))
    jd1 = EPOCH + LONG_YEARS * 365.25
    dev = torch.device("cuda", local)
    P, V = torch.from_numpy(pos).to(dev), torch.from_numpy(vel).to(dev)
    _, _, pl, _ = kete_b200.propagate_n_body_long_arrays(pos[:, :1].copy(), vel[:, :1].copy(), EPOCH,
                                                         EPOCH)
    PL = torch.from_numpy(np.ascontiguousarray(pl)).to(dev)  # massive states at the epoch

    def step():
        return kete_b200.propagate_n_body_long_arrays(P, V, EPOCH, jd1, PL, None, 10)

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        barrier(world)
        for k in range(args.steps):
            flush.zero_()
            evs[k][0].record(stream)
            out = step()
            evs[k][1].record(stream)
        torch.cuda.synchronize()
        barrier(world)
    t_total = reduce_max(sum(a.elapsed_time(b) for a, b in evs) * 1e-3, world)
    units = n * LONG_YEARS
    value = world * units * args.steps / t_total
    t = time.perf_counter()
    hp = kete_b200.propagate_n_body_long_arrays(pos, vel, EPOCH, jd1, pl, None, 10)
    e2e_s = reduce_max(time.perf_counter() - t, world)
    if rank != 0:
        return
    gp = out[0].cpu().numpy()
    # CPU oracle on a bounded sample: the first 40 batches
    k = min(n, 400)
    O.spk_reset()
    with open(spk, "rb") as f:
        O.spk_load_bytes(f.read())
    t = time.perf_counter()
    op, ov, opl, ost = O.propagate_n_body_vec(pos[:, :k], vel[:, :k], EPOCH, jd1, planets=pl,
                                              batch_size=10)
    cpu_s = time.perf_counter() - t
    err = np.abs(gp[:, :k] - op).max()
    line = {
        "metric": "system-integration object-years/s", "value": value, "unit": "object-years/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t_total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS["nbody_long_10k"].format(n=n, years=LONG_YEARS),
                   "n_objects": n, "batch": 10,
                   "l2": "flushed (256 MB write) between timed steps"},
        "roofline": {"bound": "latency", "achieved": None, "peak": None, "unit": None,
                     "frac": None, "traffic": None,
                     "note": "one thread block per batch of 10 particles and 9 massive bodies; "
                             "the block-collective evaluations bound it, not a pipe"},
        "cpu_baseline": {"value": k * LONG_YEARS / cpu_s, "unit": "object-years/s",
                         "cores": os.cpu_count(), "kind": "port",
                         "sample": f"the first {k} objects ({k // 10} batches), oracle on all "
                                   "host cores"},
        "e2e": {"value": world * units / e2e_s, "unit": "object-years/s",
                "h2d_bytes_per_step": 48 * n, "d2h_bytes_per_step": 52 * n},
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
        "parity": {"max_err_au": float(err), "objects_compared": int(k), "tolerance_au": 1e-9,
                   "status_ok": bool((ost == 0).all() and (hp[3] == 0).all())},
    }
    print(json.dumps(line), flush=True)


def thermal_inputs(n, seed=61):
    """Seeded geometries and object parameters of the thermal workload."""
    from kete_b200 import flux

    rng = np.random.default_rng(seed)
    r = rng.uniform(1.0, 4.0, n)
    lon = rng.uniform(0, 2 * np.pi, n)
    lat = np.clip(rng.normal(0, np.radians(15.0), n), -1.4, 1.4)
    s2obj = np.stack([r * np.cos(lat) * np.cos(lon), r * np.cos(lat) * np.sin(lon), r * np.sin(lat)])
    lo = rng.uniform(0, 2 * np.pi, n)
    s2obs = np.stack([np.cos(lo), np.sin(lo), np.zeros(n)])
    pv = np.minimum(np.exp(np.log(0.14) + 0.6 * rng.normal(size=n)), 0.9)
    h = rng.uniform(8.0, 20.0, n)
    diam = flux.C_V / np.sqrt(pv) * 10.0 ** (-0.2 * h)
    return (np.ascontiguousarray(s2obj), np.ascontiguousarray(s2obs), h, pv, diam,
            np.ascontiguousarray(np.stack([pv] * 4)))


def thermal_args():
    from kete_b200 import flux

    return (np.array(flux.WISE_BANDS_300K), np.array(flux.WISE_SUN_CORRECTION),
            np.array(flux.WISE_ZERO_MAG_300K))


def run_reference_thermal(args):
    """FRM WISE-band fluxes on the CPU oracle over all host threads, bounded sample."""
    from oracle import oracle as O

    n = args.n or DEFAULT_N["thermal_wise_1m"]
    s2obj, s2obs, h, pv, diam, alb = thermal_inputs(n)
    bands, sc, zm = thermal_args()
    k = min(n, args.cpu_sample * 10)

    def step(m):
        O.thermal_batch(1, s2obj[:, :m], s2obs[:, :m], h[:m], 0.15, diam[:m], pv[:m], None, 0.9,
                        bands, alb[:, :m], sc, zm, True)

    for _ in range(args.warmup):
        step(min(k, 2000))
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        step(k)
        times.append(time.perf_counter() - t)
    total = float(np.sum(times))
    value = k * args.steps / total
    line = {
        "impl": "reference", "metric": "FRM WISE-band evaluations/s", "value": value,
        "unit": "geometries/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOADS["thermal_wise_1m"].format(n=n), "n_geometries": n},
        "cpu_baseline": {"value": value, "unit": "geometries/s", "cores": os.cpu_count(),
                         "kind": "port",
                         "sample": f"the first {k} geometries per step, oracle on all host "
                                   "threads; the reference Rust/rayon path cannot be built"},
        "e2e": {"value": value, "unit": "geometries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_thermal(args, world, rank, local):
    """FRM (and, beside it, NEATM) WISE-band fluxes of every geometry on the device."""
    import ctypes

    import torch

    import kete_b200
    from kete_b200 import _lib, build, flux
    from oracle import oracle as O

    build.build()
    torch.cuda.set_device(local)
    kete_b200.init(local)
    n = args.n or DEFAULT_N["thermal_wise_1m"]
    s2obj, s2obs, h, pv, diam, alb = thermal_inputs(n, seed=61 + rank)
    bands, sc, zm = thermal_args()
    dev = torch.device("cuda", local)
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in
         dict(s2obj=s2obj, s2obs=s2obs, h=h, g=np.full(n, 0.15), diam=diam, pv=pv,
              beam=np.ones(n), emis=np.full(n, 0.9), alb=alb).items()}
    outs = [torch.empty((4, n), dtype=torch.float64, device=dev) for _ in range(4)]
    vm, vf = (torch.empty(n, dtype=torch.float64, device=dev) for _ in range(2))
    bands_c, sc_c, zm_c = (np.ascontiguousarray(x) for x in (bands, sc, zm))
    stream = torch.cuda.current_stream(dev)
    L = _lib.lib()
    v = ctypes.c_void_p
    tail_t = [ctypes.c_int, v, v, v, v, ctypes.c_int] + [v] * 6 + [ctypes.c_int, v]
    L.kete_b200_frm.argtypes = [ctypes.c_int64] + [v] * 7 + tail_t
    L.kete_b200_neatm.argtypes = [ctypes.c_int64] + [v] * 8 + tail_t
    common = [d["s2obj"].data_ptr(), d["s2obs"].data_ptr(), d["h"].data_ptr(), d["g"].data_ptr(),
              d["diam"].data_ptr(), d["pv"].data_ptr()]
    tail = ([d["emis"].data_ptr(), 4, bands_c.ctypes.data, d["alb"].data_ptr(), sc_c.ctypes.data,
             zm_c.ctypes.data, 1] + [o.data_ptr() for o in outs] +
            [vm.data_ptr(), vf.data_ptr(), 1, v(stream.cuda_stream)])

    def frm():
        _lib.check(L.kete_b200_frm(n, *common, *tail))

    def neatm():
        _lib.check(L.kete_b200_neatm(n, *common, d["beam"].data_ptr(), *tail))

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        barrier(world)
        for k in range(args.steps):
            flush.zero_()
            evs[k][0].record(stream)
            fn()
            evs[k][1].record(stream)
        torch.cuda.synchronize()
        barrier(world)
        return reduce_max(sum(a.elapsed_time(b) for a, b in evs) * 1e-3, world)

    with ClockSampler(local) as clk:
        t_total = timed(frm)
    gfl = outs[0].cpu().numpy()
    t_neatm = timed(neatm)
    ms_step = 1e3 * t_total / args.steps
    value = world * n * args.steps / t_total
    # end to end through the public API from host arrays (copies inside)
    t = time.perf_counter()
    for _ in range(args.steps):
        r = flux.frm_arrays(s2obj, s2obs, h, 0.15, diam, pv, 0.9, bands, alb, sc, zm, True)
    e2e_s = reduce_max((time.perf_counter() - t) / args.steps, world)
    if rank != 0:
        return
    k = min(n, args.cpu_sample)
    t = time.perf_counter()
    ref = O.thermal_batch(1, s2obj[:, :k], s2obs[:, :k], h[:k], 0.15, diam[:k], pv[:k], None, 0.9,
                          bands, alb[:, :k], sc, zm, True)
    cpu_s = time.perf_counter() - t
    rel = np.abs(gfl[:, :k] / ref["fluxes"] - 1.0).max()
    e2e_rel = np.abs(r["fluxes"][:, :k] / ref["fluxes"] - 1.0).max()
    line = {
        "metric": "FRM WISE-band evaluations/s", "value": value, "unit": "geometries/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOADS["thermal_wise_1m"].format(n=n), "n_geometries_per_gpu": n,
                   "l2": "flushed (256 MB write) between timed steps"},
        "roofline": {"bound": "fp64-transcendental", "achieved": None, "peak": None, "unit": None,
                     "frac": None, "traffic": None, "fp64_pipe_active_ncu": THERMAL_FP64_PIPE,
                     "note": "one exp per seen facet and band dominates and has no fixed flop "
                             "count; the FP64 pipe is busy 56 % of the kernel's cycles with "
                             "instruction issue the limit (ncu, 20k geometries)"},
        "neatm_same_inputs": {"ms_per_step": 1e3 * t_neatm / args.steps,
                              "value": world * n * args.steps / t_neatm, "unit": "geometries/s"},
        "cpu_baseline": {"value": k / cpu_s, "unit": "geometries/s", "cores": os.cpu_count(),
                         "kind": "port",
                         "sample": f"the first {k} geometries, oracle on all host threads"},
        "e2e": {"value": world * n / e2e_s, "unit": "geometries/s",
                "h2d_bytes_per_step": 8 * n * 16, "d2h_bytes_per_step": 8 * n * 18},
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
        "parity": {"max_rel_err": float(rel), "e2e_max_rel_err": float(e2e_rel),
                   "geometries_compared": int(k), "tolerance_rel": 1e-12},
    }
    print(json.dumps(line), flush=True)


def stm_inputs(n, seed=81):
    """Seeded main-belt states, spans and symmetric positive covariances."""
    from kete_b200 import synthetic

    pos, vel = synthetic.main_belt(n, seed=seed)
    rng = np.random.default_rng(seed + 1)
    jd0 = np.full(n, EPOCH)
    jd1 = EPOCH + rng.uniform(-1000.0, 1000.0, n)
    sig = np.array([1e-6] * 3 + [1e-8] * 3)
    a = rng.normal(size=(6, 6, n)) * sig[:, None, None]
    cov = np.ascontiguousarray(np.einsum("ikn,jkn->ijn", a, a))
    return (np.ascontiguousarray(pos), np.ascontiguousarray(vel), jd0, jd1, cov)


def run_reference_stm(args):
    """The corrected variational equations on kete's RK4(5) (the oracle), one thread."""
    from oracle import oracle as O

    n = args.n or DEFAULT_N["stm_cov_1m"]
    pos, vel, jd0, jd1, cov = stm_inputs(min(n, 5000))
    k = min(n, 2000)

    def step(m):
        for i in range(m):
            _, _, phi = O.compute_stm(pos[:, i], vel[:, i], jd0[i], jd1[i])
            phi @ cov[:, :, i] @ phi.T

    for _ in range(args.warmup):
        step(min(k, 50))
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        step(k)
        times.append(time.perf_counter() - t)
    total = float(np.sum(times))
    value = k * args.steps / total
    line = {
        "impl": "reference", "metric": "two-body STM + covariance objects/s", "value": value,
        "unit": "objects/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS["stm_cov_1m"].format(n=n), "n_objects": n},
        "cpu_baseline": {"value": value, "unit": "objects/s", "cores": 1, "kind": "port",
                         "sample": f"the first {k} objects per step, one thread (kete's "
                                   "compute_stm is one call per state); the reference "
                                   "Rust path cannot be built"},
        "e2e": {"value": value, "unit": "objects/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_stm(args, world, rank, local):
    """Two-body STMs with covariance propagation of every object on the device."""
    import torch

    import kete_b200
    from kete_b200 import build, state_transition
    from oracle import oracle as O

    build.build()
    torch.cuda.set_device(local)
    kete_b200.init(local)
    n = args.n or DEFAULT_N["stm_cov_1m"]
    pos, vel, jd0, jd1, cov = stm_inputs(n, seed=81 + rank)
    dev = torch.device("cuda", local)
    P, V, J0, J1, Cv = (torch.from_numpy(x).to(dev) for x in (pos, vel, jd0, jd1, cov))
    stream = torch.cuda.current_stream(dev)

    def step():
        return state_transition.compute_stm_arrays(P, V, J0, J1, 1.0, Cv)

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        barrier(world)
        for k in range(args.steps):
            flush.zero_()
            evs[k][0].record(stream)
            out = step()
            evs[k][1].record(stream)
        torch.cuda.synchronize()
        barrier(world)
    t_total = reduce_max(sum(a.elapsed_time(b) for a, b in evs) * 1e-3, world)
    ms_step = 1e3 * t_total / args.steps
    value = world * n * args.steps / t_total
    t = time.perf_counter()
    for _ in range(args.steps):
        hp = state_transition.compute_stm_arrays(pos, vel, jd0, jd1, 1.0, cov)
    e2e_s = reduce_max((time.perf_counter() - t) / args.steps, world)
    if rank != 0:
        return
    m = out[2].cpu().numpy()
    k = min(n, 300)
    t = time.perf_counter()
    err = 0.0
    for i in range(k):
        _, _, ref = O.compute_stm(pos[:, i], vel[:, i], jd0[i], jd1[i])
        err = max(err, float(np.abs(m[:, :, i] - ref).max() / np.abs(ref).max()))
    cpu_s = time.perf_counter() - t
    peak = measured_peaks().get("hbm_gbs")
    achieved = STM_BYTES_PER_OBJECT * n / (ms_step * 1e-3) / 1e9
    line = {
        "metric": "two-body STM + covariance objects/s", "value": value, "unit": "objects/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOADS["stm_cov_1m"].format(n=n), "n_objects": n,
                   "l2": "flushed (256 MB write) between timed steps"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if peak else None, "traffic": None,
                     "bytes_per_object": STM_BYTES_PER_OBJECT,
                     "note": "algorithmic bytes over the kernel time; the dual-number leaf "
                             "Jacobians make it FP64/latency-bound (ncu: 31.6% FP64 pipe)"},
        "cpu_baseline": {"value": k / cpu_s, "unit": "objects/s", "cores": 1, "kind": "port",
                         "sample": f"the first {k} objects, one thread"},
        "e2e": {"value": world * n / e2e_s, "unit": "objects/s",
                "h2d_bytes_per_step": 8 * 44 * n, "d2h_bytes_per_step": (8 * 78 + 4) * n},
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
        "parity": {"max_rel_err_vs_oracle": err, "objects_compared": k, "tolerance_rel": 2e-8,
                   "status_ok": bool((hp[4] == 0).all())},
    }
    print(json.dumps(line), flush=True)


def ctypes_probe(_lib):
    import ctypes

    L = _lib.lib()
    L.kete_b200_fp64_probe.argtypes = [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    out = ctypes.c_double()
    ms = ctypes.c_float()
    _lib.check(L.kete_b200_fp64_probe(20000, ctypes.byref(out), ctypes.byref(ms)))
    return out.value


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="kete_b200", choices=["kete_b200", "reference"])
    ap.add_argument("--n", type=int, default=0, help="objects (0 = the workload's size)")
    ap.add_argument("--workload", default="nbody_mixed_1m", choices=sorted(WORKLOADS))
    ap.add_argument("--mode", type=int, default=0, help="0 = autotune, 1 = thread, 2 = nodes")
    ap.add_argument("--variant", type=int, default=0)
    ap.add_argument("--refill", type=int, default=0)
    ap.add_argument("--fields", type=int, default=SURVEY_FIELDS, help="survey workload: fields")
    ap.add_argument("--cpu-sample", type=int, default=20000,
                    help="survey workload: objects in the CPU oracle's sample")
    ap.add_argument("--no-graph", action="store_true",
                    help="time direct launches instead of a captured CUDA graph")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the gradient-cost measurement on the differentiation workload")
    args = ap.parse_args()
    world, rank, local = dist_setup() if args.impl == "kete_b200" else (
        int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0)
    if args.impl == "reference":
        run_reference(args, world, rank)
    elif args.workload == "survey_10m":
        run_survey(args, world, rank, local)
    elif args.workload == "spk_type21_1m":
        run_spk(args, world, rank, local)
    elif args.workload == "nbody_long_10k":
        run_long(args, world, rank, local)
    elif args.workload == "thermal_wise_1m":
        run_thermal(args, world, rank, local)
    elif args.workload == "stm_cov_1m":
        run_stm(args, world, rank, local)
    elif args.workload == "adjoint_4k":
        run_adjoint(args, world, rank, local)
    else:
        run_gpu(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
