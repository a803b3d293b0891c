#!/usr/bin/env python
"""Benchmark: FP64 Gauss-Radau N-body propagation throughput (object-years/s) on B200.

Workload (default): the plain N-body configuration -- 10,000 seeded main-belt states
propagated 365.25 days under the Sun, eight planets and the Moon read from a seeded
synthetic SPK type-2 ephemeris (degree-13 Chebyshev records).  One step = one propagation
of the whole population.  ``value`` is device-resident throughput (inputs already in HBM,
one kernel launch per step, CUDA-event timed, L2 flushed between steps); ``e2e`` is the
same through the public C ABI with pinned host buffers (host->device and device->host
copies inside the timed region).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl kete_b200|reference]

With N > 1 (torchrun) every rank propagates its own population (weak scaling, no data
exchange); the time is the maximum over ranks.  ``--impl reference`` times the CPU
restatement of kete's path (the oracle) on all host cores on the same workload.
"""
from __future__ import annotations

import argparse
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
# records: positions and velocities of the Sun and Jupiter (2 x 223: their velocities enter
# the relativistic and non-gravitational terms), positions of the other 9 records (9 x 108),
# Earth/Moon + barycentre (6), 10 Newtonian terms (10 x 19) with 2 relative velocities (6),
# relativistic terms (2 x 34), solar/Jovian J2 (2 x 42), Earth J2 (30).
FLOPS_PER_EVAL = 1802
FLOPS_PER_ITER = 7 * FLOPS_PER_EVAL + 1201  # 7 node evaluations + predictor/g/b/test
FLOPS_PER_STEP = 120       # state update + step-size control


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
}
DEFAULT_N = {"nbody_mba_10k": 10_000, "nbody_mixed_1m": 1_000_000, "kepler_100k": 100_000}


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


def run_reference(args, world, rank):
    if rank != 0:
        return
    from kete_b200 import synthetic

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
        "config": {"workload": WORKLOADS[kind].format(n=n), "n_objects": n},
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
            best, sweep = tune.autotune(d["pos"], d["vel"], d["jd0"], d["jd1"], nongrav=d.get("ng"))
        else:
            best = dict(mode=args.mode, variant=args.variant, refill=args.refill)
            tune.set_config(**best)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step(arrs):
        if nbody:
            return kete_b200.propagate_n_body_arrays(arrs["pos"], arrs["vel"], arrs["jd0"],
                                                     arrs["jd1"], nongrav=arrs.get("ng"),
                                                     mode=best["mode"])
        return kete_b200.propagate_two_body_arrays(arrs["pos"], arrs["vel"], arrs["jd0"],
                                                   arrs["jd1"])

    flops = None
    steps_total = iters_total = 0
    if nbody:  # counts for the flop model (deterministic: same inputs every step)
        _, _, _, det = kete_b200.propagate_n_body_arrays(d["pos"], d["vel"], d["jd0"], d["jd1"],
                                                         nongrav=d.get("ng"), mode=best["mode"],
                                                         with_details=True)
        cnt = det["counters"].to(torch.int64).sum(dim=1).cpu().numpy()
        steps_total, iters_total, exact_total = (int(x) for x in cnt)
        flops = (iters_total * FLOPS_PER_ITER + exact_total * FLOPS_PER_EVAL +
                 steps_total * FLOPS_PER_STEP)
    launches_per_step = (3 if (nbody and best.get("refill")) else 0) + 1

    for _ in range(args.warmup):
        step(d)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()  # write > L2 (126 MB) between steps, outside the timed pair
            evs[k][0].record(stream)
            step(d)
            evs[k][1].record(stream)
        torch.cuda.synchronize()
        barrier(world)
    ms = [a.elapsed_time(b) for a, b in evs]
    t_total = reduce_max(float(np.sum(ms)) * 1e-3, world)
    ms_step = 1e3 * t_total / args.steps
    value = world * units * args.steps / t_total

    # end to end through the C ABI with pinned host buffers
    hp = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in host.items()}
    hnp = {k: v.numpy() for k, v in hp.items()}
    step(hnp)
    e2e_t = []
    out = None
    for _ in range(args.steps):
        t = time.perf_counter()
        out = step(hnp)
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
        roof = {"bound": "fp64", "achieved": achieved, "peak": tflops_probe, "unit": "TFLOP/s",
                "frac": achieved / tflops_probe if tflops_probe else None, "traffic": None,
                "peak_source": "measured DFMA probe (kete_b200_fp64_probe) in this run",
                "flops_per_launch": flops, "hbm_bytes_algorithmic": hbm_bytes}
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
    gp = out[0][:, idx]
    gst = (out[2] if nbody else out[3])[idx]
    err = np.linalg.norm(gp - op, axis=0)
    ok = (gst == 0) & (st_cpu == 0)
    tol = 1e-9 if nbody else 1e-12
    line = {
        "metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS[kind].format(n=n), "n_objects_per_gpu": n,
                   "launch": best, "autotune_sweep_ms": sweep,
                   "l2": "flushed (256 MB write) between timed steps",
                   "parallelism": f"replicas x{world} (objects independent)"},
        "roofline": roof,
        "cpu_baseline": {"value": cpu_units / cpu_dt, "unit": unit, "cores": cores,
                         "kind": "port",
                         "sample": ("the full workload" if len(idx) == n else
                                    f"seeded 1% subsample ({len(idx)} objects)") +
                                   ", oracle (C restatement of kete's FP64 path) with OpenMP on "
                                   "all host cores"},
        "e2e": {"value": e2e_value, "unit": unit, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": args.steps * launches_per_step,
        "clocks": clk.summary(),
        "parity": {"max_err_au": float(err[ok].max()) if ok.any() else None,
                   "objects_compared": int(ok.sum()),
                   "status_mismatches": int((gst != st_cpu).sum()),
                   "gpu_status_counts": np.bincount(gst, minlength=8).tolist(),
                   "cpu_status_counts": np.bincount(st_cpu, minlength=8).tolist(),
                   "tolerance_au": tol},
    }
    if nbody:
        line["object_steps_per_s"] = world * steps_total * args.steps / t_total
        line["corrector_iterations_per_step"] = iters_total / max(steps_total, 1)
    if kind == "nbody_mba_10k" and not args.no_adjoint:
        line["adjoint"] = adjoint_section(dev, max(1, args.warmup), max(1, min(args.steps, 3)))
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
    ap.add_argument("--workload", default="nbody_mba_10k", choices=sorted(WORKLOADS))
    ap.add_argument("--mode", type=int, default=0, help="0 = autotune, 1 = thread, 2 = nodes")
    ap.add_argument("--variant", type=int, default=0)
    ap.add_argument("--refill", type=int, default=0)
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the gradient-cost measurement on the differentiation workload")
    args = ap.parse_args()
    world, rank, local = dist_setup() if args.impl == "kete_b200" else (
        int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0)
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_gpu(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
