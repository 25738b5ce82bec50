#!/usr/bin/env python
"""Benchmark: greedy-fluid registration iterations at 128^3 on B200.

Metric: 128^3 fluid iterations/s (whole job, all ranks) with the achieved
HBM GB/s of the dominant kernel against the measured B200 copy bandwidth.

Workload (one "step"): every rank holds 4 independent 128^3 pairs resident
in HBM (config-2 generator: 16 Gaussian blobs + N(0, 0.02^2) noise, smooth
warp with max |u| = 6 voxels; alpha = beta = 0.01, gamma = 0.001,
MaxPert 0.5) and runs 2 greedy iterations on each pair, so a step is 8
iterations; each pair's iterations run on its own stream (a batch of
independent registrations, as an atlas or a registration service runs
them). The 4 pairs' working sets (~120 MB each) exceed the 126 MB L2,
so consecutive steps find none of their data in L2.

Pair registrations are independent: with N GPUs every rank runs its own
pairs (replicas, weak scaling); the only collective is the max of the
per-rank device times.

--impl reference times the reference's own CPU implementation
(GreedyIteratorCPU, built from its sources into oracle/_ref) on the host
cores, one 128^3 pair per thread.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 128
PAIRS = 4
ITERS_PER_PAIR = 2
ALPHA, BETA, GAMMA, MAX_PERT = 0.01, 0.01, 0.001, 0.5
E2E_ITERS = 25  # the 128^3 level of the 3-level multiscale config

# algorithmic HBM bytes per voxel of each kernel of one iteration (minimum
# traffic of that kernel's function; spectrum = 3 complex64 x (nx/2+1)/nx)
SPEC = 3 * 8 * (N // 2 + 1) / N  # bytes/voxel of the 3-channel half spectrum
STAGE_NAMES = ["force_prep", "energy", "xy_forward_fft", "z_solve", "xy_inverse_fft",
               "max_norm", "update", "xy_inverse_update"]
STAGE_BYTES = {
    "force_prep": 12 + 4 + 4 + 4,        # h, I1, I0 gather (once), I0(h) write
    "energy": 0,
    "xy_forward_fft": 4 + 4 + SPEC,      # I0(h), I1, spectrum write
    "z_solve": 2 * SPEC,                 # spectrum read + write
    "xy_inverse_fft": SPEC + 12,         # spectrum read, v write
    "max_norm": 12,
    "update": 12 + 12 + 12,              # v, h gather (once), h' write
    "xy_inverse_update": SPEC + 12 + 12,  # spectrum read, h gather (once), h' write
}
B_ITER = 92  # bytes/voxel of the fully fused 3-pass greedy iteration (each stream once)
B_ITER_INV = B_ITER + 36  # with h^-1: its read and write, v gathered at h^-1


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200",
                                          "-i", str(self.index)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_iteration_rate(I0, I1, iters=4):
    """Reference CPU (oracle/_ref) or, without it, the oracle port: steady-
    state 128^3 greedy iterations on one host thread, after the handle and
    iteration 0 (step update) are built untimed. Returns (iters/s, kind)."""
    from oracle import REF_SO, Oracle, Reference, identity
    if os.path.exists(REF_SO):
        ref = Reference()
        h = ref.greedy_open(I0, I1, max_pert=MAX_PERT, alpha=ALPHA, beta=BETA, gamma=GAMMA)
        t = time.perf_counter()
        ref.greedy_iterate(h, iters)
        dt = time.perf_counter() - t
        ref.greedy_close(h)
        return iters / dt, "reference"
    o = Oracle()
    h = identity(I0.shape)
    _, st = o.greedy_iterate(I0, I1, h, None, max_pert=MAX_PERT, alpha=ALPHA, beta=BETA,
                             gamma=GAMMA, update_step=True)
    t = time.perf_counter()
    for _ in range(iters):
        o.greedy_iterate(I0, I1, h, None, max_pert=MAX_PERT, alpha=ALPHA, beta=BETA, gamma=GAMMA,
                         step=st)
    return iters / (time.perf_counter() - t), "port"


def make_pair(seed):
    from atlaswerks_b200.synth import greedy_pair
    return greedy_pair((N, N, N), seed, n_blobs=16, umax=6.0, noise_sd=0.02)


def config(extra=None):
    c = {"workload": f"greedy-fluid pair registration, {N}^3 float32, single scale "
                     f"(finest level of the 3-level config), {PAIRS} resident pairs x "
                     f"{ITERS_PER_PAIR} iterations per step, one stream per pair",
         "grid": [N, N, N], "alpha": ALPHA, "beta": BETA, "gamma": GAMMA, "max_pert": MAX_PERT,
         "pairs_per_rank": PAIRS, "iterations_per_step_per_rank": PAIRS * ITERS_PER_PAIR,
         "l2": "inputs larger than L2: 4 pairs x ~120 MB working set, concurrent",
         "inverse_field": False}
    if extra:
        c.update(extra)
    return c


def run_reference(args):
    """CPU reference arm: the reference's GreedyIteratorCPU (oracle/_ref) on
    all host threads, one 128^3 pair each (capped at 32 for memory). Each
    thread builds its data object, iterator and FFT plans and runs iteration
    0 (the step update) before the timed region; a step is one further
    steady-state iteration of every thread's pair, the GPU arm's unit of
    work. --warmup steps run untimed first, as in the GPU arm."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import REF_SO, Oracle, Reference, identity
    kind = "reference" if os.path.exists(REF_SO) else "port"
    cores = max(1, min(os.cpu_count() or 1, 32))
    pairs = [make_pair(1000 + t) for t in range(cores)]
    if kind == "reference":
        ref = Reference()
        handles = [None] * cores

        def opener(t):
            handles[t] = ref.greedy_open(*pairs[t], max_pert=MAX_PERT, alpha=ALPHA, beta=BETA,
                                         gamma=GAMMA)

        def worker(t):
            ref.greedy_iterate(handles[t], 1)
    else:
        o = Oracle()
        state = [None] * cores

        def opener(t):
            I0, I1 = pairs[t]
            h = identity(I0.shape)
            _, st = o.greedy_iterate(I0, I1, h, None, max_pert=MAX_PERT, alpha=ALPHA, beta=BETA,
                                     gamma=GAMMA, update_step=True)
            state[t] = (h, st)

        def worker(t):
            I0, I1 = pairs[t]
            h, st = state[t]
            o.greedy_iterate(I0, I1, h, None, max_pert=MAX_PERT, alpha=ALPHA, beta=BETA,
                             gamma=GAMMA, step=st)

    def parallel(fn):
        th = [threading.Thread(target=fn, args=(t,)) for t in range(cores)]
        for x in th:
            x.start()
        for x in th:
            x.join()

    parallel(opener)
    warmup = max(args.warmup, 3)
    for _ in range(warmup):
        parallel(worker)
    t = time.perf_counter()
    for _ in range(args.steps):
        parallel(worker)
    dt = time.perf_counter() - t
    if kind == "reference":
        for h in handles:
            ref.greedy_close(h)
    value = args.steps * cores / dt
    line = {"metric": "128^3 fluid iters/s", "value": value, "unit": "iters/s",
            "impl": "reference", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
            "steps": args.steps, "warmup": warmup,
            "ms_per_step": 1000 * dt / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded blobs + smooth warp)",
            "config": config({"pairs_per_rank": cores, "iterations_per_step_per_rank": cores,
                              "workload": f"greedy-fluid pair registration, {N}^3 float32, one "
                                          f"steady-state iteration of one pair per host thread "
                                          f"per step (handles built and iteration 0 run before "
                                          f"the timed region)"}),
            "fft": "the reference's DiffOper over an FP64 FFTW-API shim: FFTW is not installed, "
                   "so single-precision FFTW would be faster than this arm",
            "cpu_baseline": {"value": value, "unit": "iters/s", "cores": cores, "kind": kind,
                             "sample": f"{args.steps} steps x {cores} threads x 1 steady-state "
                                       f"iteration of a {N}^3 pair (GreedyIteratorCPU; FFT = "
                                       f"FP64 shim, not FFTW)"},
            "e2e": {"value": value, "unit": "iters/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_b200(args):
    import numpy as np
    import torch

    from atlaswerks_b200 import _lib
    from atlaswerks_b200.greedy import (DiffOperParam, GreedyDeformationDataB200,
                                        GreedyIteratorB200, GreedyIteratorParam)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    _lib.lib()
    param = GreedyIteratorParam(DiffOperParam(ALPHA, BETA, GAMMA), MAX_PERT)
    iters, datas = [], []
    host_pairs = []
    for p in range(PAIRS):
        I0, I1 = make_pair(rank * 100 + p)
        host_pairs.append((I0, I1))
        it = GreedyIteratorB200((N, N, N))
        it.SetScaleLevel((N, N, N), (1.0, 1.0, 1.0), param)
        if args.fast_interp:
            it.SetFastInterpolation(True)
        d = GreedyDeformationDataB200(torch.from_numpy(I0).cuda(), torch.from_numpy(I1).cuda())
        it.Run(d, 1, update_first=True)
        iters.append(it)
        datas.append(d)
    stream = torch.cuda.current_stream()
    # each pair runs on its own stream, so one pair's kernels fill the SMs
    # that another pair's kernel leaves idle (tails, single-wave grids)
    pair_streams = [torch.cuda.Stream() for _ in range(PAIRS)]

    def step():
        fork = torch.cuda.Event()
        fork.record(stream)
        joins = []
        for it, d, ps in zip(iters, datas, pair_streams):
            ps.wait_event(fork)
            with torch.cuda.stream(ps):
                it.Run(d, ITERS_PER_PAIR, update_first=False)
                j = torch.cuda.Event()
                j.record(ps)
            joins.append(j)
        for j in joins:
            stream.wait_event(j)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()

    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        start.record(stream)
        for _ in range(args.steps):
            step()
        end.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = start.elapsed_time(end)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    per_rank_iters = args.steps * PAIRS * ITERS_PER_PAIR
    value = world * per_rank_iters / (ms / 1000.0)
    ms_per_step = ms / args.steps
    ms_per_iter = ms / per_rank_iters

    # --- the same iterations maintaining the inverse field h^-1 too (the
    # reference's default: WriteInvDefField, GreedyWarpParam.h:31): 36 more
    # algorithmic bytes per voxel (h^-1 read, v gathered at h^-1, h^-1' write)
    inv_datas = []
    for it, (I0h, I1h) in zip(iters, host_pairs):
        di = GreedyDeformationDataB200(torch.from_numpy(I0h).cuda(), torch.from_numpy(I1h).cuda(),
                                       compute_inverse=True)
        it.Run(di, 1, update_first=True)
        inv_datas.append(di)

    def inv_step():
        fork = torch.cuda.Event()
        fork.record(stream)
        joins = []
        for it, d, ps in zip(iters, inv_datas, pair_streams):
            ps.wait_event(fork)
            with torch.cuda.stream(ps):
                it.Run(d, ITERS_PER_PAIR, update_first=False)
                j = torch.cuda.Event()
                j.record(ps)
            joins.append(j)
        for j in joins:
            stream.wait_event(j)

    for _ in range(3):
        inv_step()
    torch.cuda.synchronize()
    inv_steps = max(args.steps // 2, 5)
    i0 = torch.cuda.Event(enable_timing=True)
    i1 = torch.cuda.Event(enable_timing=True)
    i0.record(stream)
    for _ in range(inv_steps):
        inv_step()
    i1.record(stream)
    torch.cuda.synchronize()
    inv_ms = i0.elapsed_time(i1)
    if dist:
        t = torch.tensor([inv_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        inv_ms = float(t.item())
    inv_value = world * inv_steps * PAIRS * ITERS_PER_PAIR / (inv_ms / 1000.0)
    del inv_datas

    # --- per-kernel roofline (pair 0, each stage timed alone with events) ---
    peak, peak_kind = peaks()
    it0, d0 = iters[0], datas[0]
    h, ho = d0.Def1To0(), d0._next()[0]
    ms_stage = (ctypes.c_float * len(STAGE_NAMES))()
    z = [None, None, None]
    _lib.check(_lib.lib().aw_greedy_profile(
        it0._h, d0.I0.data_ptr(), d0.I1.data_ptr(), *[t.data_ptr() for t in h],
        *[t.data_ptr() for t in ho], *z, *z, 20, stream.cuda_stream, ms_stage))
    stage_ms = {n: float(ms_stage[i]) for i, n in enumerate(STAGE_NAMES)}
    # a steady-state iteration (no step update, no inverse field): the
    # inverse transform and the update run as one kernel
    per_iter_stages = ["force_prep", "energy", "xy_forward_fft", "z_solve", "xy_inverse_update"]
    dom = max(per_iter_stages, key=lambda n: stage_ms[n])
    nvox = N ** 3
    dom_bytes = STAGE_BYTES[dom] * nvox
    achieved = dom_bytes / (stage_ms[dom] / 1000.0) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "greedy_128_dram_traffic.json")
    if os.path.exists(tfile):
        traffic = json.load(open(tfile)).get(dom)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                "algorithmic_bytes_per_launch": dom_bytes,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs, burst copy)"
                if peak_kind == "measured" else "fallback 6.65 TB/s"}
    iter_gbs = B_ITER * nvox / (ms_per_iter / 1000.0) / 1e9
    iteration_roofline = {"bytes_per_iteration": B_ITER * nvox, "achieved": iter_gbs,
                          "peak": peak, "unit": "GB/s", "frac": iter_gbs / peak,
                          "stage_ms": stage_ms}
    inv_gbs = B_ITER_INV * nvox * (inv_value / world) / 1e9
    inverse_field = {"value": inv_value, "unit": "iters/s", "steps": inv_steps,
                     "bytes_per_iteration": B_ITER_INV * nvox, "achieved": inv_gbs,
                     "peak": peak, "frac": inv_gbs / peak,
                     "workload": "the same pairs and iterations, h^-1 updated too "
                                 "(composeVHInv, PARTIAL_ZERO)"}

    # --- end to end through the public API with host buffers ---
    # a step registers PAIRS pairs from pinned host memory, each on its own
    # stream (H2D of I0 and I1, identity init, E2E_ITERS iterations with the
    # step update at iteration 0, D2H of h), so one pair's copies overlap the
    # others' iterations, as a registration service runs them
    e2e = None
    if rank == 0 or world > 1:
        jobs = []
        for p in range(PAIRS):
            I0d = torch.empty((N, N, N), device="cuda")
            I1d = torch.empty((N, N, N), device="cuda")
            it = GreedyIteratorB200((N, N, N))
            it.SetScaleLevel((N, N, N), (1.0, 1.0, 1.0), param)
            if args.fast_interp:
                it.SetFastInterpolation(True)
            jobs.append({"I0h": torch.from_numpy(host_pairs[p][0]).pin_memory(),
                         "I1h": torch.from_numpy(host_pairs[p][1]).pin_memory(),
                         "hh": torch.empty((3, N, N, N), dtype=torch.float32).pin_memory(),
                         "I0d": I0d, "I1d": I1d, "it": it,
                         "de": GreedyDeformationDataB200(I0d, I1d),
                         "s": torch.cuda.Stream()})

        # the pairs' uploads go one pair after another on one copy stream,
        # so the first pair computes while the others' images still cross
        # the bus (issued together, they would share it and land together)
        copy_stream = torch.cuda.Stream()

        def e2e_step():
            fork = torch.cuda.Event()
            fork.record(stream)
            copy_stream.wait_event(fork)
            landed = []
            with torch.cuda.stream(copy_stream):
                for j in jobs:
                    j["I0d"].copy_(j["I0h"], non_blocking=True)
                    j["I1d"].copy_(j["I1h"], non_blocking=True)
                    ev = torch.cuda.Event()
                    ev.record(copy_stream)
                    landed.append(ev)
            joins = []
            for j, ready in zip(jobs, landed):
                j["s"].wait_event(fork)
                with torch.cuda.stream(j["s"]):
                    j["de"].SetToIdentity()
                    j["s"].wait_event(ready)
                    j["it"].Run(j["de"], E2E_ITERS, update_first=True)
                    j["hh"].copy_(j["de"].Def1To0(), non_blocking=True)
                    ev = torch.cuda.Event()
                    ev.record(j["s"])
                joins.append(ev)
            for ev in joins:
                stream.wait_event(ev)

        for _ in range(2):
            e2e_step()
        torch.cuda.synchronize()
        reps = 3
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(reps):
            e2e_step()
        s1.record(stream)
        torch.cuda.synchronize()
        ems = s0.elapsed_time(s1) / reps
        e2e_val = PAIRS * E2E_ITERS / (ems / 1000.0)
        if dist:
            t = torch.tensor([ems], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_val = world * PAIRS * E2E_ITERS / (float(t.item()) / 1000.0)
        e2e = {"value": e2e_val, "unit": "iters/s", "h2d_bytes_per_step": PAIRS * 2 * 4 * nvox,
               "d2h_bytes_per_step": PAIRS * 3 * 4 * nvox,
               "step": f"{PAIRS} pairs, each on its own stream: H2D of I0, I1 (pinned; the "
                       f"pairs' uploads in order on one copy stream) + identity init + "
                       f"{E2E_ITERS}-iteration registration (step update at iteration 0) + "
                       f"D2H of h, via GreedyIteratorB200.Run"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, kind = cpu_reference_iteration_rate(*host_pairs[0], iters=4)
        cpu = {"value": rate, "unit": "iters/s", "cores": 1, "kind": kind,
               "sample": f"4 steady-state greedy iterations of one {N}^3 pair on 1 host thread "
                         f"(GreedyIteratorCPU{'' if kind == 'reference' else ' port'}; FFT = "
                         f"FP64 shim, not FFTW)"}

    # five launches per steady-state iteration: force-prep, energy,
    # xy-forward, z-solve, xy-inverse fused with the update
    launches = 5 * per_rank_iters
    line = {"metric": "128^3 fluid iters/s", "value": value, "unit": "iters/s",
            "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3),
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Gaussian blobs + smooth random warp, no dataset)",
            "config": config({"interpolation": "float fused multiply-add trees (fast mode)"
                              if args.fast_interp else "double weights and sums (bit-exact)"}),
            "roofline": roofline,
            "iteration_roofline": iteration_roofline, "inverse_field": inverse_field,
            "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk.summary()}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


def run_ncu_case(args):
    """A short, untimed workload for ncu captures: one 128^3 pair, a step
    update, then `--steps` iterations through the graph path (with
    --workload ldmm: `--steps` LDMM IterateNew iterations at 128^3, T = 10,
    sigma 1, step 0.01; with --workload adshoot: `--steps` adjoint shooting
    iterations at 128^3, T = 5, sigma 1, step 0.0002)."""
    import torch
    if args.workload == "ldmm":
        from atlaswerks_b200.ldmm import ldmm_register
        from atlaswerks_b200.synth import greedy_pair
        I0, I1 = greedy_pair((N, N, N), 7, 8, 3.0)
        ldmm_register(torch.from_numpy(I0).cuda(), torch.from_numpy(I1).cuda(), 10, args.steps,
                      sigma=1.0, step=0.01)
        torch.cuda.synchronize()
        print(json.dumps({"ncu_case": "ldmm 128^3 T=10", "iterations": args.steps}))
        return 0
    if args.workload == "adshoot":
        from atlaswerks_b200.greedy import DiffOperParam
        from atlaswerks_b200.ldmm import LDMMIteratorParam
        from atlaswerks_b200.shooting import LDMMAdShootingIteratorB200, LDMMShootingDefDataB200
        from atlaswerks_b200.synth import greedy_pair
        I0, I1 = greedy_pair((N, N, N), 7, 8, 3.0)
        it = LDMMAdShootingIteratorB200((N, N, N), n_time_steps=5)
        it.SetScaleLevel((N, N, N), (1.0, 1.0, 1.0),
                         LDMMIteratorParam(DiffOperParam(ALPHA, BETA, GAMMA), 1.0, 0.0002, False))
        data = LDMMShootingDefDataB200(torch.from_numpy(I0).cuda(), torch.from_numpy(I1).cuda())
        for _ in range(args.steps):
            it.Iterate(data)
        torch.cuda.synchronize()
        print(json.dumps({"ncu_case": "adshoot 128^3 T=5", "iterations": args.steps}))
        return 0

    from atlaswerks_b200.greedy import (DiffOperParam, GreedyDeformationDataB200,
                                        GreedyIteratorB200, GreedyIteratorParam)
    I0, I1 = make_pair(0)
    it = GreedyIteratorB200((N, N, N))
    it.SetScaleLevel((N, N, N), (1.0, 1.0, 1.0),
                     GreedyIteratorParam(DiffOperParam(ALPHA, BETA, GAMMA), MAX_PERT))
    if args.fast_interp:
        it.SetFastInterpolation(True)
    d = GreedyDeformationDataB200(torch.from_numpy(I0).cuda(), torch.from_numpy(I1).cuda())
    it.Run(d, 1 + args.steps, update_first=True)
    torch.cuda.synchronize()
    print(json.dumps({"ncu_case": "greedy 128^3", "iterations": 1 + args.steps}))
    return 0


# ---- the other hot-path rows, measured on request (--workload) ------------------
def _timed(fn, steps, warmup, stream):
    import torch
    for _ in range(max(warmup, 3)):
        fn()
    torch.cuda.synchronize()
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        s0.record(stream)
        for _ in range(steps):
            fn()
        s1.record(stream)
        torch.cuda.synchronize()
    return s0.elapsed_time(s1), clk.summary()


def _atlas_subject(args):
    """One uneven-grid atlas subject (the atlas generator, per-subject seed)."""
    import numpy as np
    from atlaswerks_b200.synth import rng_for, smooth_displacement, warp
    seed, params, size = args
    rng = rng_for(seed)
    nx, ny, nz = size
    z, y, x = np.meshgrid((np.arange(nz) + 0.5) / nz, (np.arange(ny) + 0.5) / ny,
                          (np.arange(nx) + 0.5) / nx, indexing="ij")
    img = np.zeros((nz, ny, nx))
    for c, sg, a in params:
        img += a * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (2 * sg * sg))
    img = np.clip(img, 0, 1).astype(np.float32)
    u = smooth_displacement((nz, ny, nx), 5.0, rng)
    return (warp(img, u) * np.float32(rng.uniform(0.9, 1.1))).astype(np.float32)


def run_atlas(args):
    """32 subjects, per-axis sizes in {96,...,160}, template 128^3, mean
    every 10 iterations; a step = 10 iterations of every subject + the mean.
    With N ranks (one per GPU), rank r owns subjects i mod N = r and the mean
    is one NCCL all-reduce of the ranks' weighted sums per update (strong
    scaling: the 32 subjects are the whole job)."""
    import multiprocessing as mp

    import torch

    from atlaswerks_b200.atlas import GreedyAtlasBuilderB200, GreedyAtlasParam, local_subjects
    from atlaswerks_b200.greedy import DiffOperParam
    from atlaswerks_b200.synth import rng_for
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    ns, T, period = 32, 128, 10
    rng = rng_for(4)
    params = [(rng.uniform(0.15, 0.85, 3), rng.uniform(0.03, 0.07), rng.uniform(0.3, 1.0))
              for _ in range(24)]
    sizes = [tuple(int(rng.choice([96, 112, 128, 144, 160])) for _ in range(3)) for _ in range(ns)]
    mine = local_subjects(ns, rank, world)
    # subject images are generated before the first CUDA call (spawned pool)
    with mp.get_context("spawn").Pool(min(32, os.cpu_count() or 1)) as pool:
        imgs = pool.map(_atlas_subject, [(100 + i, params, sizes[i]) for i in mine])
    torch.cuda.set_device(local)
    dist = None
    group = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        group = dist.group.WORLD
    dev = [None] * ns
    for i, a in zip(mine, imgs):
        dev[i] = torch.from_numpy(a).cuda()
    b = GreedyAtlasBuilderB200(dev, (T, T, T), GreedyAtlasParam(DiffOperParam(ALPHA, BETA, GAMMA),
                                                                 MAX_PERT, 100, period),
                               group=group)
    b._update_mean()
    b.engine.iterate(2, True)
    stream = torch.cuda.current_stream()

    def step():
        b.engine.iterate(period, False)
        b._update_mean()

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        s0.record(stream)
        for _ in range(args.steps):
            step()
        s1.record(stream)
        torch.cuda.synchronize()
    ms = s0.elapsed_time(s1)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    clocks = clk.summary()
    subj_iters = ns * period * args.steps
    value = subj_iters / (ms / 1000.0)
    peak, kind = peaks()
    gbs = B_ITER * T ** 3 * subj_iters / (ms / 1000.0) / 1e9
    line = {
        "metric": "atlas subject-iterations/s (template 128^3)", "value": value,
        "unit": "subject-iters/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (24-blob template, per-subject smooth warp max 5, intensity scale "
                "U(0.9,1.1))",
        "config": {"workload": "greedy atlas, 32 subjects of uneven grids {96..160}^3, deformations "
                   "on a 128^3 template grid, mean every 10 iterations", "subjects": ns,
                   "subject_sizes": sizes, "template": [T, T, T], "mean_period": period,
                   "parallelism": f"subjects sharded over {world} rank(s), one all-reduce of the "
                                  f"weighted sum per mean update"},
        "roofline": {"bound": "hbm", "achieved": gbs / world, "peak": peak, "unit": "GB/s",
                     "frac": gbs / world / peak, "traffic": None, "per": "GPU",
                     "algorithmic_bytes_per_subject_iteration": B_ITER * T ** 3},
        "gpu_launches": (6 * period * len(mine) + 1) * args.steps, "clocks": clocks}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


def run_ldmm(args):
    """LDMM relaxation (IterateNew) at 128^3 with T = 10 time steps,
    sigma = 0.1, fixed step 0.005; a step = one iteration."""
    import torch

    from atlaswerks_b200.ldmm import (LDMMDeformationDataB200, LDMMIteratorB200,
                                      LDMMIteratorParam)
    from atlaswerks_b200.greedy import DiffOperParam
    from atlaswerks_b200.synth import greedy_pair
    T = 10
    I0, I1 = greedy_pair((N, N, N), 7, 8, 3.0)
    it = LDMMIteratorB200((N, N, N), n_time_steps=T)
    it.SetScaleLevel((N, N, N), (1.0, 1.0, 1.0),
                     LDMMIteratorParam(DiffOperParam(ALPHA, BETA, GAMMA), 0.1, 0.005, False, 0.1))
    data = LDMMDeformationDataB200(torch.from_numpy(I0).cuda(), torch.from_numpy(I1).cuda(), T)
    stream = torch.cuda.current_stream()
    ms, clocks = _timed(lambda: it.Run(data, 1), args.steps, args.warmup, stream)
    value = args.steps / (ms / 1000.0)
    peak, kind = peaks()
    b_ldmm = 176 * N ** 3 * T
    gbs = b_ldmm * value / 1e9
    print(json.dumps({
        "metric": "128^3 LDMM iterations/s (T=10)", "value": value, "unit": "iters/s",
        "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded blobs + smooth warp)",
        "config": {"workload": "LDMM relaxation IterateNew, 128^3, 10 time steps, sigma 0.1, "
                   "step 0.005", "grid": [N, N, N], "time_steps": T},
        "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                     "frac": gbs / peak, "traffic": None,
                     "algorithmic_bytes_per_iteration": b_ldmm},
        "clocks": clocks}))
    return 0


def run_adshoot(args):
    """LDMM adjoint geodesic shooting (LDMMAdShootingIterator) at 128^3 with
    T = 5 time steps, sigma 1, fixed step 0.0002 (the fine level of the
    reference's LDMMAdShootingWarp regression); a step = one iteration
    (shooting, backward adjoint sweep, alpha0 update)."""
    import torch

    from atlaswerks_b200.greedy import DiffOperParam
    from atlaswerks_b200.ldmm import LDMMIteratorParam
    from atlaswerks_b200.shooting import LDMMAdShootingIteratorB200, LDMMShootingDefDataB200
    from atlaswerks_b200.synth import greedy_pair
    T = 5
    I0, I1 = greedy_pair((N, N, N), 7, 8, 3.0)
    it = LDMMAdShootingIteratorB200((N, N, N), n_time_steps=T)
    it.SetScaleLevel((N, N, N), (1.0, 1.0, 1.0),
                     LDMMIteratorParam(DiffOperParam(ALPHA, BETA, GAMMA), 1.0, 0.0002, False))
    data = LDMMShootingDefDataB200(torch.from_numpy(I0).cuda(), torch.from_numpy(I1).cuda())
    stream = torch.cuda.current_stream()
    ms, clocks = _timed(lambda: it.Iterate(data), args.steps, args.warmup, stream)
    value = args.steps / (ms / 1000.0)
    peak, kind = peaks()
    # per voxel: T x (advance 100 + velocity 20 + 4S) + T x backward step (176 + 4S)
    # + the kinetic energy from the force (20), the image residual (12), the first
    # adjoint splat (20), clearing alpha~ (4), the alpha0 update (28) and the map
    # copies (48): 132
    b_iter = (T * (296 + 8 * SPEC) + 132) * N ** 3
    gbs = b_iter * value / 1e9
    print(json.dumps({
        "metric": "128^3 adjoint shooting iterations/s (T=5)", "value": value, "unit": "iters/s",
        "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded blobs + smooth warp)",
        "config": {"workload": "LDMM adjoint shooting (LDMMAdShootingIterator), 128^3, 5 time "
                   "steps, sigma 1, step 0.0002", "grid": [N, N, N], "time_steps": T},
        "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                     "frac": gbs / peak, "traffic": None,
                     "algorithmic_bytes_per_iteration": b_iter},
        "clocks": clocks}))
    return 0


def run_ldmm_atlas(args):
    """LDMM relaxation atlas: 4 subjects at 128^3, T = 5 time steps,
    IterateNew, sigma 1, fixed step 0.01, JacobianScale mean after every
    iteration; a step = one atlas iteration (every subject's LDMM iteration,
    then GetI1At0 + ComputeJacDet of every subject and the mean)."""
    import torch

    from atlaswerks_b200.greedy import DiffOperParam
    from atlaswerks_b200.ldmm import LDMMIteratorParam
    from atlaswerks_b200.ldmm_atlas import LDMMAtlasBuilderB200, LDMMAtlasParam
    from atlaswerks_b200.synth import greedy_pair
    ns, T = 4, 5
    imgs = [torch.from_numpy(greedy_pair((N, N, N), 300 + k, 8, 3.0)[1]).cuda() for k in range(ns)]
    param = LDMMAtlasParam(LDMMIteratorParam(DiffOperParam(ALPHA, BETA, GAMMA), 1.0, 0.01, False,
                                             0.1), NTimeSteps=T, NIterations=1,
                           JacobianScale=True)
    b = LDMMAtlasBuilderB200(imgs, (N, N, N), param)
    b._update_mean()
    stream = torch.cuda.current_stream()

    def step():
        b.engine.iterate(first=False)
        b._update_mean()

    ms, clocks = _timed(step, args.steps, args.warmup, stream)
    value = args.steps / (ms / 1000.0)
    peak, kind = peaks()
    # per subject: the LDMM iteration (176 N per time step) and the mean's
    # backward sweep (compose 36 N + Jacobian transport 20 N per time step,
    # the pulled-back image 4 N, the two sums 20 N)
    b_iter = ns * (176 * T + 56 * T + 24) * N ** 3
    gbs = b_iter * value / 1e9
    print(json.dumps({
        "metric": "128^3 LDMM atlas iterations/s (4 subjects, T=5)", "value": value,
        "unit": "atlas-iters/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded blobs + smooth warp)",
        "config": {"workload": "LDMM relaxation atlas (IterateNew, JacobianScale), 4 subjects "
                   "128^3, 5 time steps, sigma 1, step 0.01, mean every iteration",
                   "grid": [N, N, N], "subjects": ns, "time_steps": T},
        "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                     "frac": gbs / peak, "traffic": None,
                     "algorithmic_bytes_per_atlas_iteration": b_iter},
        "clocks": clocks}))
    return 0


def run_warmstart(args):
    """Learned warm start + refinement against the plain GPU greedy solve on
    held-out pairs of the pair-registration generator, with the committed
    trained weights (the network at half the pair's grid on the downsampled
    pair). A step = one pair through both paths."""
    import numpy as np
    import torch

    from atlaswerks_b200 import warmstart as W
    n = args.grid or 128
    if n not in W.TRAINED:
        print(json.dumps({"metric": f"{n}^3 warm-start registrations/s", "unavailable":
                          f"no trained weights for {n}^3 pairs"}))
        return 0
    pairs = W.make_pairs(range(10_000_000, 10_000_000 + args.pairs), n,
                         min(32, os.cpu_count() or 1))
    net = W.trained(n)
    W.evaluate(net, pairs[:2])  # warm-up (module loads, graph capture, pools)
    res = W.evaluate(net, pairs)
    pm = float(np.sum([r["plain_ms"] for r in res]))
    wm = float(np.sum([r["warm_ms"] for r in res]))
    # against the 3-level multiscale plain solve (its finest-level energy the
    # target, and the fallback)
    res_ms = W.evaluate(net, pairs, plain="multiscale")
    pm_ms = float(np.sum([r["plain_ms"] for r in res_ms]))
    wm_ms = float(np.sum([r["warm_ms"] for r in res_ms]))
    multiscale = {
        "plain": "3-level multiscale greedy, 100/50/25 iterations at n/4, n/2, n",
        "plain_pairs_per_s": 1000.0 * len(res_ms) / pm_ms,
        "warm_pairs_per_s": 1000.0 * len(res_ms) / wm_ms,
        "wall_ratio_warm_over_plain": wm_ms / pm_ms,
        "plain_ms_median": float(np.median([r["plain_ms"] for r in res_ms])),
        "warm_ms_median": float(np.median([r["warm_ms"] for r in res_ms])),
        "iters_warm_run_mean": float(np.mean([r["warm_iters_run"] for r in res_ms])),
        "reached_fraction": float(np.mean([r["reached"] for r in res_ms])),
        "fallback_fraction": float(np.mean([r["fallback"] for r in res_ms]))}
    print(json.dumps({
        "metric": f"{n}^3 registrations/s to the plain method's final energy (+1%)",
        "value": 1000.0 * len(res) / wm, "unit": "pairs/s", "n_gpus": 1, "steps": len(res),
        "higher_is_better": True, "dtype": "bf16 network, f32 registration",
        "data": "synthetic held-out seeds (8 blobs, smooth warp max 3 voxels)",
        "config": {"workload": "warm start (trained encoder-decoder, one graph replay) + greedy "
                   "refinement with fallback vs plain greedy (50 iterations from the identity)",
                   "grid": [n] * 3, "network_grid": [net.D, net.H, net.W], "pairs": len(res)},
        "plain_pairs_per_s": 1000.0 * len(res) / pm, "wall_ratio_warm_over_plain": wm / pm,
        "predict_ms_median": float(np.median([r["predict_ms"] for r in res])),
        "warm_ms_median": float(np.median([r["warm_ms"] for r in res])),
        "plain_ms_median": float(np.median([r["plain_ms"] for r in res])),
        "iters_plain_mean": float(np.mean([r["plain_iters"] for r in res])),
        "iters_warm_mean": float(np.mean([r["warm_iters"] for r in res])),
        "iters_warm_run_mean": float(np.mean([r["warm_iters_run"] for r in res])),
        "reached_fraction": float(np.mean([r["reached"] for r in res])),
        "fallback_fraction": float(np.mean([r["fallback"] for r in res])),
        "vs_multiscale": multiscale, "network": network_rates(net, args)}))
    return 0


def network_rates(net, args):
    """The network's own rates on its grid: the forward pass (one graph
    replay inside the predictor is the same launches) and a training step
    (forward, loss, backward, Adam), each timed with CUDA events, with the
    convolutions' FLOPs (2 * taps * Cin * Cout per voxel) against the
    measured dense BF16 peak."""
    import torch

    from atlaswerks_b200 import warmstart as W
    D, H, Wd = net.D, net.H, net.W
    fwd = 0.0
    for name, ci, co, t in W.LAYERS:
        lvl = net._level_of(name)
        fwd += 2.0 * t * ci * co * net._vox(lvl)
    train_flops = 3.0 * fwd  # forward + data gradient + weight gradient
    trainee = W.WarmStartNet((D, H, Wd), seed=3)
    I0 = torch.rand((D, H, Wd), device="cuda")
    I1 = torch.rand((D, H, Wd), device="cuda")
    tgt = torch.zeros((3, D, H, Wd), device="cuda")
    for _ in range(3):
        net.forward(I0, I1)
        trainee.train_step(I0, I1, tgt)
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    reps = 20
    e[0].record()
    for _ in range(reps):
        net.forward(I0, I1)
    e[1].record()
    for _ in range(reps):
        trainee.train_step(I0, I1, tgt)
    e[2].record()
    torch.cuda.synchronize()
    f_ms = e[0].elapsed_time(e[1]) / reps
    t_ms = e[1].elapsed_time(e[2]) / reps
    peak = None
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        peak = float(json.load(open(pp))["bf16_tflops"])
    out = {"grid": [D, H, Wd], "forward_ms": f_ms, "forward_gflop": fwd / 1e9,
           "forward_tflops": fwd / (f_ms / 1000.0) / 1e12, "train_step_ms": t_ms,
           "train_steps_per_s": 1000.0 / t_ms, "train_step_gflop": train_flops / 1e9,
           "train_tflops": train_flops / (t_ms / 1000.0) / 1e12,
           "peak_bf16_tflops": peak, "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst)"}
    if peak:
        out["forward_frac_of_peak"] = out["forward_tflops"] / peak
        out["train_frac_of_peak"] = out["train_tflops"] / peak
    return out


def _launch_ranks(n):
    """--gpus n > 1 without a launcher: run this same command as n ranks,
    one per GPU, through torch.distributed.run on 127.0.0.1."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fast-interp", action="store_true",
                    help="greedy: float fused-multiply-add interpolation (not bit-exact)")
    ap.add_argument("--ncu-case", action="store_true",
                    help="run a short untimed 128^3 workload for ncu captures")
    ap.add_argument("--workload", default="greedy",
                    choices=["greedy", "atlas", "ldmm", "ldmm_atlas", "warmstart", "adshoot"],
                    help="the headline greedy line (default) or another hot-path row")
    ap.add_argument("--grid", type=int, default=0, help="warmstart: pair grid (64 or 128; default 128)")
    ap.add_argument("--pairs", type=int, default=32, help="warmstart: held-out pairs")
    args = ap.parse_args()
    if "WORLD_SIZE" in os.environ:
        if int(os.environ["WORLD_SIZE"]) != args.gpus:
            print(f"bench.py: --gpus {args.gpus} but the launcher started "
                  f"{os.environ['WORLD_SIZE']} ranks", file=sys.stderr)
            return 2
    elif args.gpus > 1:
        return _launch_ranks(args.gpus)
    if args.ncu_case:
        return run_ncu_case(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "atlas":
        return run_atlas(args)
    if args.workload != "greedy":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0  # the other rows are single-GPU measurements
        import torch
        torch.cuda.set_device(0)
        return {"ldmm": run_ldmm, "ldmm_atlas": run_ldmm_atlas, "warmstart": run_warmstart,
                "adshoot": run_adshoot}[args.workload](args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
