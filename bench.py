#!/usr/bin/env python
"""Throughput benchmark of the spectral-fluid step engine.

Workload (default): the plain single-instance path at the larger size --
a 32^3 voxel box with a solid sphere of radius 8 voxels at its centre,
N = 128 Laplacian eigenmodes (C 128^3 and Phi stored FP32, state FP64),
w ~ N(0, 1) with seed 2 scaled to unit energy, constant forcing of 0.1 per
step on the lowest mode, dt = 0.005, 262,144 particles uniform in the fluid
(seed 3) traced with RK4.  One step = contraction + state update +
reconstruction + particle tracing for one instance.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under ``torch.distributed.run`` every rank steps its own replica (instances
are independent; no per-step collective): weak scaling, ``value`` is the
whole-job instance-steps/s, timed as the max over ranks of the device time.
``--impl reference`` times the reference's CPU step (the FP64 restatement of
Solver/SolverImpl/psfsolver.cpp:21-234; the reference itself does not build
here) on all host cores.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from parallelspectralfluids3d_b200 import replicas  # noqa: E402

WORKLOADS = {
    "sphere32_n128_p262144_rk4": dict(
        domain=("sphere", 32, 8.0), n_modes=128, seed_w=2, seed_p=3, particles=262144, dt=0.005,
        force0=0.1, integrator=4, full_steps=1000,
        describe="32^3 box with a solid sphere of radius 8 voxels, N=128, 262144 particles, RK4, "
                 "forcing 0.1/step on mode 0, dt=0.005"),
    "box16_n64_p4096_rk4": dict(
        domain=("box", 16, None), n_modes=64, seed_w=0, seed_p=1, particles=4096, dt=0.01,
        force0=0.0, integrator=4, full_steps=100,
        describe="16^3 all-wall box, N=64, 4096 particles, RK4, dt=0.01"),
}
# Batched (tensor-core, BF16 hi/lo) workloads.  "members" lists
# (domain, n_max, slots, n_modes per instance, particles per instance).
BATCH_WORKLOADS = {
    # The plain workload above, 64 independent instances (seeds 2+i / 3+i) on one basis.
    "sphere32_n128_p262144_rk4_b64": dict(
        bases=[(("sphere", 32, 8.0), 128)], instances=64, n_modes=lambda i, rng: 128, particles=262144,
        dt=0.005, force0=0.1, integrator=4, seed_w=lambda i: 2 + i, seed_p=lambda i: 3 + i, full_steps=1000,
        check=[0, 63], check_particles=[0],
        describe="64 instances of the 32^3 + sphere r=8, N=128, 262144-particle RK4 workload, one batch"),
    # Precision form: 48^3 channel (all-wall box), N=256, B=64 trajectories, seeds 100-163, 1M particles each.
    "channel48_n256_b64_p1m": dict(
        bases=[(("channel", (48, 48, 48), None), 256)], instances=64, n_modes=lambda i, rng: 256,
        particles=1 << 20, dt=0.005, force0=0.0, integrator=4, seed_w=lambda i: 100 + i,
        seed_p=lambda i: 10100 + i, full_steps=1000, check=[0, 31, 63], check_particles=[0, 31, 63],
        describe="48^3 channel, N=256 (C, Phi as BF16 hi+lo), 64 trajectories x 1M particles, RK4, dt=0.005"),
    # The serving configuration's largest tile shape: 64 instances of N=384 on one 384-mode basis.
    "channel64_n384_b64_p16384": dict(
        bases=[(("channel", (64, 32, 32), None), 384)], instances=64, n_modes=lambda i, rng: 384,
        particles=16384, dt=0.005, force0=0.0, integrator=4, seed_w=lambda i: 300 + i, seed_p=lambda i: 400 + i,
        full_steps=500, check=[0, 63], check_particles=[0],
        describe="64 instances of N=384 on the 64x32x32 channel, 16384 particles each, RK4, dt=0.005"),
    # Batching form: 512 instances, N ~ U{32..256}, domains in rotation, 16384 particles each.
    "mixed512_p16384": dict(
        bases=[(("box", 32, None), 256), (("sphere", 40, 10.0), 256), (("channel", (64, 32, 32), None), 256)],
        instances=512, n_modes=lambda i, rng: int(rng.choice([32, 64, 96, 128, 192, 256])), particles=16384,
        dt=0.005, force0=0.0, integrator=4, seed_w=lambda i: 1000 + i, seed_p=lambda i: 5000 + i,
        full_steps=500, check=[0, 1, 2, 511], check_particles=[0],
        describe="512 instances, N uniform in {32,64,96,128,192,256}, domains 32^3 box / 40^3 + sphere r=10 / "
                 "64x32x32 channel in rotation, 16384 particles each, RK4"),
}
BIG_BASIS_CACHE = os.path.join(ROOT, ".basis_big")
BASIS_CACHES = [os.path.join(ROOT, d) for d in (".basis_cache", ".basis_big", ".basis_c3")]


def basis_cache_for(name, n):
    """The cache directory holding a basis (full or compact file), else the large-basis cache."""
    for d in BASIS_CACHES:
        if any(os.path.exists(os.path.join(d, f"{name}_n{n}.{ext}")) for ext in ("psfb", "psfc")):
            return d
    return BIG_BASIS_CACHE
DEFAULT_WORKLOAD = "sphere32_n128_p262144_rk4"
REFERENCE_MIN_STEPS = 300
FORM_WORKLOAD = "sphere32_n128_p262144_rk4_b64"
MIXED_WORKLOAD = "mixed512_p16384"
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2

# DRAM bytes (read + write) per launch from one ncu capture of each kernel on
# the named workload (profiles/step_kernels_sphere32_n128_p262144_rk4.md).
NCU_TRAFFIC = {
    ("sphere32_n128_p262144_rk4", "contract_state"): 8410880,
    ("sphere32_n128_p262144_rk4", "reconstruct"): 46189056,
    ("sphere32_n128_p262144_rk4", "trace"): 5003776,
}


def make_domain(spec):
    from parallelspectralfluids3d_b200.domain import box_domain, channel_domain, sphere_obstacle_domain

    kind, n, r = spec
    if kind == "sphere":
        return sphere_obstacle_domain(n, r)
    if kind == "channel":
        return channel_domain(n)
    return box_domain(n)


def plain_config(name, b, wl, parts, world=1):
    """The ``config`` object of a plain-workload line (the same for both arms)."""
    return {"workload": name, "describe": wl["describe"], "n_modes": b.n_modes, "faces_active": b.n_active,
            "particles": int(parts.shape[0]), "integrator": "rk4" if wl["integrator"] == 4 else "rk1",
            "dt": wl["dt"], "l2": "flushed before every timed step (256 MB write, then 256 MB read)",
            "parallelism": f"replicas x{world}"}


def load_workload(name, device):
    from parallelspectralfluids3d_b200.fixture import cached_basis, initial_coefficients, initial_particles

    wl = WORKLOADS[name]
    b = cached_basis(make_domain(wl["domain"]), wl["n_modes"], device=device)
    w0 = initial_coefficients(b.n_modes, wl["seed_w"])
    parts = initial_particles(b, wl["particles"], wl["seed_p"])
    force = np.zeros(b.n_modes)
    force[0] = wl["force0"] / wl["dt"]
    return wl, b, w0, parts, force


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def kernel_bytes(b, P, kind):
    """Algorithmic bytes one launch must move (per kernel, FP32 basis)."""
    N = b.n_modes
    Np = (N + 3) // 4 * 4
    Fa = b.n_active
    if kind == "contract_state":
        return 4 * N * N * Np + 8 * N * 3
    if kind == "reconstruct":  # Phi read once, face ids and pair slots read, u and pairs written
        return 4 * N * Fa + 4 * Fa + 4 * Fa + 8 * Fa + 8 * N
    return 32 * P  # trace: read + write float4 per particle


# -------------------------------------------------------------- our arm
def run_ours(args, rank, world, local_rank):
    import torch

    from parallelspectralfluids3d_b200 import _lib as L
    from parallelspectralfluids3d_b200.solver import Context

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    dist = world > 1
    if dist:
        import torch.distributed as td

    def barrier():
        if dist:
            td.barrier(device_ids=[local_rank])

    if rank == 0:
        wl, b, w0, parts, force = load_workload(args.workload, "cuda")
    barrier()
    if rank != 0:
        wl, b, w0, parts, force = load_workload(args.workload, "cuda")

    params = L.make_params(dt=wl["dt"], integrator=wl["integrator"],
                           flags=L.PSF_FLAG_RENORM | (L.PSF_FLAG_FORCING if wl["force0"] else 0))
    ctx = Context(b, params, device=local_rank)
    ctx.set_forcing(force)
    ctx.set_state(w0)
    ctx.set_particles(parts)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    flush_w = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    flush_r = torch.ones(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    sink = torch.empty((), dtype=torch.float32, device=dev)

    def flush_l2():
        # Write a buffer larger than L2, then read another one: the timed kernels
        # start from a cold L2 that holds no dirty lines of the flush itself.
        flush_w.zero_()
        torch.sum(flush_r, dim=0, out=sink)

    K = args.steps
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    clocks = ClockSampler(local_rank).start()
    # Pre-roll under load so that the clock samples cover the timed region,
    # then restart from the configured initial state and warm up.
    t_end = time.perf_counter() + 1.5
    while time.perf_counter() < t_end:
        ctx.step(50)
        ctx.sync()
    ctx.set_state(w0)
    ctx.set_particles(parts)
    ctx.step(max(3, args.warmup))
    ctx.sync()
    barrier()
    torch.cuda.synchronize(dev)
    with torch.cuda.stream(stream):
        for i in range(K):
            flush_l2()
            starts[i].record(stream)
            ctx.step(1)
            ends[i].record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    clk = clocks.stop()
    per_step = np.array([s.elapsed_time(e) for s, e in zip(starts, ends)])
    total_ms = float(per_step.sum())
    (total_ms,) = replicas.slowest([total_ms], device=dev)
    value = world * K / (total_ms / 1e3)

    # Kernel breakdown: each kernel between its own events, L2 flushed before each step.
    M = min(K, 64)
    names = ["contract_state", "reconstruct", "trace"][: ctx.kernels_per_step()]
    acc = np.zeros(len(names))
    for _ in range(M):
        with torch.cuda.stream(stream):
            flush_l2()
        acc += ctx.profile_step()
    kms = acc / M
    dom_i = int(np.argmax(kms))
    peak, peak_kind = measured_peak_hbm()
    alg = kernel_bytes(b, ctx.P, names[dom_i])
    achieved = alg / (kms[dom_i] / 1e3) / 1e9
    roofline = {"kernel": names[dom_i], "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "algorithmic_bytes": int(alg),
                "traffic": NCU_TRAFFIC.get((args.workload, names[dom_i])),
                "all_kernels": {n: {"ms": round(float(m), 5),
                                    "GB/s": round(kernel_bytes(b, ctx.P, n) / (m / 1e3) / 1e9, 1)}
                                for n, m in zip(names, kms)}}

    # End to end through the public API: host (pinned) buffers, copies inside the region.
    E = min(K, 50)
    w_host = torch.from_numpy(ctx.get_state()).pin_memory()
    p_host = torch.from_numpy(ctx.get_particles()).pin_memory()
    w_np, p_np = w_host.numpy(), p_host.numpy()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize(dev)
    e0.record(stream)
    for _ in range(E):
        ctx.set_state(w_np)
        ctx.set_particles(p_np)
        ctx.step(1)
        ctx.get_state(w_np)
        ctx.get_particles(p_np)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = e0.elapsed_time(e1)
    (e2e_ms,) = replicas.slowest([e2e_ms], device=dev)
    e2e = {"value": round(world * E / (e2e_ms / 1e3), 2), "unit": "instance-steps/s",
           "h2d_bytes_per_step": int(8 * b.n_modes + 16 * ctx.P),
           "d2h_bytes_per_step": int(8 * b.n_modes + 16 * ctx.P), "steps": E}
    ctx.close()

    # Accuracy of the full configured run against the FP64 oracle, and the CPU baseline.
    extra = {}
    if rank == 0 and world == 1 and not args.no_cpu:
        extra = accuracy_and_cpu(b, wl, w0, parts, force, params, local_rank)
    barrier()

    line = {
        "metric": "instance-steps/s", "value": round(value, 2), "unit": "instance-steps/s",
        "n_gpus": world, "steps": K, "warmup": max(3, args.warmup), "ms_per_step": round(total_ms / K, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "state_dtype": "f64", "data": "synthetic",
        "config": plain_config(args.workload, b, wl, parts, world),
        "p50_ms": round(float(np.percentile(per_step, 50)), 5),
        "p99_ms": round(float(np.percentile(per_step, 99)), 5),
        "particle_steps_per_s": round(value * parts.shape[0], 1),
        "gpu_launches": int(K * len(names)),
        "kernel_ms": {n: round(float(m), 5) for n, m in zip(names, kms)},
        "roofline": roofline, "e2e": e2e, "clocks": clk,
    }
    line.update(extra)
    if rank == 0 and world == 1 and not args.no_forms:
        form = run_batch(args, FORM_WORKLOAD, local_rank, plain=False)
        form["speedup_vs_plain"] = round(form["value"] / value, 3)
        form["e2e_speedup_vs_plain"] = round(form["e2e"]["value"] / e2e["value"], 3)
        line["forms"] = {"batched_bf16x2": dict(workload=FORM_WORKLOAD, **form)}
        line["gpu_launches"] += form["gpu_launches"]
        # The batching form (512 instances of uneven N on three domains): its
        # bases come from the GPU precompute on this device, and its plain-path
        # denominator is the single-instance path on a sample of the same instances.
        t0 = time.perf_counter()
        mixed = run_batch(args, MIXED_WORKLOAD, local_rank, plain=True)
        mixed["wall_s"] = round(time.perf_counter() - t0, 1)
        line["forms"]["batched_mixed512"] = dict(workload=MIXED_WORKLOAD, **mixed)
        line["gpu_launches"] += mixed["gpu_launches"]
        # The serving form (continuous batching of the Poisson request mix).
        line["forms"]["served"] = dict(workload=SERVE_WORKLOAD, **run_serve_form(args, local_rank))
    return line


def accuracy_and_cpu(b, wl, w0, parts, force, params, device):
    """Full configured run on the GPU vs the FP64 oracle; the oracle run is the CPU baseline."""
    from oracle import oracle as O
    from parallelspectralfluids3d_b200.solver import Context

    S = wl["full_steps"]
    ctx = Context(b, params, device=device)
    ctx.set_forcing(force)
    ctx.set_state(w0)
    ctx.set_particles(parts)
    ctx.step(S)
    w_gpu = ctx.get_state()
    p_gpu = ctx.get_particles()
    ctx.close()
    ref = O.OracleRollout(b, w0, parts, dt=wl["dt"], integrator=wl["integrator"], forcing=force)
    t0 = time.perf_counter()
    ref.step(S)
    cpu_s = time.perf_counter() - t0
    rel = float(np.linalg.norm(w_gpu - ref.w) / np.linalg.norm(ref.w))
    d = np.abs(p_gpu[:, :3] - ref.pos).max(axis=1) / b.h
    # The same FP64 rollout with positions stored in FP32 after every step, as
    # the reference stores them: particles that come within an FP32 rounding of
    # a wall snap onto it (normal velocity exactly 0 there) in both.
    ref32 = O.OracleRollout(b, w0, parts, dt=wl["dt"], integrator=wl["integrator"], forcing=force,
                            reconstruct=True, positions="f32").step(S)
    d32 = np.abs(p_gpu[:, :3] - ref32.pos).max(axis=1) / b.h
    return {
        "accuracy": {"steps": S, "rel_err_w_vs_fp64": rel, "max_particle_err_voxels": float(d.max()),
                     "p99_particle_err_voxels": float(np.percentile(d, 99)),
                     "p50_particle_err_voxels": float(np.percentile(d, 50)),
                     "vs_fp64_with_fp32_positions": {"max_particle_err_voxels": float(d32.max()),
                                                     "p99_particle_err_voxels": float(np.percentile(d32, 99))}},
        "cpu_baseline": {"value": round(S / cpu_s, 3), "unit": "instance-steps/s", "cores": O.num_threads(),
                         "kind": "port", "sample": f"full {S}-step run of the workload, FP64, OpenMP"},
    }


# -------------------------------------------------------- reference arm
def run_reference(args):
    """The reference's CPU step (FP64 restatement) on all host threads."""
    from oracle import oracle as O

    if args.workload in BATCH_WORKLOADS:
        return run_reference_batch(args)
    wl, b, w0, parts, force = load_workload(args.workload, "cpu")
    O.build()
    ref = O.OracleRollout(b, w0, parts, dt=wl["dt"], integrator=wl["integrator"], forcing=force)
    ref.step(max(3, args.warmup))
    # At least REFERENCE_MIN_STEPS steps (about 2 s on the workload) so that the
    # rate is not a handful of noisy steps; never more than the full run.
    K = min(max(args.steps, REFERENCE_MIN_STEPS), wl["full_steps"])
    t0 = time.perf_counter()
    ref.step(K)
    dt = time.perf_counter() - t0
    value = K / dt
    return {
        "impl": "reference", "metric": "instance-steps/s", "value": round(value, 3), "unit": "instance-steps/s",
        "n_gpus": 1, "steps": K, "warmup": max(3, args.warmup), "ms_per_step": round(1e3 * dt / K, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": plain_config(args.workload, b, wl, parts),
        "cpu_baseline": {"value": round(value, 3), "unit": "instance-steps/s", "cores": O.num_threads(),
                         "kind": "port",
                         "sample": f"{K} steps of the full workload (reference does not build: Eigen/glm absent)"},
        "e2e": {"value": round(value, 3), "unit": "instance-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------------------ batched arm
def load_batch_workload(name, device, particles=None):
    """Bases and per-instance inputs of a batched workload (seeded, synthetic)."""
    from parallelspectralfluids3d_b200.fixture import cached_basis, initial_coefficients, initial_particles

    wl = BATCH_WORKLOADS[name]
    bases = []
    for spec, n in wl["bases"]:
        dom = make_domain(spec)
        bases.append(cached_basis(dom, n, cache_dir=basis_cache_for(dom.name, n), device=device))
    rng = np.random.default_rng(4)
    insts = []
    for i in range(wl["instances"]):
        g = i % len(bases)
        n = wl["n_modes"](i, rng)
        w0 = initial_coefficients(n, wl["seed_w"](i))
        f = np.zeros(n)
        f[0] = wl["force0"] / wl["dt"]
        insts.append(dict(basis=g, slot=i // len(bases), n=n, w0=w0, force=f, seed_p=wl["seed_p"](i)))
    slots = [sum(1 for x in insts if x["basis"] == g) for g in range(len(bases))]
    for x in insts:
        x["parts"] = initial_particles(bases[x["basis"]], wl["particles"] if particles is None else particles,
                                       x["seed_p"])
    return wl, bases, slots, insts


def assign_slots(insts, n_bases):
    """Number each instance's slot within its basis (in order) and count the slots per basis."""
    counts = [0] * n_bases
    for x in insts:
        x["slot"] = counts[x["basis"]]
        counts[x["basis"]] += 1
    return [max(1, c) for c in counts]


def batch_params(wl, x):
    from parallelspectralfluids3d_b200 import _lib as L

    flags = L.PSF_FLAG_RENORM | (L.PSF_FLAG_FORCING if wl["force0"] else 0)
    return L.make_params(dt=wl["dt"], integrator=wl["integrator"], flags=flags, seed=x["seed_p"],
                         precision=L.PSF_PRECISION_BF16X2)


def fill_batch(batch, wl, insts):
    status = batch.set_instances([
        {"basis": x["basis"], "slot": x["slot"], "w0": x["w0"], "params": batch_params(wl, x), "particles": x["parts"],
         "forcing": x["force"] if wl["force0"] else None} for x in insts])
    if np.any(status != 0):
        raise RuntimeError(f"placement failed: {sorted(set(status.tolist()))}")


def batch_kernel_bytes(bases, slots, insts, kind):
    """Algorithmic bytes (and tensor FLOPs) of one launch of a batched kernel."""
    tot, flops = 0, 0
    for b, cap in zip(bases, slots):
        N, Fa = b.n_modes, b.n_active
        at = (N + 127) // 128
        if kind == "contract":
            tot += 4 * N ** 3 + 8 * N * cap + 32 * N * at * cap
            flops += 3 * 2 * N * N * ((N + 63) // 64 * 64) * ((cap + 15) // 16 * 16)
        elif kind == "reconstruct":
            tot += 4 * Fa * N + 8 * Fa * cap
            flops += 3 * 2 * Fa * ((N + 63) // 64 * 64) * ((cap + 15) // 16 * 16)
        elif kind == "state":
            tot += cap * (8 * N * 2 + 8 * N * at * 4 + 4 * N)
    if kind == "trace":
        tot = 32 * sum(len(x["parts"]) for x in insts)
    return tot, flops


def run_batch(args, name, local_rank, flush=True, check=True, plain=True, rank=0, world=1):
    """Time a batched workload: device instance-steps/s, kernel roofline, e2e rollouts, FP64 error.

    With ``world > 1`` this rank takes its round-robin share of the instances
    (replicas.shard) and steps them as its own batch.
    """
    import torch

    from parallelspectralfluids3d_b200.batch import Batch

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    wl, bases, slots, insts = load_batch_workload(name, "cuda")
    n_total = len(insts)
    if world > 1:
        insts = replicas.shard(insts, rank, world)
        slots = assign_slots(insts, len(bases))
    P = wl["particles"]
    t0 = time.perf_counter()
    batch = Batch(bases, slots=slots, max_particles=P, device=local_rank, autotune=True)
    tune_s = time.perf_counter() - t0
    fill_batch(batch, wl, insts)
    stream = torch.cuda.ExternalStream(batch.stream, device=dev)
    flush_w = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    flush_r = torch.ones(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    sink = torch.empty((), dtype=torch.float32, device=dev)
    K = max(1, args.batch_steps)
    batch.step(max(3, args.warmup))
    batch.sync()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    with torch.cuda.stream(stream):
        for i in range(K):
            if flush:
                flush_w.zero_()
                torch.sum(flush_r, dim=0, out=sink)
            starts[i].record(stream)
            batch.step(1)
            ends[i].record(stream)
    torch.cuda.synchronize(dev)
    per_step = np.array([a.elapsed_time(b) for a, b in zip(starts, ends)])
    total_ms = float(per_step.sum())
    B = len(insts)
    value = B * K / (total_ms / 1e3)
    # Per kernel, L2 flushed before each profiled step: the phases as separate
    # launches, and the step as it runs (one fused tensor-core launch + tracer).
    names = ["contract", "state", "reconstruct", "trace"]
    acc = np.zeros(4)
    fused_acc = None
    M = min(K, 20)
    for _ in range(M):
        with torch.cuda.stream(stream):
            flush_w.zero_()
            torch.sum(flush_r, dim=0, out=sink)
        acc += batch.profile_phases()
        if batch.info()["kernels_per_step"] == 2:
            with torch.cuda.stream(stream):
                flush_w.zero_()
                torch.sum(flush_r, dim=0, out=sink)
            f = batch.profile_step()
            fused_acc = f if fused_acc is None else fused_acc + f
    kms = acc / M
    peak, peak_kind = measured_peak_hbm()
    tpeak = measured_peak_tensor()
    kern = {}
    for n_, m in zip(names, kms):
        by, fl = batch_kernel_bytes(bases, slots, insts, n_)
        kern[n_] = {"ms": round(float(m), 5), "algorithmic_bytes": int(by), "GB/s": round(by / (m / 1e3) / 1e9, 1),
                    "frac_hbm": round(by / (m / 1e3) / 1e9 / peak, 4)}
        if fl:
            kern[n_]["TFLOP/s"] = round(fl / (m / 1e3) / 1e12, 1)
            kern[n_]["frac_tensor"] = round(fl / (m / 1e3) / 1e12 / tpeak, 4)
    if fused_acc is not None:
        fms = fused_acc / M
        by = sum(kern[n_]["algorithmic_bytes"] for n_ in ("contract", "state", "reconstruct"))
        fl = sum(batch_kernel_bytes(bases, slots, insts, n_)[1] for n_ in ("contract", "reconstruct"))
        kern["step_tc"] = {"ms": round(float(fms[0]), 5), "algorithmic_bytes": int(by),
                           "GB/s": round(by / (fms[0] / 1e3) / 1e9, 1),
                           "frac_hbm": round(by / (fms[0] / 1e3) / 1e9 / peak, 4),
                           "TFLOP/s": round(fl / (fms[0] / 1e3) / 1e12, 1),
                           "frac_tensor": round(fl / (fms[0] / 1e3) / 1e12 / tpeak, 4),
                           "note": "one cooperative launch: contraction, FP64 state update, reconstruction"}
        kern["trace_in_step"] = {"ms": round(float(fms[1]), 5)}
        kms_step = {"step_tc": kern["step_tc"]["ms"], "trace": kern["trace_in_step"]["ms"]}
    else:
        kms_step = {n_: kern[n_]["ms"] for n_ in names}
    dom = max(kms_step, key=kms_step.get)
    if dom == "trace":
        dom_k = "trace"
    else:
        dom_k = dom
    roof = {"kernel": dom_k, "bound": "hbm", "achieved": kern[dom_k]["GB/s"], "peak": peak, "unit": "GB/s",
            "frac": kern[dom_k]["frac_hbm"], "peak_source": peak_kind,
            "algorithmic_bytes": kern[dom_k]["algorithmic_bytes"],
            "traffic": NCU_TRAFFIC.get((name, dom_k)), "all_kernels": kern}
    # End to end through the public API: every rollout set from host buffers,
    # stepped, and read back (state and particles), per E steps.
    E = max(1, min(K, 20))
    t0e = torch.cuda.Event(enable_timing=True)
    t1e = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    t0e.record(stream)
    fill_batch(batch, wl, insts)
    batch.step(E)
    h2d = d2h = 0
    for x in insts:
        w = batch.get_state(x["basis"], x["slot"])
        p = batch.get_particles(x["basis"], x["slot"])
        d2h += w.nbytes + p.nbytes
        h2d += x["w0"].nbytes + x["parts"].nbytes
    t1e.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = t0e.elapsed_time(t1e)
    e2e = {"value": round(B * E / (e2e_ms / 1e3), 2), "unit": "instance-steps/s",
           "h2d_bytes_per_step": int(h2d // E), "d2h_bytes_per_step": int(d2h // E),
           "rollout_steps": E}
    out = {"value": round(value, 2), "unit": "instance-steps/s", "instances": B, "instances_total": n_total,
           "steps": K,
           "ms_per_step": round(total_ms / K, 5), "p50_ms": round(float(np.percentile(per_step, 50)), 5),
           "p99_ms": round(float(np.percentile(per_step, 99)), 5),
           "particle_steps_per_s": round(value * P, 1), "kernel_ms": kms_step,
           "phase_ms": {n_: round(float(m), 5) for n_, m in zip(names, kms)},
           "roofline": roof, "e2e": e2e, "gpu_launches": int(batch.info()["kernels_per_step"] * K),
           "batch": batch.info(),
           "autotune_s": round(tune_s, 3), "describe": wl["describe"]}
    if check:
        out["accuracy"] = batch_accuracy(batch, wl, bases, insts, local_rank)
    batch.close()
    if plain and args.plain_sample > 0:
        out["plain_path"] = plain_sample(wl, bases, insts, local_rank, args.plain_sample)
        out["speedup_vs_plain"] = round(value / out["plain_path"]["instance_steps_per_s"], 3)
    return out


def plain_sample(wl, bases, insts, device, count):
    """The plain FP32 single-instance path (one context per instance) on a sample of the same instances."""
    import torch

    from parallelspectralfluids3d_b200 import _lib as L
    from parallelspectralfluids3d_b200.solver import Context

    idx = np.linspace(0, len(insts) - 1, min(count, len(insts))).astype(int)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps, ms = 0, 0.0
    for i in idx:
        x = insts[i]
        flags = L.PSF_FLAG_RENORM | (L.PSF_FLAG_FORCING if wl["force0"] else 0)
        ctx = Context(bases[x["basis"]].truncate(x["n"]), L.make_params(dt=wl["dt"], integrator=wl["integrator"],
                                                                         flags=flags), device=device)
        if wl["force0"]:
            ctx.set_forcing(x["force"])
        ctx.set_state(x["w0"])
        ctx.set_particles(x["parts"])
        ctx.step(3)
        ctx.sync()
        st = torch.cuda.ExternalStream(ctx.stream)
        k = 20
        e0.record(st)
        ctx.step(k)
        e1.record(st)
        ctx.sync()
        ms += e0.elapsed_time(e1)
        steps += k
        ctx.close()
    return {"instances": int(len(idx)), "steps_each": 20, "instance_steps_per_s": round(steps / (ms / 1e3), 1),
            "note": "one context per instance, stepped back to back (graph replay), same inputs as the batch"}


def batch_accuracy(batch, wl, bases, insts, device):
    """Relative error of w (and particle error) against the FP64 oracle after the full step count."""
    from oracle import oracle as O

    S = wl["full_steps"]
    fill_batch(batch, wl, insts)
    batch.step(S)
    res = []
    for i in wl["check"]:
        x = insts[i]
        b = bases[x["basis"]].truncate(x["n"])
        withp = i in wl["check_particles"]
        ref = O.OracleRollout(b, x["w0"], x["parts"] if withp else None, dt=wl["dt"], integrator=wl["integrator"],
                              forcing=x["force"] if wl["force0"] else None, seed=x["seed_p"],
                              reconstruct=withp).step(S)
        w = batch.get_state(x["basis"], x["slot"])
        r = {"instance": i, "n_modes": x["n"], "rel_err_w_vs_fp64": float(np.linalg.norm(w - ref.w) / np.linalg.norm(ref.w))}
        if withp:
            p = batch.get_particles(x["basis"], x["slot"])
            d = np.abs(p[:, :3] - ref.pos).max(axis=1) / bases[x["basis"]].h
            r["max_particle_err_voxels"] = float(d.max())
            r["p99_particle_err_voxels"] = float(np.percentile(d, 99))
        res.append(r)
    return {"steps": S, "instances": res,
            "max_rel_err_w": max(r["rel_err_w_vs_fp64"] for r in res)}


def run_batch_line(args, rank, world, local_rank):
    """Bench line of a batched workload (every rank runs its own batch: weak scaling)."""
    import torch

    args.batch_steps = args.steps if args.steps else args.batch_steps
    clocks = ClockSampler(local_rank).start()
    r = run_batch(args, args.workload, local_rank, check=(rank == 0 and world == 1 and not args.no_cpu),
                  plain=(world == 1), rank=rank, world=world)
    clk = clocks.stop()
    total_ms = r["ms_per_step"] * r["steps"]
    e2e_v = r["e2e"]["value"]
    total_ms, inv = replicas.slowest([total_ms, 1.0 / max(e2e_v, 1e-30)], device=torch.device("cuda", local_rank))
    e2e_v = 1.0 / inv
    # Whole job: every rank's instances (a round-robin share of the workload)
    # over the slowest rank's device time.
    value = r["instances_total"] * r["steps"] / (total_ms / 1e3)
    e2e = dict(r["e2e"], value=round(e2e_v * r["instances_total"] / r["instances"], 2))
    line = {"metric": "instance-steps/s", "value": round(value, 2), "unit": "instance-steps/s", "n_gpus": world,
            "steps": r["steps"], "warmup": max(3, args.warmup), "ms_per_step": r["ms_per_step"],
            "higher_is_better": True, "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
            "dtype": "bf16x2", "state_dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "describe": r["describe"], "instances": r["instances_total"],
                       "instances_per_gpu": r["instances"],
                       "l2": "flushed before every timed step (256 MB write, then 256 MB read)",
                       "parallelism": f"instances sharded round-robin over {world} GPU(s)"},
            "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"], "particle_steps_per_s": round(value * r["particle_steps_per_s"] / max(r["value"], 1e-30), 1),
            "gpu_launches": r["gpu_launches"], "kernel_ms": r["kernel_ms"], "roofline": r["roofline"], "e2e": e2e,
            "clocks": clk, "batch": r["batch"]}
    if "accuracy" in r:
        line["accuracy"] = r["accuracy"]
    for k in ("plain_path", "speedup_vs_plain"):
        if k in r:
            line[k] = r[k]
    return line


def measured_peak_tensor():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["bf16_tflops"])
    return 1590.0



def run_reference_batch(args):
    """The reference CPU step on a bounded sample of a batched workload's instances."""
    from oracle import oracle as O

    O.build()
    wl, bases, slots, insts = load_batch_workload(args.workload, "cpu")
    K = max(1, min(args.steps, 10))
    sample = insts[: min(len(insts), len(bases) * 2)]
    rolls = [O.OracleRollout(bases[x["basis"]].truncate(x["n"]), x["w0"], x["parts"], dt=wl["dt"],
                             integrator=wl["integrator"], forcing=x["force"] if wl["force0"] else None,
                             seed=x["seed_p"]) for x in sample]
    for r in rolls:
        r.step(max(1, min(3, args.warmup)))
    t0 = time.perf_counter()
    for r in rolls:
        r.step(K)
    dt = time.perf_counter() - t0
    value = len(rolls) * K / dt
    desc = f"{K} steps of each of {len(rolls)} instances (one at a time, all threads), FP64"
    return {
        "impl": "reference", "metric": "instance-steps/s", "value": round(value, 3), "unit": "instance-steps/s",
        "n_gpus": 1, "steps": K, "warmup": max(3, args.warmup), "ms_per_step": round(1e3 * dt / (K * len(rolls)), 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "describe": wl["describe"]},
        "cpu_baseline": {"value": round(value, 3), "unit": "instance-steps/s", "cores": O.num_threads(),
                         "kind": "port", "sample": desc},
        "e2e": {"value": round(value, 3), "unit": "instance-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------------------ serving arm
SERVE_WORKLOAD = "serve_poisson200"
SERVE_DOMAINS = [(("box", 32, None), 384), (("sphere", 40, 10.0), 384), (("channel", (64, 32, 32), None), 384)]


def serve_requests(seconds, rate=200.0, seed=7, n_max=384):
    """Poisson request stream: arrival time, domain, N, steps, particle count, seeds."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            break
        out.append(dict(t=t, basis=int(rng.integers(0, 3)), n=int(rng.integers(64, n_max + 1)),
                        steps=int(rng.integers(50, 1001)), P=int(np.exp(rng.uniform(np.log(1e4), np.log(1e6)))),
                        seed=int(rng.integers(0, 2**31 - 1))))
    return out


def run_serve(args, local_rank, rank=0, world=1, shared=None):
    """Continuous-batching serving run: real-time Poisson arrivals through the engine.

    With ``world > 1`` every rank runs its own engine on its round-robin share
    of the request stream (same arrival times), and rank 0 combines the
    ranks' completions (replicas.combine_serving): whole-job instance-steps/s
    over the span from the first submission to the last completion on any
    rank, latency percentiles over every request.  ``shared`` (a dict) keeps
    the bases, particle clouds and the plain-path sample between runs of
    different arrival rates: the request parameters do not depend on the rate.
    """
    import threading

    import torch

    from parallelspectralfluids3d_b200 import _lib as L
    from parallelspectralfluids3d_b200.engine import Engine
    from parallelspectralfluids3d_b200.fixture import cached_basis, initial_coefficients, initial_particles

    torch.cuda.set_device(local_rank)
    shared = {} if shared is None else shared
    if "bases" not in shared:
        bases = []
        for spec, n in SERVE_DOMAINS:
            dom = make_domain(spec)
            bases.append(cached_basis(dom, n, cache_dir=basis_cache_for(dom.name, n), device="cuda"))
        shared["bases"] = bases
        # Particle sources: one seeded cloud per domain, each request takes a slice.
        shared["clouds"] = [initial_particles(b, 2_000_000, 70 + i) for i, b in enumerate(bases)]
    bases, clouds = shared["bases"], shared["clouds"]
    all_reqs = serve_requests(args.serve_seconds, rate=args.serve_rate, n_max=min(b.n_modes for b in bases))
    for i, q in enumerate(all_reqs):
        q["index"] = i
    reqs = replicas.shard(all_reqs, rank, world) if world > 1 else all_reqs
    for q in reqs:
        off = int(np.random.default_rng(q["seed"]).integers(0, 2_000_000 - q["P"]))
        q["off"] = off
        q["w0"] = initial_coefficients(q["n"], q["seed"])
    params = L.make_params(dt=0.005, integrator=L.PSF_RK4, precision=L.PSF_PRECISION_BF16X2)
    eng = Engine(bases, slots=args.serve_slots, max_particles=1_000_000, particle_pool=args.serve_pool,
                 hbm_budget_bytes=int(args.serve_budget_gb * 2**30), chunk_steps=args.serve_chunk,
                 device=local_rank, autotune=True)
    ids = {}
    lat, done = [], []
    stop = threading.Event()

    def producer():
        t0 = time.perf_counter()
        for i, q in enumerate(reqs):
            dt = q["t"] - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            parts = clouds[q["basis"]][q["off"]: q["off"] + q["P"]]
            ids[eng.submit(q["basis"], q["w0"], q["steps"], params, particles=parts)] = i

    def consumer():
        while not stop.is_set() or len(done) < len(reqs):
            got = eng.poll(4096)
            if not got:
                if stop.is_set() and len(done) >= len(reqs):
                    break
                time.sleep(0.002)
                continue
            for rid in got:
                w, p, info = eng.collect(rid, want_particles=True)
                lat.append(info["t_done"] - info["t_submit"])
                done.append((ids.get(rid), info, w))

    cons = threading.Thread(target=consumer)
    cons.start()
    t_start = time.perf_counter()
    prod = threading.Thread(target=producer)
    prod.start()
    prod.join()
    eng.drain(3600)
    stop.set()
    cons.join()
    wall = time.perf_counter() - t_start
    st = eng.stats()
    eng.close()
    lat = np.array(lat)
    total_steps = sum(q["steps"] for q in reqs)
    first = min(info["t_submit"] for _, info, _ in done)
    last = max(info["t_done"] for _, info, _ in done)
    if world > 1:
        # Host-side gather of every rank's completions (CLOCK_MONOTONIC is shared by the processes).
        mine = {"requests": [reqs[i]["index"] for i, _, _ in done if i is not None], "latencies": lat.tolist(),
                "steps": total_steps, "first": first, "last": last, "particle_steps": st["particle_steps"]}
        recs = replicas.gather_objects(mine)
        job = replicas.combine_serving(recs)
        lat = np.array([x for r in recs for x in r["latencies"]])
        total_steps = job["instance_steps"]
        first = min(r["first"] for r in recs)
        last = max(r["last"] for r in recs)
        st["particle_steps"] = sum(r["particle_steps"] for r in recs)
        st["per_rank_completed"] = job["per_rank_completed"]
        if rank != 0:
            return None
    out = {"requests": len(all_reqs), "completed": int(lat.size), "arrival_window_s": args.serve_seconds,
           "arrival_rate_per_s": args.serve_rate, "gpus": world,
           # Work offered per second of the arrival window: the served rate
           # cannot exceed it while the engine keeps up with the arrivals.
           "offered_instance_steps_per_s": round(sum(q["steps"] for q in all_reqs) / args.serve_seconds, 1),
           "instance_steps": total_steps, "instance_steps_per_s": round(total_steps / (last - first), 1),
           "particle_steps_per_s": round(st["particle_steps"] / (last - first), 1),
           "p50_latency_s": round(float(np.percentile(lat, 50)), 4),
           "p99_latency_s": round(float(np.percentile(lat, 99)), 4),
           "mean_latency_s": round(float(lat.mean()), 4), "makespan_s": round(last - first, 3),
           "wall_s": round(wall, 3), "engine": st,
           "config": {"arrival_rate_per_s": args.serve_rate, "arrival_window_s": args.serve_seconds,
                      "slots_per_domain": args.serve_slots, "particle_pool": args.serve_pool,
                      "hbm_budget_gb": args.serve_budget_gb, "chunk_steps": args.serve_chunk,
                      "n_range": [64, min(b.n_modes for b in bases)]}}
    # Accuracy of a few served rollouts against the FP64 oracle (w only).
    if not args.no_cpu:
        from oracle import oracle as O

        by_idx = {i: w for i, _, w in done if i is not None}
        errs = []
        refs = shared.setdefault("oracle_w", {})  # FP64 results by request parameters
        for i in sorted(by_idx)[:3]:
            q = reqs[i]
            rk = (q["basis"], q["n"], q["steps"], q["seed"])
            if rk not in refs:
                refs[rk] = O.OracleRollout(bases[q["basis"]].truncate(q["n"]), q["w0"], None, dt=0.005, integrator=4,
                                           reconstruct=False).step(q["steps"]).w
            ref_w = refs[rk]
            errs.append({"request": i, "n_modes": q["n"], "steps": q["steps"],
                         "rel_err_w_vs_fp64": float(np.linalg.norm(by_idx[i] - ref_w) / np.linalg.norm(ref_w))})
        out["accuracy"] = errs
    # The plain FP32 single-instance path on a sample of the same requests.
    from parallelspectralfluids3d_b200.solver import Context

    sample = reqs[: args.serve_plain_sample]
    key = tuple((q["basis"], q["n"], q["steps"], q["P"], q["seed"]) for q in sample)
    if shared.get("plain_key") == key:
        out["plain_path_instance_steps_per_s"] = shared["plain_rate"]
        out["speedup_vs_plain"] = round(out["instance_steps_per_s"] / out["plain_path_instance_steps_per_s"], 3)
        return out
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    plain_steps, plain_ms = 0, 0.0
    for q in sample:
        b = bases[q["basis"]].truncate(q["n"])
        ctx = Context(b, L.make_params(dt=0.005, integrator=L.PSF_RK4), device=local_rank)
        ctx.set_state(q["w0"])
        ctx.set_particles(clouds[q["basis"]][q["off"]: q["off"] + q["P"]])
        k = min(q["steps"], 50)
        # Four untimed steps: the first steps after set-up capture the
        # pipelined step's graphs (after a change, start-up, steady state).
        ctx.step(4)
        ctx.sync()
        st_ = torch.cuda.ExternalStream(ctx.stream)
        ev0.record(st_)
        ctx.step(k)
        ev1.record(st_)
        ctx.sync()
        plain_ms += ev0.elapsed_time(ev1)
        plain_steps += k
        ctx.close()
    out["plain_path_instance_steps_per_s"] = round(plain_steps / (plain_ms / 1e3), 1)
    out["speedup_vs_plain"] = round(out["instance_steps_per_s"] / out["plain_path_instance_steps_per_s"], 3)
    shared["plain_key"], shared["plain_rate"] = key, out["plain_path_instance_steps_per_s"]
    return out


# Serving form of the default line: the configured request mix at 200 req/s
# over a 15 s window (latency at a load the engine keeps up with; the served
# rate then equals the offered one), and the same mix arriving at 2000 req/s
# over 4 s (about 8,000 requests queued at once: the engine's capacity).  The
# engine's slots and chunk differ: a step's tensor-core work grows with the
# slots, not with the rollouts in them, so the latency run keeps 96 slots per
# domain (about 55 rollouts per domain are in flight at 200 req/s) and the
# capacity run takes 192 with 16-step chunks.
SERVE_FORM_RUNS = (
    ("poisson200_15s", 200.0, 15.0, dict(serve_slots=96, serve_pool=64_000_000, serve_budget_gb=16.0,
                                         serve_chunk=8)),
    ("saturated_2000_4s", 2000.0, 4.0, dict(serve_slots=192, serve_pool=128_000_000, serve_budget_gb=32.0,
                                            serve_chunk=16)),
)


def run_serve_form(args, local_rank):
    import copy

    shared, out = {}, {}
    for name, rate, seconds, engine in SERVE_FORM_RUNS:
        a = copy.copy(args)
        a.serve_rate, a.serve_seconds = rate, seconds
        for k, v in engine.items():
            setattr(a, k, v)
        t0 = time.perf_counter()
        r = run_serve(a, local_rank, shared=shared)
        r["wall_s"] = round(time.perf_counter() - t0, 1)
        out[name] = r
    return out



def run_for_profiler(args):
    """Set up the workload and launch ``args.ncu`` steps kernel by kernel (for ncu captures)."""
    import torch

    from parallelspectralfluids3d_b200 import _lib as L
    from parallelspectralfluids3d_b200.solver import Context

    if args.workload in BATCH_WORKLOADS:
        from parallelspectralfluids3d_b200.batch import Batch

        wl, bases, slots, insts = load_batch_workload(args.workload, "cuda",
                                                      particles=args.ncu_particles or None)
        if args.ncu_instances:
            insts = insts[: args.ncu_instances]
            slots = assign_slots(insts, len(bases))
        batch = Batch(bases, slots=slots, max_particles=max(len(x["parts"]) for x in insts), autotune=False)
        fill_batch(batch, wl, insts)
        for _ in range(args.ncu):
            # --ncu-phases: contraction, state update, reconstruction and tracer as separate launches.
            ms = batch.profile_phases() if args.ncu_phases else batch.profile_step()
        torch.cuda.synchronize()
        print(json.dumps({"profiled_steps": args.ncu, "batch": batch.info(),
                          "last_step_kernel_ms": [round(float(m), 5) for m in ms]}))
        batch.close()
        return
    wl, b, w0, parts, force = load_workload(args.workload, "cuda")
    params = L.make_params(dt=wl["dt"], integrator=wl["integrator"],
                           flags=L.PSF_FLAG_RENORM | (L.PSF_FLAG_FORCING if wl["force0"] else 0))
    ctx = Context(b, params, device=0)
    ctx.set_forcing(force)
    ctx.set_state(w0)
    ctx.set_particles(parts)
    for _ in range(args.ncu):
        ms = ctx.profile_step()
    torch.cuda.synchronize()
    print(json.dumps({"profiled_steps": args.ncu, "last_step_kernel_ms": [round(float(m), 5) for m in ms]}))
    ctx.close()


# ---------------------------------------------------------------- the steps before and after the path
# Mesh voxeliser (Graphics/Model/Model.cpp:203-451) and particle density volume + ray march
# (Solver/SolverImpl/psfsolvergpu.cpp:876-1022): not on the instance-steps/s metric; each prints
# its own line.
AUX_WORKLOADS = {
    "voxel_sphere_512": "icosphere with 1,310,720 triangles (radius 0.45) voxelised at 512^3, geometric mode",
    "volume_cloud256": "16,777,216 particles (normal cloud, sigma 0.12) splatted into 256^3 FP16 density, "
                       "ray-marched at 1280x720 with shadow rays",
}


def run_aux(args):
    """One JSON line for a voxeliser or volume workload (device time, end to end, CPU sample)."""
    from parallelspectralfluids3d_b200 import volume as VOL
    from parallelspectralfluids3d_b200 import voxel as VX

    peak, peak_kind = measured_peak_hbm()
    clocks = ClockSampler(0).start()
    steps = max(1, args.steps if args.steps <= 50 else 20)
    if args.workload == "voxel_sphere_512":
        v, t = VX.icosphere(8, 0.45)
        res = 0.9 / 512
        (W, H, D), _, _ = VX.grid(v, res, VX.GEOMETRIC)
        nvox = W * H * D
        vz = VX.Voxelizer(len(v), len(t), nvox)
        for _ in range(max(1, args.warmup)):
            inside, *_ = vz.run(v, t, res, VX.GEOMETRIC)
        t0 = time.perf_counter()
        for _ in range(steps):
            inside, *_ = vz.run(v, t, res, VX.GEOMETRIC)
        e2e_s = (time.perf_counter() - t0) / steps
        ms = vz.profile(steps)
        vz.close()
        words = D // 32 + 1
        alg = 12 * len(v) + 16 * len(v) + 12 * len(t) + 48 * len(t) + 4 * words * W * H + nvox
        line = {"metric": "voxels/s", "value": nvox / (ms / 1e3), "unit": "voxels/s", "ms_per_mesh": ms,
                "e2e": {"value": nvox / e2e_s, "unit": "voxels/s", "h2d_bytes_per_step": 12 * len(v) + 12 * len(t),
                        "d2h_bytes_per_step": nvox},
                "roofline": {"bound": "hbm", "achieved": alg / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                             "frac": alg / (ms / 1e3) / 1e9 / peak, "peak_kind": peak_kind, "traffic": None,
                             "note": "three kernels (transform, raster, unpack) timed together"},
                "inside_voxels": int(inside.sum())}
        if not args.no_cpu:
            from oracle import voxel_oracle as VO

            t0 = time.perf_counter()
            want = VO.voxelize(v, t, res, VO.GEOMETRIC)
            cpu_s = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": want.size / cpu_s, "unit": "voxels/s", "cores": 1, "kind": "port",
                                    "sample": "the whole workload once (oracle, one thread)"}
            line["matches_oracle"] = bool(np.array_equal(want, inside))
    else:
        rng = np.random.default_rng(11)
        P = 1 << 24
        p = np.concatenate([rng.normal(0.0, 0.12, (P, 3)), np.full((P, 1), 100.0)], 1).astype(np.float32)
        mn = np.array([-0.5] * 3, np.float32)
        mx = -mn
        view = VOL.make_view(1280, 720, eye=(0.3, 0.4, 1.6))
        vol = VOL.Volume(256)
        for _ in range(max(1, args.warmup)):
            vol.splat(p, mn, mx)
            img = vol.render(view)
        t0 = time.perf_counter()
        for _ in range(steps):
            vol.splat(p, mn, mx)
            img = vol.render(view)
        e2e_s = (time.perf_counter() - t0) / steps
        splat_ms, render_ms = vol.profile(view, steps)
        vol.close()
        cells = 256 ** 3
        alg = 16 * P + 4 * cells * 3 + 2 * cells  # particles in, counts read+cleared (+atomics), FP16 out
        line = {"metric": "frames/s", "value": 1e3 / (splat_ms + render_ms), "unit": "frames/s",
                "splat_ms": splat_ms, "render_ms": render_ms,
                "e2e": {"value": 1.0 / e2e_s, "unit": "frames/s", "h2d_bytes_per_step": 16 * P,
                        "d2h_bytes_per_step": 16 * 1280 * 720},
                "roofline": {"bound": "hbm", "achieved": alg / (splat_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                             "frac": alg / (splat_ms / 1e3) / 1e9 / peak, "peak_kind": peak_kind, "traffic": None,
                             "note": "splat kernels only; the ray march is bound by L2-resident samples"},
                "mean_transmittance": float(img[..., 3].mean())}
        if not args.no_cpu:
            from oracle import volume_oracle as VO

            t0 = time.perf_counter()
            d = VO.density(VO.histogram(p, mn, mx, 256))
            cpu_splat = time.perf_counter() - t0
            small = dict(view, width=320, height=180)
            t0 = time.perf_counter()
            VO.render(d, small, mn, mx)
            cpu_px = (time.perf_counter() - t0) / (320 * 180)
            cpu_frame = cpu_splat + cpu_px * 1280 * 720
            line["cpu_baseline"] = {"value": 1.0 / cpu_frame, "unit": "frames/s", "cores": 1, "kind": "port",
                                    "sample": "full splat + the same view at 320x180, scaled per pixel to 1280x720 "
                                              "(oracle, one thread)"}
    line.update({"n_gpus": 1, "steps": steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                 "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                 "config": {"workload": args.workload, "describe": AUX_WORKLOADS[args.workload]},
                 "gpu_launches": 3 * steps,  # transform, raster, unpack / histogram, density, render
                 "clocks": clocks.stop()})
    return line



def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + sorted(BATCH_WORKLOADS) + [SERVE_WORKLOAD]
                    + sorted(AUX_WORKLOADS),
                    default=DEFAULT_WORKLOAD)
    ap.add_argument("--no-cpu", action="store_true", help="skip the FP64 accuracy/CPU baseline leg")
    ap.add_argument("--no-forms", action="store_true", help="skip the batched tensor-core form in the default line")
    ap.add_argument("--batch-steps", type=int, default=50, help="timed steps of a batched workload")
    ap.add_argument("--ncu-instances", type=int, default=0, help="profiling driver: only the first K instances")
    ap.add_argument("--ncu-particles", type=int, default=0, help="profiling driver: particles per instance")
    ap.add_argument("--ncu-phases", action="store_true",
                    help="profiling driver: run the batched phases as separate launches")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="serving: length of the arrival window")
    ap.add_argument("--serve-rate", type=float, default=200.0, help="serving: Poisson arrival rate (requests/s)")
    ap.add_argument("--serve-slots", type=int, default=96, help="serving: concurrent rollouts per domain")
    ap.add_argument("--serve-pool", type=int, default=64_000_000, help="serving: particles resident at once")
    ap.add_argument("--serve-budget-gb", type=float, default=16.0, help="serving: device budget of admitted rollouts")
    ap.add_argument("--serve-chunk", type=int, default=8, help="serving: steps between admission rounds")
    ap.add_argument("--serve-plain-sample", type=int, default=32, help="serving: requests timed on the plain path")
    ap.add_argument("--plain-sample", type=int, default=12, help="batched: instances timed on the plain path")
    ap.add_argument("--ncu", type=int, default=0, metavar="S",
                    help="profiling driver: set up the workload, then run S steps kernel by kernel and exit")
    args = ap.parse_args()
    if args.ncu:
        run_for_profiler(args)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.workload in AUX_WORKLOADS:
        if rank == 0 and args.impl == "ours":
            print(json.dumps(run_aux(args)), flush=True)
        elif rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference runs this step through OpenGL, "
                              "which is unavailable on this box; the CPU restatement is reported as cpu_baseline"}))
        return

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return

    if world > 1:
        import datetime

        import torch
        import torch.distributed as td

        torch.cuda.set_device(local_rank)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                              device_id=torch.device("cuda", local_rank))
    try:
        if args.workload == SERVE_WORKLOAD:
            clocks = ClockSampler(local_rank).start()
            r = run_serve(args, local_rank, rank, world)
            clk = clocks.stop()
            line = None
            if rank == 0:
                line = {"metric": "instance-steps/s", "value": r["instance_steps_per_s"], "unit": "instance-steps/s",
                        "n_gpus": world, "higher_is_better": True, "scaling": "strong" if world > 1 else "weak",
                        "vs_baseline": None, "dtype": "bf16x2", "state_dtype": "f64", "data": "synthetic",
                        "p50_ms": round(1e3 * r["p50_latency_s"], 2), "p99_ms": round(1e3 * r["p99_latency_s"], 2),
                        "config": {"workload": SERVE_WORKLOAD, **r.pop("config")}, "serve": r, "clocks": clk}
        elif args.workload in BATCH_WORKLOADS:
            line = run_batch_line(args, rank, world, local_rank)
        else:
            line = run_ours(args, rank, world, local_rank)
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as td

            td.destroy_process_group()


if __name__ == "__main__":
    main()
