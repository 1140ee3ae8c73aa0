"""Benchmark: face-updates/sec of fvmhd3d's per-timestep fluid hot path on B200.

One step = the reference's full per-step sequence on the GPU (slope limiter,
corrector flux + scatter, mesh velocity, CFL timestep, predictor flux +
scatter, gradient reconstruction) over every active face of a fixed periodic
Voronoi mesh.  One face-update = one active face through one such step.

Default workload: MHD blast wave on 128^3 = 2,097,152 jittered-lattice
generators (the 2M-point blast of the target), global timestep, plain FP64.
The state (~2 GB) is far larger than the 126 MB L2, so no L2 flush is needed
between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fvm|reference]

Under torchrun (N > 1) every rank runs an independent replica on its own GPU
(the single-GPU path does not shard: replicas only); value = all ranks' face
updates / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "face-updates/sec on 1 B200"
UNIT = "face-updates/s"

# Algorithmic (compulsory) HBM bytes of each kernel class, per launch, as a
# function of cells N and active faces F: every array the kernel must read or
# write, touched once.  Face record = s1,s2 (8) + normal (24) + centroid (24)
# = 56 B, as in the reference's Face.
def kernel_bytes(name, N, F, prec_bytes=8):
    w = prec_bytes
    table = {
        # reads Wrec (50 w) + tlast/flags per cell, face records; writes tau (10 w)
        # and the two extrapolated face states (20 w per face)
        "limiter": N * (50 * w + 8 + 1) + F * 56 + N * 10 * w + F * 20 * w,
        # reads the face states, face records, vel + tlast per cell; writes the
        # face contribution (14 w) and code
        "corr_flux": F * 20 * w + F * 56 + N * (24 + 8) + F * (14 * w + 1),
        # reads face contributions, U, dU, Wrec w,t, tau; writes U, dU
        "corr_cell": F * (14 * w + 1) + N * (80 + 112 + 20 * w + 10 * w) + N * (80 + 112),
        "pred_flux": N * (10 * w + 24) + F * 56 + F * (14 * w + 1),
        # reads face contributions and U; writes Wrec t, rung, tend
        "pred_cell": F * (14 * w + 1) + N * 80 + N * (10 * w + 12),
        # reads Wst (neighbours), face records, Wrec t; writes Wrec
        "recon": F * 56 + N * (10 * w + 24 + 10 * w) + N * 50 * w,
        "timestep": N * (80 + 24 + 8 + 8) + F * 8 + N * 8,
        "pvel": N * (80 + 24 + 24 + 8) + N * 24,
        "wst": N * 80 + N * 10 * w,
        "flags": N * 4 + F * 8 + N,
        "rungs": N * (8 + 4 + 8 + 8),
        "sync": N * 12,
    }
    return table.get(name)


# DRAM bytes (read + write) per launch measured by ncu on the 64^3 blast
# (262144 cells, 2085347 faces; profiles/cell_and_face_kernels_blast64_*_full.md),
# per face; a launch on another mesh of the same kind moves these bytes times
# its face count.
NCU_FACES_64 = 2085347
NCU_TRAFFIC_64 = {
    ("limiter", 8): 293.388800e6 + 305.387264e6, ("limiter", 4): 168.422656e6 + 129.603584e6,
    ("corr_flux", 8): 495.818752e6 + 205.004032e6, ("corr_flux", 4): 328.471296e6 + 95.712000e6,
    ("corr_cell", 8): 460.649728e6 + 42.046464e6, ("corr_cell", 4): 275.880960e6 + 34.968064e6,
    ("pred_flux", 8): 181.350912e6 + 183.134720e6, ("pred_flux", 4): 170.220032e6 + 84.814848e6,
    ("pred_cell", 8): 353.519104e6 + 24.941824e6, ("pred_cell", 4): 192.598272e6 + 16.507392e6,
    ("recon", 8): 416.417024e6 + 127.086336e6, ("recon", 4): 243.891968e6 + 49.104128e6,
}
# FP64 floating-point operations per launch on the same 64^3 launches (ncu
# thread-instruction counts: 2 per DFMA, 1 per DADD and DMUL; this includes
# the FMAs inside the compiler's divide and square-root sequences).  The plain
# FP64 path is compared with the measured FP64 FMA peak (fvm_fp64_peak).
NCU_FP64_FLOPS_64 = {
    "limiter": 0.8236e9, "corr_flux": 1.4451e9, "corr_cell": 0.2531e9, "pred_flux": 1.4389e9,
    "pred_cell": 0.2497e9, "recon": 1.0849e9,
}


def step_bytes(N, F, prec_bytes=8):
    """Bytes per face-update of the whole step (compulsory traffic, per-cell
    data amortised over F/N): face 56 B + cell 1048 B / f for FP64."""
    cell = 1048 if prec_bytes == 8 else 648
    return (56 * F + cell * N) / F


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.out = None

    def start(self):
        try:
            self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.flush()
        rows = []
        with open(self.out.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.out.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- CPU legs --

def _cpu_worker(args):
    """One single-rank reference (or oracle port) process on its own replica
    of the shared host-built mesh: `warmup` untimed and `steps` timed global
    steps of `problem`."""
    mesh_path, problem, steps, warmup, kind = args
    sys.path.insert(0, ROOT)
    import fvmhd3d_b200 as F
    from oracle import pyoracle
    m = F.mesh.Mesh.load(mesh_path)
    W = getattr(F.problems, problem)(m.pos)
    S = pyoracle.RefSystem() if kind == "reference" else pyoracle.OracleSystem()
    S.set_mesh(m)
    S.init_problem(W)
    for _ in range(warmup):
        S.step(shared=True)
    t0 = time.perf_counter()
    for _ in range(steps):
        S.step(shared=True)
    return m.nface * steps, time.perf_counter() - t0


# Host memory one single-rank reference process holds per cell (its system
# arrays plus the loaded mesh; measured 4.9 KB per cell on the 64^3 blast).
CPU_BYTES_PER_CELL = 5000


def host_memory_available():
    """Bytes the host can still give: MemAvailable, capped by a cgroup limit."""
    avail = None
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    avail = int(line.split()[1]) * 1024
    except OSError:
        pass
    for path in ("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory/memory.limit_in_bytes"):
        try:
            with open(path) as f:
                v = f.read().strip()
            if v.isdigit():
                lim = int(v)
                usage = 0
                for up in ("/sys/fs/cgroup/memory.current", "/sys/fs/cgroup/memory/memory.usage_in_bytes"):
                    if os.path.exists(up):
                        with open(up) as g:
                            usage = int(g.read().strip())
                        break
                avail = lim - usage if avail is None else min(avail, lim - usage)
        except (OSError, ValueError):
            pass
    return avail


def cpu_leg(m, problem, steps, warmup, procs=None):
    """Aggregate face-updates/s of P concurrent single-rank CPU processes,
    each on its own replica of the mesh m (the workload's own mesh, built
    once on the host and shared through a file).  Uses the reference's own
    code (oracle/_ref/libfvmref.so) when it was built, else the C oracle.  P
    is the host's core count, lowered when host memory cannot hold that many
    replicas."""
    import multiprocessing as mp
    from oracle import pyoracle
    kind = "reference" if os.path.exists(pyoracle.REF_SO) else "port"
    if not os.path.exists(pyoracle.REF_SO if kind == "reference" else pyoracle.ORACLE_SO):
        raise RuntimeError("CPU checkers are not built (run __graft_entry__.build())")
    P = procs or os.cpu_count() or 1
    avail = host_memory_available()
    if avail:
        P = max(1, min(P, int(0.6 * avail // (CPU_BYTES_PER_CELL * m.ncell))))
    fd, path = tempfile.mkstemp(suffix=".npz")
    os.close(fd)
    try:
        m.save(path)
        ctx = mp.get_context("spawn")
        with ctx.Pool(P) as pool:
            res = pool.map(_cpu_worker, [(path, problem, steps, warmup, kind)] * P)
    finally:
        os.unlink(path)
    faces = sum(r[0] for r in res)
    t = max(r[1] for r in res)
    return {"value": faces / t, "unit": UNIT, "cores": P, "kind": kind,
            "sample": f"{P} concurrent single-rank processes, each {steps} global step(s) of the {problem} on its "
                      f"own replica of the workload's mesh ({m.ncell} cells, {m.nface} faces, Peano-Hilbert "
                      f"order) after {warmup} untimed; no halo exchange"}


# ---------------------------------------------------------------- GPU leg ---

def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def allreduce_max(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def make_workload(F, problem, nside, ncell, order, rank=0):
    """(mesh, primitives, boundary codes, System arguments, global timestep)
    of a workload.  The lattice problems (blast, alfven, orszag_tang) run on
    nside^3 jittered generators with a global timestep; the Keplerian disk on
    ncell generators with individual power-of-two timesteps, isothermal EOS
    and static generators (the mesh is built once; generators that followed
    the flow would need the mesh rebuilt every step).  Cells in
    Peano-Hilbert order (the reference's sort_local_data) unless order is
    "native"."""
    if problem == "disk":
        pos, box = F.problems.disk_generators(ncell, seed=3 + rank)
        if order == "hilbert":
            pos = pos[F.sort_local_data(pos, box)]
        m = F.build_periodic(pos, box)
        W, bnd = F.problems.disk(pos, box)
        sysargs = dict(gamma=1.0, courant=0.4, box=tuple(box), dtmax=1.0 / 16, eos=1, iso_GM=1.0, iso_cfac=0.05,
                       static_mesh=True)
        return m, W, bnd, sysargs, False
    pos = F.jittered_lattice(nside, 0.1, seed=1 + rank)
    if order == "hilbert":
        pos = pos[F.sort_local_data(pos, 1.0)]
    m = F.build_periodic(pos, 1.0)
    return m, getattr(F.problems, problem)(m.pos), None, {}, True


def timed_run(torch, S, steps, shared):
    """(cells, faces, ms) of `steps` steps replayed from the captured step
    graph (captured beforehand), CUDA events on the context's stream."""
    stream = torch.cuda.ExternalStream(S.stream_ptr)
    S.run(1, shared=shared)  # capture outside the timed region
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    cells, faces = S.run(steps, shared=shared)
    e1.record(stream)
    torch.cuda.synchronize()
    return cells, faces, e0.elapsed_time(e1)


def device_bytes_of(torch, local, build):
    """(object, device bytes it holds) of build() by cudaMemGetInfo."""
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(local)[0]
    obj = build()
    torch.cuda.synchronize()
    return obj, free0 - torch.cuda.mem_get_info(local)[0]


def rel_l1(Ub, Ua):
    rel = np.abs(Ub - Ua).sum(axis=0) / np.maximum(np.abs(Ua).sum(axis=0), 1e-300)
    return {"density": float(rel[0]), "energy": float(rel[4]), "momentum": float(rel[1:4].max()),
            "magnetic": float(rel[5:8].max())}


def config2_leg(F, torch, steps=50):
    """The mixed-precision configuration: the blast on 64^3 generators, 50
    global steps, FP32 bulk (reconstruction, limiter, flux) with FP64
    geometry and compensated accumulation: face-updates/s of both paths and
    the FP32 path's relative L1 error per conserved variable against the
    plain FP64 path over the same steps."""
    m, W, _, _, _ = make_workload(F, "blast", 64, 0, "hilbert")
    out = {"workload": "blast 64^3 jittered Voronoi (Peano-Hilbert order), 50 global steps",
           "ncell": m.ncell, "nface": m.nface}
    U = {}
    for name, prec in (("plain_fp64", F.FVM_PREC_FP64), ("fp32_bulk", F.FVM_PREC_FP32)):
        S = F.System(precision=prec)
        S.set_mesh(m)
        S.init_problem(W)
        _, faces, ms = timed_run(torch, S, steps, True)
        U[name] = S.get_state()["U"]
        out[name] = {"value": faces / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps}
        S.close()
    # the first (untimed) step of timed_run is part of both runs alike
    out["fp32_bulk"]["rel_l1_vs_plain_fp64"] = rel_l1(U["fp32_bulk"], U["plain_fp64"])
    out["steps"] = steps + 1
    return out


def config3_leg(F, torch, local, steps=64):
    """The rung-batching configuration: the Keplerian disk on 1,048,576
    generators, individual power-of-two timesteps, FP32 bulk, launch choices
    by the autotuner, each step one replay of the captured step graph."""
    m, W, bnd, sysargs, _ = make_workload(F, "disk", 0, 1 << 20, "hilbert")

    def build():
        S = F.System(precision=F.FVM_PREC_FP32, device=local, **sysargs)
        S.set_mesh(m)
        S.init_problem(W, bnd=bnd)
        return S
    S, dev_bytes = device_bytes_of(torch, local, build)
    for _ in range(8):
        S.step(shared=False)
    tuned = S.autotune(shared=False, steps=3)
    out = {"workload": f"Keplerian disk {m.ncell} static generators, individual timesteps, FP32 bulk",
           "nface": m.nface, "device_bytes": int(dev_bytes), "autotuned": tuned, "steps": steps}
    # the same steps with the persistent rung kernel taking the steps that
    # involve at most 16384 cells (one launch instead of the stage kernels)
    state = S.get_state()
    ticks = S.tsys_ticks
    for key, fused in (("stage_kernels", 0), ("persistent_small_steps", 16384)):
        S.set_state(tsys_ticks=ticks, **{k: state[k] for k in ("vel", "tlast", "tend", "rung", "U", "dU", "wrec")})
        S.set_fused(fused)
        S.run(1, shared=False)  # capture outside the timed region
        f0 = S.fused_steps
        stream = torch.cuda.ExternalStream(S.stream_ptr)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        cells, faces = S.run(steps, shared=False)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out[key] = {"value": faces / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps,
                    "mean_active_cells": cells / steps, "mean_active_faces": faces / steps,
                    "fused_steps": S.fused_steps - f0}
    out["value"] = max(out["stage_kernels"]["value"], out["persistent_small_steps"]["value"])
    out["unit"] = UNIT
    rung = S.get_state()["rung"]
    used, counts = np.unique(rung, return_counts=True)
    out["rungs"] = {int(r): int(c) for r, c in zip(used, counts)}
    S.close()
    return out


def config5_leg(F, torch, local, steps=24):
    """The combined configuration: the Orszag-Tang vortex on 160^3
    generators with individual power-of-two timesteps, plain FP64 against
    learned flux + FP32 bulk, the same steps from the same start: face-updates/s,
    rungs in use, device bytes and the learned path's relative L1 error per
    conserved variable."""
    from fvmhd3d_b200 import learned as L
    m, W, _, _, _ = make_workload(F, "orszag_tang", 160, 0, "hilbert")
    model = L.load_model()
    out = {"workload": "Orszag-Tang vortex 160^3 jittered Voronoi (Peano-Hilbert order), individual timesteps",
           "ncell": m.ncell, "nface": m.nface, "steps": steps}
    U, T = {}, {}
    for name, prec, learned in (("plain_fp64", F.FVM_PREC_FP64, False), ("learned_fp32", F.FVM_PREC_FP32, True)):
        def build():
            S = F.System(precision=prec, device=local)
            S.set_mesh(m)
            S.init_problem(W)
            if learned:
                L.apply(S, model)
                S.set_flux_mode(1, judge=1024, **L.GATE)
            return S
        S, dev_bytes = device_bytes_of(torch, local, build)
        cells, faces, ms = timed_run(torch, S, steps, False)
        st = S.get_state()
        U[name], T[name] = st["U"], S.time
        used, counts = np.unique(st["rung"], return_counts=True)
        r = {"value": faces / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps,
             "mean_active_faces": faces / steps, "rungs": {int(a): int(b) for a, b in zip(used, counts)},
             "device_bytes": int(dev_bytes)}
        if learned:
            ls = S.learn_stats()
            r["network_faces_fraction"] = ls["deferred"] / max(2 * faces, 1)
            r["fallback_fraction"] = ls["fallback"] / max(ls["deferred"], 1)
            r["judged_rel_l1"] = ls["judged_rel_l1"]
        out[name] = r
        S.close()
    out["same_time"] = T["plain_fp64"] == T["learned_fp32"]
    out["learned_fp32"]["rel_l1_vs_plain_fp64"] = rel_l1(U["learned_fp32"], U["plain_fp64"])
    out["speedup_learned_vs_plain_fp64"] = out["learned_fp32"]["value"] / out["plain_fp64"]["value"]
    return out


def remesh_leg(F, S, m, e2e, bnd=None):
    """The mesh installation the reference repeats every step
    (MPI/iterate.cpp:150 rebuilds the mesh; the fluid path then starts from
    the new face and cell lists and generator positions): fvm_set_mesh and
    fvm_set_positions from pinned host arrays (a host that remeshes every
    step keeps them pinned, as it keeps its state for fvm_step_host), with
    the checks and per-link tables they build on the device, timed by the
    host clock around the calls (they synchronise).  With the host's own
    mesh build excluded, as for the reference, the end-to-end rate of a step
    that also reinstalls the mesh is faces / (e2e step time + this time)."""
    import torch

    def pinned(a, dt):
        a = np.ascontiguousarray(a, dt)
        t = torch.empty(a.shape, dtype=torch.from_numpy(a[:0]).dtype, pin_memory=True)
        t.numpy()[...] = a
        return t.numpy()

    arrs = [pinned(m.s1, np.int32), pinned(m.s2, np.int32), pinned(m.n, np.float64), pinned(m.centroid, np.float64),
            pinned(m.volume, np.float64), pinned(m.cell_centroid, np.float64), pinned(m.cell_face_off, np.int64),
            pinned(m.cell_face_ids, np.int32)]
    pos = pinned(m.pos, np.float64)
    b = None if bnd is None else pinned(bnd, np.int32)
    p = F.system._p
    torch.cuda.synchronize()
    ts = []
    for _ in range(3):
        t0 = time.perf_counter()
        S._check(S.L.fvm_set_mesh(S.h, m.ncell, m.nface, *[p(a) for a in arrs]), "fvm_set_mesh")
        S._check(S.L.fvm_set_positions(S.h, p(pos), p(b)), "fvm_set_positions")
        ts.append(time.perf_counter() - t0)
    out = {"set_mesh_ms": round(1e3 * min(ts), 2), "ncell": m.ncell, "nface": m.nface,
           "path": "fvm_set_mesh + fvm_set_positions from pinned host arrays (upload, validation, link and "
                   "reconstruction tables), host clock"}
    if e2e:
        step_s = m.nface / e2e["value"]
        out["e2e_with_remesh"] = {"value": m.nface / (step_s + min(ts)), "unit": UNIT}
    return out


def run_gpu(args):
    import torch
    import fvmhd3d_b200 as F

    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    t0 = time.perf_counter()
    prec = F.FVM_PREC_FP32 if args.precision == "fp32" else F.FVM_PREC_FP64
    m, W, bnd, sysargs, shared = make_workload(F, args.problem, args.nside, args.ncell, args.order, rank)
    mesh_s = time.perf_counter() - t0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(local)[0]
    S = F.System(precision=prec, device=local, **sysargs)
    S.set_mesh(m)
    S.init_problem(W, bnd=bnd)
    torch.cuda.synchronize()
    footprint = free0 - torch.cuda.mem_get_info(local)[0]
    stream = torch.cuda.ExternalStream(S.stream_ptr, device=local)

    for _ in range(args.warmup):
        S.step(shared=shared)
    # launch choices by the library's autotuner (trial steps on a restored state)
    tuned = S.autotune(shared=shared, steps=3)
    fp64_peak = S.fp64_peak() if prec == F.FVM_PREC_FP64 and shared else None  # FLOP/s, this GPU
    torch.cuda.synchronize()
    barrier(ws)

    # per-kernel CUDA-event timing: a profiled pass of eager steps
    S.set_profiling(True)
    n0 = S.launch_count
    prof_steps = max(2, min(args.steps, 5))
    prof_cells = prof_faces = 0
    for _ in range(prof_steps):
        prof_cells += S.step(shared=shared)
        prof_faces += S.active_face_count()
    torch.cuda.synchronize()
    launches_per_step = (S.launch_count - n0) / prof_steps
    ktimes = S.kernel_times()
    S.set_profiling(False)

    # timed region: K steps replayed from the captured step graph
    S.run(1, shared=shared)  # capture outside the timed region
    torch.cuda.synchronize()
    barrier(ws)
    sampler = ClockSampler(local)
    sampler.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    cells, faces = S.run(args.steps, shared=shared)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = int(round(launches_per_step * args.steps))
    ms = ev0.elapsed_time(ev1)
    clocks = sampler.stop()
    ms_max = allreduce_max(ms, ws)
    value = faces * ws / (ms_max / 1e3)

    # end to end through the C-ABI with host-owned state: every step uploads
    # the state from pinned host buffers, steps, and reads the state back
    # (fvm_step_host: the copies of U and dU overlap the stage kernels)
    e2e = None
    if not args.no_e2e:
        n = m.ncell
        pin = lambda shape, dt: torch.empty(shape, dtype=dt, pin_memory=True).numpy()
        st = S.get_state()
        host = {"vel": pin((n, 3), torch.float64), "tlast": pin(n, torch.float64), "tend": pin(n, torch.float64),
                "rung": pin(n, torch.int32), "U": pin((n, 10), torch.float64), "dU": pin((n, 14), torch.float64),
                "wrec": pin((n, 50), torch.float64)}
        for k in host:
            host[k][...] = st[k]
        ticks = S.tsys_ticks
        bytes_in = sum(a.nbytes for a in host.values())
        e_steps = max(1, min(args.steps, 5))
        torch.cuda.synchronize()
        barrier(ws)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e_faces = 0
        for _ in range(e_steps):
            S.step_host(host, shared=shared, tsys_ticks=ticks)
            ticks = S.tsys_ticks
            e_faces += S.active_face_count()
        e1.record(stream)
        torch.cuda.synchronize()
        e_ms = allreduce_max(e0.elapsed_time(e1), ws)
        e2e = {"value": e_faces * ws / (e_ms / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(bytes_in), "d2h_bytes_per_step": int(bytes_in),
               "steps": e_steps,
               "path": "fvm_step_host: pinned host state in and out, U and dU copies overlapped with the stage kernels"}

    peak, peak_kind = load_peaks()
    N, Fc = m.ncell, m.nface
    pb = 8 if prec == F.FVM_PREC_FP64 else 4
    dom = max(ktimes.items(), key=lambda kv: kv[1][0])[0] if ktimes else None
    roofline = None
    if dom:
        tot, calls = ktimes[dom]
        per_launch_s = tot / max(calls, 1) / 1e3
        # bytes of the mean step of the profiled pass: individual steps touch
        # only their active cells and faces
        alg = kernel_bytes(dom, prof_cells / prof_steps, prof_faces / prof_steps, pb) or 0
        ach = alg / per_launch_s / 1e9
        roofline = {"bound": "hbm", "kernel": dom, "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                    "frac": round(ach / peak, 4), "peak_source": peak_kind,
                    "algorithmic_bytes_per_launch": int(alg),
                    "traffic": (int(NCU_TRAFFIC_64[(dom, pb)] * Fc / NCU_FACES_64)
                                if (dom, pb) in NCU_TRAFFIC_64 and shared else None),
                    "traffic_source": "ncu dram bytes of the 64^3 blast launch, scaled by face count",
                    "step_bytes_per_face_update": round(step_bytes(N, Fc, pb), 1),
                    "step_frac": round(value / ws * step_bytes(N, Fc, pb) / 1e9 / peak, 4)}
        if fp64_peak and shared and roofline:
            # the FP64 roof: the same launches' FP64 operations (per face, scaled
            # from the 64^3 counts) over the measured FMA throughput
            scale = Fc / NCU_FACES_64
            fl = {k: NCU_FP64_FLOPS_64[k] * scale for k in NCU_FP64_FLOPS_64}
            kfl = {k: fl[k] / (ktimes[k][0] / max(ktimes[k][1], 1) / 1e3) for k in fl if k in ktimes}
            step_fl = sum(NCU_FP64_FLOPS_64.values()) / NCU_FACES_64  # per face-update
            roofline["fp64"] = {
                "kernel": dom, "achieved": round(kfl.get(dom, 0.0) / 1e12, 3), "peak": round(fp64_peak / 1e12, 3),
                "unit": "TFLOP/s", "frac": round(kfl.get(dom, 0.0) / fp64_peak, 4),
                "flops_per_launch": int(fl.get(dom, 0)),
                "per_kernel_frac": {k: round(v / fp64_peak, 4) for k, v in kfl.items()},
                "step_flops_per_face_update": round(step_fl, 1),
                "step_frac": round(value / ws * step_fl / fp64_peak, 4),
                "source": "ncu FP64 instruction counts of the 64^3 blast launches scaled by face count; "
                          "peak: fvm_fp64_peak (FMA chains, full occupancy, this GPU)"}
    breakdown = {k: {"ms_per_launch": round(v[0] / max(v[1], 1), 4), "share": round(v[0] / max(1e-9, sum(
        x[0] for x in ktimes.values())), 4)} for k, v in ktimes.items()}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if pb == 8 else "f32", "data": "synthetic",
        "config": {"workload": (f"{args.problem} {args.nside}^3 jittered Voronoi, global timestep, "
                                if shared else f"Keplerian disk {N} static generators, individual timesteps, ") +
                               f"{'plain FP64' if pb == 8 else 'FP32 bulk'} path",
                   "steps_mean_active_faces": round(faces / max(args.steps, 1), 1),
                   "ncell": N, "nface_per_step": Fc, "cell_order": args.order, "faces_per_cell": round(Fc / N, 3),
                   "l2": "inputs larger than L2 (state > 2 GB), no flush", "parallelism": f"replicas x{ws}",
                   "mesh_build_s": round(mesh_s, 2), "device_bytes": int(footprint), "autotuned": tuned},
        "roofline": roofline, "kernels": breakdown, "gpu_launches": launches, "e2e": e2e, "clocks": clocks,
        "timing": "value: CUDA events around K graph-replayed steps on the context stream; kernels/roofline: "
                  "CUDA events around each kernel of a separate profiled pass of eager steps",
    }
    # the metric's comparison: learned flux + FP32 bulk against this plain FP64
    # run, same mesh and steps (relative L1 error per conserved variable)
    weights = os.path.join(ROOT, "fvmhd3d_b200", "data", "flux_mlp.npz")
    if (not args.no_learned and shared and args.problem == "blast" and pb == 8 and os.path.exists(weights)):
        line["learned_fp32"] = learned_leg(F, m, W, 100, weights, stream_of=torch.cuda.ExternalStream)
    if not args.no_remesh:
        line["e2e_remesh"] = remesh_leg(F, S, m, e2e, bnd)
    S.close()
    # the other configurations of the target, each on its own mesh (parity
    # cases of the headline are in tests/); rank 0 of a single-GPU run only
    if rank == 0 and ws == 1 and not args.no_configs and args.problem == "blast" and pb == 8:
        for key, fn in (("config2_blast64_fp32", lambda: config2_leg(F, torch)),
                        ("config3_disk1m_fp32_rungs", lambda: config3_leg(F, torch, local)),
                        ("config5_orszag_tang160_learned", lambda: config5_leg(F, torch, local))):
            try:
                line[key] = fn()
            except Exception as e:  # the headline stands without them
                line[key] = {"error": f"{type(e).__name__}: {e}"}
    if rank == 0 and ws == 1 and not args.no_cpu:
        try:
            line["cpu_baseline"] = cpu_leg(m, args.problem, args.cpu_steps, 0)
        except Exception as e:  # the GPU number stands without it
            line["cpu_baseline"] = {"error": str(e)}
    if rank == 0:
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def learned_leg(F, m, W, steps, weights, stream_of):
    """The learned-flux + FP32 bulk path on the same mesh and initial state
    for `steps` global steps: face-updates/s (CUDA events), its relative L1
    error per conserved variable against a plain FP64 run of the same steps
    from the same start, and the judge's error of the network on the faces it
    serves.  The same steps are repeated with the gated faces taking the
    central flux alone (no dissipation) and the local Lax-Friedrichs
    dissipation instead of the network: the network earns its place when its
    error is below both."""
    import torch
    from fvmhd3d_b200 import learned as L
    model = L.load_model(weights)
    ref = F.System(precision=F.FVM_PREC_FP64)
    ref.set_mesh(m)
    ref.init_problem(W)
    ref.run(steps, shared=True)
    Ua = ref.get_state()["U"]
    ref.close()

    def rel_l1(Ub):
        rel = np.abs(Ub - Ua).sum(axis=0) / np.maximum(np.abs(Ua).sum(axis=0), 1e-300)
        return {"density": float(rel[0]), "energy": float(rel[4]), "momentum": float(rel[1:4].max()),
                "magnetic": float(rel[5:8].max())}

    out = {}
    for sur in ("network", "central", "llf"):
        s = F.System(precision=F.FVM_PREC_FP32)
        s.set_mesh(m)
        s.init_problem(W)
        L.apply(s, model)
        s.set_flux_mode(1, judge=1024, **L.GATE)
        s.set_flux_surrogate(sur)
        st = stream_of(s.stream_ptr)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        _, faces = s.run(steps, shared=True)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        stats = s.learn_stats()
        r = {"rel_l1_vs_plain_fp64": rel_l1(s.get_state()["U"]), "judged_rel_l1": stats["judged_rel_l1"]}
        if sur == "network":
            r.update({"value": faces / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps, "steps": steps,
                      "network_faces_fraction": stats["deferred"] / max(2 * faces, 1),
                      "fallback_fraction": stats["fallback"] / max(stats["deferred"], 1),
                      "positivity_fallback_fraction": stats["positivity_fallback"] / max(stats["deferred"], 1),
                      "judged_faces": stats["judged"],
                      "judged_mean_abs_scaled": stats["judged_mean_abs"],
                      "judged_max_abs_scaled": stats["judged_max_abs"],
                      "dtype": "f32 bulk + f16 network", "weights": "fvmhd3d_b200/data/flux_mlp.npz"})
            out.update(r)
        else:
            out[f"gated_faces_{sur}"] = r
        s.close()
    return out


def run_reference(args):
    """The reference arm: the reference's own hot path (oracle/_ref, compiled
    from its sources) on the host cores, on this arm's workload and mesh.  A
    step is one full global step of one single-rank process on its own
    replica of the mesh; the K timed and W warm-up steps are spread over P
    concurrent processes (ceil(K/P) and ceil(W/P) each)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import fvmhd3d_b200 as F
    steps = max(1, args.steps)
    t0 = time.perf_counter()
    m, _, _, _, shared = make_workload(F, args.problem, args.nside, args.ncell, args.order)
    if not shared:
        print(json.dumps({"impl": "reference", "unavailable": "the CPU sample runs the global-timestep workloads"}))
        return
    mesh_s = time.perf_counter() - t0
    P = os.cpu_count() or 1
    avail = host_memory_available()
    if avail:
        P = max(1, min(P, int(0.6 * avail // (CPU_BYTES_PER_CELL * m.ncell))))
    per = math.ceil(steps / P)
    wper = math.ceil(max(0, args.warmup) / P)
    cb = cpu_leg(m, args.problem, per, wper, procs=P)
    wall = time.perf_counter() - t0
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": ws,
            "steps": steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{args.problem} {args.nside}^3 jittered Voronoi, global timestep, plain FP64",
                       "ncell": m.ncell, "nface_per_step": m.nface, "cell_order": args.order,
                       "mesh_build_s": round(mesh_s, 2),
                       "steps_run": f"{cb['cores']} processes x {per} timed step(s) after {wper} warm-up"},
            "cpu_baseline": {"value": cb["value"], "unit": UNIT, "cores": cb["cores"], "kind": cb["kind"],
                             "sample": cb["sample"]},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": round(wall, 2)}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fvm", choices=["fvm", "reference"])
    ap.add_argument("--nside", type=int, default=128)
    ap.add_argument("--ncell", type=int, default=1048576, help="generators of the disk workload")
    ap.add_argument("--problem", default="blast")
    ap.add_argument("--order", default="hilbert", choices=["hilbert", "native"],
                    help="cell order: Peano-Hilbert (the reference's sort_local_data) or as generated")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--cpu-steps", type=int, default=1, help="timed steps per process of the CPU sample")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-flux + FP32 comparison leg")
    ap.add_argument("--no-remesh", action="store_true", help="skip timing the per-step mesh installation")
    ap.add_argument("--no-configs", action="store_true", help="skip the 64^3, disk and 160^3 configurations")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "fvm":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
