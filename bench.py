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
    """One single-rank reference (or oracle port) process on its own replica."""
    nside, problem, steps, warmup, kind, seed = args
    sys.path.insert(0, ROOT)
    import fvmhd3d_b200 as F
    from oracle import pyoracle
    pos = F.jittered_lattice(nside, 0.1, seed=seed)
    m = F.build_periodic(pos[F.sort_local_data(pos, 1.0)], 1.0, nthreads=1)
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


def cpu_leg(nside, problem, steps, warmup, procs=None):
    """Aggregate face-updates/s of P concurrent single-rank CPU processes (one
    per host core), each on its own replica mesh.  Uses the reference's own
    code (oracle/_ref/libfvmref.so) when it was built, else the C oracle."""
    import multiprocessing as mp
    from oracle import pyoracle
    kind = "reference" if os.path.exists(pyoracle.REF_SO) else "port"
    if not os.path.exists(pyoracle.REF_SO if kind == "reference" else pyoracle.ORACLE_SO):
        raise RuntimeError("CPU checkers are not built (run __graft_entry__.build())")
    P = procs or os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    with ctx.Pool(P) as pool:
        res = pool.map(_cpu_worker, [(nside, problem, steps, warmup, kind, 100 + r) for r in range(P)])
    faces = sum(r[0] for r in res)
    t = max(r[1] for r in res)
    return {"value": faces / t, "unit": UNIT, "cores": P, "kind": kind,
            "sample": f"{P} concurrent single-rank processes, each {steps} global steps of the {problem} "
                      f"on its own {nside}^3 jittered-lattice replica in Peano-Hilbert order ({faces // (P * steps)} faces); "
                      f"no halo exchange"}


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


def run_gpu(args):
    import torch
    import fvmhd3d_b200 as F

    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    t0 = time.perf_counter()
    prec = F.FVM_PREC_FP32 if args.precision == "fp32" else F.FVM_PREC_FP64
    bnd = None
    if args.problem == "disk":
        # Keplerian disk, isothermal EOS, individual power-of-two timesteps, on
        # static generators (the mesh is built once; generators that followed
        # the flow would need the mesh rebuilt every step)
        pos, box = F.problems.disk_generators(args.ncell, seed=3 + rank)
        if args.order == "hilbert":  # the reference's sort_local_data
            pos = pos[F.sort_local_data(pos, box)]
        m = F.build_periodic(pos, box)
        W, bnd = F.problems.disk(pos, box)
        sysargs = dict(gamma=1.0, courant=0.4, box=tuple(box), dtmax=1.0 / 16, eos=1, iso_GM=1.0, iso_cfac=0.05,
                       static_mesh=True)
        shared = False
    else:
        pos = F.jittered_lattice(args.nside, 0.1, seed=1 + rank)
        if args.order == "hilbert":
            pos = pos[F.sort_local_data(pos, 1.0)]
        m = F.build_periodic(pos, 1.0)
        W = getattr(F.problems, args.problem)(m.pos)
        sysargs = {}
        shared = True
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
            S.set_state(tsys_ticks=ticks, **host)
            nact = S.step(shared=shared)
            ticks = S.tsys_ticks
            e_faces += S.active_face_count()
            S.L.fvm_get_state(S.h, None, *[F.system._p(host[k]) for k in ("vel", "tlast", "tend", "rung", "U",
                                                                              "dU", "wrec")])
        e1.record(stream)
        torch.cuda.synchronize()
        e_ms = allreduce_max(e0.elapsed_time(e1), ws)
        e2e = {"value": e_faces * ws / (e_ms / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(bytes_in), "d2h_bytes_per_step": int(bytes_in),
               "steps": e_steps, "path": "fvm_set_state -> fvm_step -> fvm_get_state, pinned host buffers"}

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
        line["learned_fp32"] = learned_leg(F, m, W, S, 100, weights, stream_of=torch.cuda.ExternalStream)
    if rank == 0 and ws == 1 and not args.no_cpu:
        try:
            line["cpu_baseline"] = cpu_leg(args.cpu_nside, args.problem, args.cpu_steps, 1)
        except Exception as e:  # the GPU number stands without it
            line["cpu_baseline"] = {"error": str(e)}
    if rank == 0:
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def learned_leg(F, m, W, plain, steps, weights, stream_of):
    """The learned-flux + FP32 bulk path on the same mesh and initial state
    for `steps` global steps: face-updates/s (CUDA events) and its relative
    L1 error per conserved variable against the plain FP64 context `plain`
    advanced by the same number of steps from the same start."""
    import torch
    from fvmhd3d_b200 import learned as L
    z = np.load(weights)
    model = {k: z[k] for k in ("params", "mu_x", "sd_x", "mu_y", "sd_y")}
    ref = F.System(precision=F.FVM_PREC_FP64)
    ref.set_mesh(m)
    ref.init_problem(W)
    ref.run(steps, shared=True)
    s = F.System(precision=F.FVM_PREC_FP32)
    s.set_mesh(m)
    s.init_problem(W)
    L.apply(s, model)
    s.set_flux_mode(1, **L.GATE)
    st = stream_of(s.stream_ptr)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    _, faces = s.run(steps, shared=True)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    Ua, Ub = ref.get_state()["U"], s.get_state()["U"]
    rel = np.abs(Ub - Ua).sum(axis=0) / np.maximum(np.abs(Ua).sum(axis=0), 1e-300)
    stats = s.learn_stats()
    out = {"value": faces / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps, "steps": steps,
           "rel_l1_vs_plain_fp64": {"density": float(rel[0]), "energy": float(rel[4]),
                                    "momentum": float(rel[1:4].max()), "magnetic": float(rel[5:8].max())},
           "network_faces_fraction": stats["deferred"] / max(2 * faces, 1),
           "fallback_fraction": stats["fallback"] / max(stats["deferred"], 1),
           "judged_mean_abs_scaled": stats["judged_mean_abs"], "judged_max_abs_scaled": stats["judged_max_abs"],
           "judged_rel_l1": stats["judged_rel_l1"],
           "dtype": "f32 bulk + bf16 network", "weights": "fvmhd3d_b200/data/flux_mlp.npz"}
    ref.close()
    s.close()
    return out


def run_reference(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    steps = max(1, args.steps)
    t0 = time.perf_counter()
    cb = cpu_leg(args.cpu_nside, args.problem, steps, max(1, min(args.warmup, 2)))
    wall = time.perf_counter() - t0
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": ws,
            "steps": steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{args.problem} {args.nside}^3 jittered Voronoi, global timestep, plain FP64 "
                                   f"(bounded CPU sample: {args.cpu_nside}^3 replicas)"},
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
    ap.add_argument("--cpu-nside", type=int, default=32)
    ap.add_argument("--cpu-steps", type=int, default=4)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-flux + FP32 comparison leg")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "fvm":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
