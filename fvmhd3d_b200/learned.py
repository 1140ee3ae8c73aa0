"""Learned face flux: harvesting, training and evaluation on the GPU.

The network (16 -> 128 -> 128 -> 128 -> 8, GELU; FP16 operands for
inference, BF16 for training, FP32 accumulation) predicts, on smooth faces, the dissipative part of the HLLD
flux in the face frame (the HLLD flux minus the mean of the two sides'
physical fluxes) divided by the size m of the face's scaled jump; the flux
pass multiplies the output by m in FP32, so the network's error is relative
to the dissipation on every face.  csrc/flux_learn.cuh describes the
features, the gate and the exact fallback.  Harvested rows hold the features
(x[14] = m) and the scaled dissipation y itself; the training target is y / m.
This module runs the pipeline with the library's own kernels:

1. ``harvest``: exact runs of the Alfven-wave (32^3, 10 global steps) and
   blast-wave (64^3, 50 global steps) workloads in harvesting mode collect
   (features, targets) of gated faces, about 20M pairs;
2. ``train``: Adam on the GPU (``System.mlp_train``, BF16 tensor-core
   forward/backward kernels) from a seeded initialisation;
3. ``evaluate``: the 128^3 blast for 100 steps with the learned flux and the
   FP32 bulk path against the plain FP64 path: per-variable relative L1
   error, fallback fraction, judged network error, and throughput.

    python -m fvmhd3d_b200.learned --out weights.npz      # harvest + train
    python -m fvmhd3d_b200.learned --profile-rows 524288  # network alone (for ncu)
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import mesh as _mesh
from . import problems
from .ordering import sort_local_data
from .system import FVM_PREC_FP32, FVM_PREC_FP64, MLP_NPARAM, System

# gate: relative density and pressure jumps, normal Mach number in the face
# frame, and the size of the scaled jump: the network serves faces whose
# dissipation is close to linear in the jump
GATE = dict(drho=0.05, dp=0.05, mach=1.0, jmax=0.01)
# loss weight per output (MASS, MOMX..Z, ENER, WBX..Z); the normal induction
# flux is exact (-w Bn) and not learned
OUTPUT_WEIGHTS = np.array([1, 1, 1, 1, 1, 0, 1, 1], np.float32)
HIDDEN, NIN, NOUT = 128, 16, 8


def init_params(seed=0) -> np.ndarray:
    """Seeded He-uniform weights, zero biases, in the parameter order of
    fvm_mlp_set_weights."""
    rng = np.random.default_rng(seed)
    parts = []
    for rows, cols in ((HIDDEN, NIN), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (NOUT, HIDDEN)):
        lim = np.sqrt(6.0 / cols)
        parts.append(rng.uniform(-lim, lim, rows * cols))
        parts.append(np.zeros(rows))
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == MLP_NPARAM
    return p


def _lattice_mesh(nside, seed, order):
    """Jittered-lattice periodic mesh with its cells in lattice order or in
    Peano-Hilbert order (sort_local_data)."""
    pos = _mesh.jittered_lattice(nside, 0.1, seed=seed)
    if order == "hilbert":
        pos = pos[sort_local_data(pos, 1.0)]
    return _mesh.build_periodic(pos, 1.0)


def harvest_run(problem, nside, steps, hstride, hcap, seed=1, order="native"):
    """(X, Y) harvested from an exact run (global timestep, FP32 bulk)."""
    m = _lattice_mesh(nside, seed, order)
    W = getattr(problems, problem)(m.pos)
    s = System(precision=FVM_PREC_FP32)
    s.set_mesh(m)
    s.init_problem(W)
    s.set_flux_mode(2, hstride=hstride, hcap=hcap, **GATE)
    for _ in range(steps):
        s.step(shared=True)
    X, Y = s.harvest()
    s.close()
    return X, Y


def harvest(scale=1.0):
    """About 20M pairs from the Alfven (32^3, 10 steps) and blast (64^3, 50
    steps) workloads, each run once with its cells in lattice order and once
    in Peano-Hilbert order: a face's orientation (which cell is s1) follows
    the cell numbering, so the two orders give the network both orientations
    of the same faces.  Only faces the gate passes are harvested.  `scale`
    shrinks the run sizes for tests."""
    if scale >= 1.0:
        runs = [("alfven", 32, 10, 2, 3_000_000), ("blast", 64, 50, 24, 8_000_000)]
    else:
        runs = [("alfven", 16, 4, 2, 200_000), ("blast", 24, 10, 4, 500_000)]
    Xs, Ys = [], []
    for (problem, nside, steps, stride, cap), order in ((r, o) for r in runs for o in ("native", "hilbert")):
        X, Y = harvest_run(problem, nside, steps, stride, cap, order=order)
        Xs.append(X)
        Ys.append(Y)
    return np.concatenate(Xs), np.concatenate(Ys)


M_COL = 14  # feature column holding the jump size m


def targets(X, Y):
    """Training targets: the scaled dissipation divided by the jump size m
    (rows with m = 0 have zero dissipation and are dropped by the caller)."""
    m = np.asarray(X[:, M_COL], np.float64)[:, None]
    return (np.asarray(Y, np.float64) / np.where(m > 0, m, 1.0)).astype(np.float32)


def usable(X):
    """Rows that carry a jump (m > 0)."""
    return X[:, M_COL] > 0


def standardisation(X, T):
    """Per-feature and per-target mean and spread of a harvested set (the
    unlearned normal induction output keeps spread 1)."""
    mu_x = X.mean(axis=0, dtype=np.float64)
    sd_x = X.std(axis=0, dtype=np.float64)
    sd_x = np.maximum(sd_x, 1e-3)  # features nearly constant in training keep a usable spread
    mu_y = T.mean(axis=0, dtype=np.float64)
    sd_y = T.std(axis=0, dtype=np.float64)
    sd_y = np.where((sd_y > 1e-12) & (OUTPUT_WEIGHTS > 0), sd_y, 1.0)
    mu_y = np.where(OUTPUT_WEIGHTS > 0, mu_y, 0.0)
    return {k: v.astype(np.float32) for k, v in (("mu_x", mu_x), ("sd_x", sd_x), ("mu_y", mu_y), ("sd_y", sd_y))}


# Version tag of the network's input and output definition, stored with the
# weights; weights of another form would be fed the wrong features.
FORM = "jump-scaled dissipation, features v2"
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "flux_mlp.npz")


def load_model(path=DEFAULT_WEIGHTS):
    """Parameters and standardisation of a trained network (.npz written by
    main); raises if the file holds another form of the network."""
    z = np.load(path)
    form = str(z["form"]) if "form" in z else "(none)"
    if form != FORM:
        raise ValueError(f"{path}: network form {form!r}, expected {FORM!r}")
    return {k: z[k] for k in ("params", "mu_x", "sd_x", "mu_y", "sd_y")}


def apply(sys, model):
    """Load a trained model (parameters and standardisation) into a System."""
    sys.mlp_set_weights(model["params"])
    sys.mlp_set_norm(model["mu_x"], model["sd_x"], model["mu_y"], model["sd_y"])


def predict(sys, model, X):
    """Scaled dissipation the loaded model predicts for raw features X
    (m times the unstandardised network output, as the flux pass forms it)."""
    Xn = (X - model["mu_x"]) / model["sd_x"]
    return X[:, [M_COL]] * (model["mu_y"] + model["sd_y"] * sys.mlp_eval(Xn))


def train(X, Y, steps=12000, batch=8192, seed=0, lr_schedule=(2e-3, 1e-3, 3e-4, 1e-4), sys=None):
    """Train from init_params(seed) on the GPU on the standardised set of
    targets y / m; returns (model dict, loss history)."""
    s = sys or System()
    keep = usable(X)
    X, T = X[keep], targets(X[keep], Y[keep])
    model = standardisation(X, T)
    Xn = ((X - model["mu_x"]) / model["sd_x"]).astype(np.float32)
    Yn = ((T - model["mu_y"]) / model["sd_y"]).astype(np.float32)
    s.mlp_set_weights(init_params(seed))
    hist = []
    per = max(1, steps // len(lr_schedule))
    for k, lr in enumerate(lr_schedule):
        hist.append(s.mlp_train(Xn, Yn, OUTPUT_WEIGHTS, batch=batch, steps=per, lr=lr, seed=seed * 1000 + k + 1))
    model["params"] = s.mlp_get_weights()
    return model, np.concatenate(hist)


def llf_dissipation(X):
    """Scaled face-frame dissipation of the local Lax-Friedrichs (Rusanov)
    flux, -(max wave speed)/2 times the jump of the conserved state, in the
    network's output units, from the features to first order in the jump
    (the flux pass evaluates it exactly from the side states): the method
    without the network."""
    x = np.asarray(X, np.float64)
    u, v, w, p, bx, by, bz = (x[:, k] for k in range(7))
    jump = x[:, 7:14] * x[:, [M_COL]]
    dr, du, dv, dw, dpr, dby, dbz = (jump[:, k] for k in range(7))
    smax = np.abs(u) + np.abs(du) / 2 + 1.0  # |u| + c (c = 1 in these units)
    # conserved jumps with rho = 1 + dr/2 on the right, 1 - dr/2 on the left
    dmom = [u * dr + du, v * dr + dv, w * dr + dw]
    kin = 0.5 * (u * u + v * v + w * w)
    # energy density e + rho v^2/2 + B^2/2 with e = p / (gamma - 1), gamma = 5/3
    dE = 1.5 * dpr + kin * dr + (u * du + v * dv + w * dw) + (by * dby + bz * dbz)
    D = np.zeros((x.shape[0], 8))
    D[:, 0] = -0.5 * smax * dr
    for k in range(3):
        D[:, 1 + k] = -0.5 * smax * dmom[k]
    D[:, 4] = -0.5 * smax * dE
    D[:, 6] = -0.5 * smax * dby
    D[:, 7] = -0.5 * smax * dbz
    return D


def holdout(model, problem="blast", nside=128, steps=20, hstride=64, order="hilbert"):
    """The network on faces harvested from a run it was not trained on:
    mean and largest absolute error per output (scaled units), the targets'
    mean magnitude, the LLF dissipation's error, and the largest standardised
    input seen."""
    X, Y = harvest_run(problem, nside, steps, hstride, 4_000_000, order=order)
    s = System()
    apply(s, model)
    P = predict(s, model, X)
    w = OUTPUT_WEIGHTS.astype(bool)
    z = np.abs((X - model["mu_x"]) / model["sd_x"])
    inside = (z <= 8.0).all(axis=1)  # the faces the device gate would hand to the network
    err = np.abs(P - Y)[inside][:, w]
    return {"pairs": int(X.shape[0]), "in_distribution": float(inside.mean()),
            "mean_abs_err": float(err.mean()), "max_abs_err": float(err.max()),
            "mean_abs_target": float(np.abs(Y[inside][:, w]).mean()),
            "mean_abs_err_llf": float(np.abs(llf_dissipation(X[inside]) - Y[inside])[:, w].mean()),
            "max_std_input": float(z.max()), "max_std_input_feature": int(z.max(axis=0).argmax())}


def evaluate(model, nside=128, steps=100, judge=1024, order="hilbert"):
    """The blast with the learned flux + FP32 bulk path against the plain
    FP64 path after `steps` global steps: relative L1 error per conserved
    variable, fallback and judged statistics, and face-updates/s.  The same
    run is repeated with the gated faces taking the central flux alone (no
    dissipation) and the local Lax-Friedrichs dissipation in place of the
    network, and with the exact solver everywhere (FP32 bulk)."""
    import torch
    m = _lattice_mesh(nside, 1, order)
    W = problems.blast(m.pos)
    out = {"cell_order": order}
    states = {}
    runs = (("plain_fp64", FVM_PREC_FP64, 0, None), ("fp32", FVM_PREC_FP32, 0, None),
            ("learned_fp32", FVM_PREC_FP32, 1, "network"), ("central_fp32", FVM_PREC_FP32, 1, "central"),
            ("llf_fp32", FVM_PREC_FP32, 1, "llf"))
    for name, prec, mode, sur in runs:
        s = System(precision=prec)
        s.set_mesh(m)
        s.init_problem(W)
        if mode == 1:
            apply(s, model)
            s.set_flux_mode(1, judge=judge, **GATE)
            s.set_flux_surrogate(sur)
        stream = torch.cuda.ExternalStream(s.stream_ptr)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        cells, faces = s.run(steps, shared=True)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        states[name] = s.get_state()["U"]
        out[name] = {"face_updates_per_s": faces / (ms / 1e3), "ms_per_step": ms / steps}
        if mode == 1:
            st = s.learn_stats()
            st["deferred_fraction"] = st["deferred"] / max(2 * faces, 1)
            st["fallback_fraction"] = st["fallback"] / max(st["deferred"], 1)
            out[name]["learned"] = st
        s.close()
    ref = states["plain_fp64"]
    for name, *_ in runs[1:]:
        d = np.abs(states[name] - ref).sum(axis=0) / np.maximum(np.abs(ref).sum(axis=0), 1e-300)
        out[name]["rel_l1_vs_fp64"] = {k: float(d[i]) for i, k in
                                       enumerate(["mass", "momx", "momy", "momz", "energy", "bx", "by", "bz",
                                                  "psi", "entropy"])}
    out["speedup_learned_vs_plain_fp64"] = (out["learned_fp32"]["face_updates_per_s"] /
                                            out["plain_fp64"]["face_updates_per_s"])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None, help="write the trained parameters here (.npz)")
    ap.add_argument("--steps", type=int, default=12000)
    ap.add_argument("--evaluate", action="store_true")
    ap.add_argument("--weights", default=None, help="evaluate these parameters instead of training")
    ap.add_argument("--profile-rows", type=int, default=0, help="only run the network on N random rows")
    ap.add_argument("--profile-train-steps", type=int, default=0,
                    help="only run N training steps (batch 8192) on random pairs (for ncu)")
    ap.add_argument("--eval-nside", type=int, default=128, help="blast lattice size of --evaluate")
    ap.add_argument("--eval-steps", type=int, default=100, help="global steps of --evaluate")
    ap.add_argument("--eval-order", default="hilbert", choices=["hilbert", "native"],
                    help="cell order of the --evaluate mesh")
    args = ap.parse_args()
    if args.profile_train_steps:
        s = System()
        s.mlp_set_weights(init_params(1))
        rng = np.random.default_rng(0)
        X = rng.normal(size=(200000, NIN)).astype(np.float32)
        T = rng.normal(size=(200000, NOUT)).astype(np.float32)
        t = time.perf_counter()
        hist = s.mlp_train(X, T, batch=8192, steps=args.profile_train_steps, lr=1e-3, seed=1)
        print(json.dumps({"train_steps": args.profile_train_steps, "wall_s": time.perf_counter() - t,
                          "last_loss": float(hist[-1])}))
        return
    if args.profile_rows:
        s = System()
        s.mlp_set_weights(init_params(1))
        X = np.random.default_rng(0).normal(size=(args.profile_rows, NIN)).astype(np.float32)
        for _ in range(3):
            t = time.perf_counter()
            Y = s.mlp_eval(X)
            dt = time.perf_counter() - t
        print(json.dumps({"rows": args.profile_rows, "wall_ms_with_copies": dt * 1e3,
                          "finite": bool(np.isfinite(Y).all())}))
        return
    if args.weights:
        model = load_model(args.weights)
    else:
        t0 = time.perf_counter()
        X, Y = harvest()
        t1 = time.perf_counter()
        model, hist = train(X, Y, steps=args.steps)
        t2 = time.perf_counter()
        rng = np.random.default_rng(9)
        idx = rng.choice(X.shape[0], min(200000, X.shape[0]), replace=False)
        s = System()
        apply(s, model)
        pred = predict(s, model, X[idx])
        w = OUTPUT_WEIGHTS.astype(bool)
        e_mlp = np.abs(pred - Y[idx])[:, w]
        e_llf = np.abs(llf_dissipation(X[idx]) - Y[idx])[:, w]
        ref = np.abs(Y[idx])[:, w]
        print(json.dumps({"pairs": int(X.shape[0]), "harvest_s": t1 - t0, "train_s": t2 - t1,
                          "final_loss": float(hist[-200:].mean()), "mean_abs_err_network": float(e_mlp.mean()),
                          "mean_abs_err_llf": float(e_llf.mean()), "mean_abs_target": float(ref.mean()),
                          "rel_l1_network": float(e_mlp.sum() / ref.sum()),
                          "rel_l1_llf": float(e_llf.sum() / ref.sum())}))
        if args.out:
            np.savez_compressed(args.out, loss=hist, gate=json.dumps(GATE), form=FORM, **model)
    if args.evaluate:
        print(json.dumps({"holdout_blast128": holdout(model, order=args.eval_order)}))
        print(json.dumps(evaluate(model, nside=args.eval_nside, steps=args.eval_steps, order=args.eval_order)))


if __name__ == "__main__":
    main()
