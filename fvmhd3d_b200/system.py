"""Host-side mirror of the reference's ``struct system`` hot-path interface.

The reference drives its fluid update through argument-free member functions
of ``fvmhd3d::system`` (MPI/fvmhd3d.h:298-575):

    fluid_update(true)  = slope_limiter, compute_update, compute_pvel,
                          compute_timesteps(false)      (MPI/iterate.cpp:97-107)
    fluid_update(false) = compute_update0, compute_reconstruction
                                                        (MPI/iterate.cpp:108-112)

:class:`System` keeps those names and that order over the C-ABI of
``libfvmhd3d_b200.so`` (include/fvmhd3d_b200.h); all arrays live on the GPU
inside the context.  Errors raise :class:`FvmError` (the reference aborts on
a failed ``assert``).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from .mesh import Mesh

MLP_NPARAM = 36232
FVM_PREC_FP64 = 0
FVM_PREC_FP32 = 1


class FvmError(RuntimeError):
    pass


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class System:
    """One context on one CUDA device (one rank of the reference)."""

    def __init__(self, gamma=5.0 / 3.0, courant=0.4, box=(1.0, 1.0, 1.0), dtmax=1.0 / 64, eos=0,
                 iso_GM=1.0, iso_cfac=0.05, precision=FVM_PREC_FP64, device=0, static_mesh=False):
        self.L = _lib.lib()
        prm = _lib.FvmParams()
        prm.gamma, prm.courant = gamma, courant
        box = np.broadcast_to(np.asarray(box, dtype=np.float64), (3,))
        for a in range(3):
            prm.box[a] = float(box[a])
        prm.dtmax, prm.eos, prm.iso_GM, prm.iso_cfac, prm.precision = dtmax, eos, iso_GM, iso_cfac, precision
        prm.static_mesh = 1 if static_mesh else 0
        self.params = prm
        h = self.L.fvm_create(ctypes.byref(prm), int(device))
        if not h:
            raise FvmError("fvm_create failed (no CUDA device?)")
        self.h = ctypes.c_void_p(h)
        self.mesh: Mesh | None = None

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.L.fvm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc < 0:
            raise FvmError(f"{what}: rc={rc}: {self.L.fvm_last_error(self.h).decode()}")
        return rc

    # -- inputs -----------------------------------------------------------
    def set_mesh(self, m: Mesh):
        self.mesh = m
        arrs = [np.ascontiguousarray(m.s1, np.int32), np.ascontiguousarray(m.s2, np.int32),
                np.ascontiguousarray(m.n, np.float64), np.ascontiguousarray(m.centroid, np.float64),
                np.ascontiguousarray(m.volume, np.float64), np.ascontiguousarray(m.cell_centroid, np.float64),
                np.ascontiguousarray(m.cell_face_off, np.int64), np.ascontiguousarray(m.cell_face_ids, np.int32)]
        self._check(self.L.fvm_set_mesh(self.h, m.ncell, m.nface, *[_p(a) for a in arrs]), "fvm_set_mesh")

    def set_positions(self, pos, bnd=None) -> None:
        """Generator positions (and boundary codes) of the installed mesh and
        the tables built from them, keeping the fluid state: after
        set_mesh, before set_state / step_host."""
        p = np.ascontiguousarray(pos, np.float64)
        b = None if bnd is None else np.ascontiguousarray(bnd, np.int32)
        self._check(self.L.fvm_set_positions(self.h, _p(p), _p(b)), "fvm_set_positions")

    def init_problem(self, W, bnd=None, rung_offset=0):
        W = np.ascontiguousarray(W, np.float64)
        pos = np.ascontiguousarray(self.mesh.pos, np.float64)
        b = None if bnd is None else np.ascontiguousarray(bnd, np.int32)
        self._check(self.L.fvm_init_problem(self.h, _p(W), _p(pos), _p(b), int(rung_offset)), "fvm_init_problem")

    # -- the reference call sequence --------------------------------------
    def begin_step(self):
        return self._check(self.L.fvm_begin_step(self.h), "fvm_begin_step")

    def slope_limiter(self):
        self._check(self.L.fvm_slope_limiter(self.h), "fvm_slope_limiter")

    def compute_update(self):
        self._check(self.L.fvm_compute_update(self.h), "fvm_compute_update")

    def compute_pvel(self):
        self._check(self.L.fvm_compute_pvel(self.h), "fvm_compute_pvel")

    def compute_timesteps(self, shared=False):
        dt = ctypes.c_double(0.0)
        self._check(self.L.fvm_compute_timesteps(self.h, int(bool(shared)), ctypes.byref(dt)),
                    "fvm_compute_timesteps")
        return dt.value

    def collect_results(self):
        self._check(self.L.fvm_collect_results(self.h), "fvm_collect_results")

    def compute_update0(self):
        self._check(self.L.fvm_compute_update0(self.h), "fvm_compute_update0")

    def compute_reconstruction(self):
        self._check(self.L.fvm_compute_reconstruction(self.h), "fvm_compute_reconstruction")

    def end_step(self, shared=False):
        return self._check(self.L.fvm_end_step(self.h, int(bool(shared))), "fvm_end_step")

    def fluid_update(self, flag: bool, shared=False):
        """system::fluid_update (MPI/iterate.cpp:95-113)."""
        if flag:
            self.slope_limiter()
            self.compute_update()
            self.compute_pvel()
            self.compute_timesteps(shared)
        else:
            self.compute_update0()
            self.compute_reconstruction()

    def iterate_step(self, shared=True):
        """One step of the reference's iterate_step on the fixed mesh; returns
        the number of active cells."""
        return self._check(self.L.fvm_step(self.h, int(bool(shared))), "fvm_step")

    step = iterate_step

    def run(self, nsteps, shared=True):
        """nsteps steps replayed from a captured CUDA graph; returns
        (active cells summed over the steps, active faces summed)."""
        faces = ctypes.c_longlong(0)
        cells = self._check(self.L.fvm_run(self.h, int(nsteps), int(bool(shared)), ctypes.byref(faces)), "fvm_run")
        return cells, faces.value

    # -- outputs ----------------------------------------------------------
    @property
    def time(self) -> float:
        return self.L.fvm_time(self.h)

    @property
    def tsys_ticks(self) -> int:
        return int(self.L.fvm_tsys_ticks(self.h))

    def get_state(self) -> dict:
        n = self.mesh.ncell
        st = dict(pos=np.zeros((n, 3)), vel=np.zeros((n, 3)), tlast=np.zeros(n), tend=np.zeros(n),
                  rung=np.zeros(n, np.int32), U=np.zeros((n, 10)), dU=np.zeros((n, 14)), wrec=np.zeros((n, 50)))
        self._check(self.L.fvm_get_state(self.h, *[_p(st[k]) for k in
                                                   ("pos", "vel", "tlast", "tend", "rung", "U", "dU", "wrec")]),
                    "fvm_get_state")
        return st

    def get_motion(self) -> dict:
        """orig_pos, orig_vel (the reference's correct()) and divBi (float32)."""
        n = self.mesh.ncell
        out = dict(orig_pos=np.zeros((n, 3)), orig_vel=np.zeros((n, 3)), divb=np.zeros(n, np.float32))
        self._check(self.L.fvm_get_motion(self.h, _p(out["orig_pos"]), _p(out["orig_vel"]), _p(out["divb"])),
                    "fvm_get_motion")
        return out

    def adjust_stats(self):
        """(dirty sites, parallel replays, sequential sweep ran) of the last
        individual-timestep step's adjust_timesteps."""
        v = [ctypes.c_int(0) for _ in range(3)]
        self._check(self.L.fvm_last_adjust_stats(self.h, *[ctypes.byref(x) for x in v]), "fvm_last_adjust_stats")
        return tuple(x.value for x in v)

    # -- learned face flux ---------------------------------------------------
    def mlp_set_weights(self, params) -> None:
        """Network parameters (FVM_MLP_NPARAM floats, order of
        fvmhd3d_b200.learned.unpack)."""
        p = np.ascontiguousarray(params, np.float32).ravel()
        if p.size != MLP_NPARAM:
            raise ValueError(f"expected {MLP_NPARAM} parameters, got {p.size}")
        self._check(self.L.fvm_mlp_set_weights(self.h, _p(p)), "fvm_mlp_set_weights")

    def mlp_eval(self, X) -> np.ndarray:
        """Network outputs (n x 8) for inputs X (n x 16) on the tensor cores."""
        X = np.ascontiguousarray(X, np.float32)
        Y = np.zeros((X.shape[0], 8), np.float32)
        self._check(self.L.fvm_mlp_eval(self.h, X.shape[0], _p(X), _p(Y)), "fvm_mlp_eval")
        return Y

    def mlp_eval_counted(self, X, n, Y0=None) -> np.ndarray:
        """The network with its row count n read on the device (the form the
        flux passes launch): rows n.. of the result keep Y0 (zeros)."""
        X = np.ascontiguousarray(X, np.float32)
        Y = np.zeros((X.shape[0], 8), np.float32) if Y0 is None else np.array(Y0, np.float32, copy=True)
        self._check(self.L.fvm_mlp_eval_counted(self.h, X.shape[0], int(n), _p(X), _p(Y)), "fvm_mlp_eval_counted")
        return Y

    def set_flux_surrogate(self, kind) -> None:
        """What stands in for the dissipation on gated faces: "network" (the
        default), "central" (none) or "llf" (local Lax-Friedrichs)."""
        k = {"network": 0, "central": 1, "llf": 2}[kind] if isinstance(kind, str) else int(kind)
        self._check(self.L.fvm_set_flux_surrogate(self.h, k), "fvm_set_flux_surrogate")

    def set_flux_mode(self, mode, drho=0.05, dp=0.05, mach=1.0, jmax=float("inf"), judge=1024, hstride=1,
                      hcap=0) -> None:
        """Learned-flux mode of the flux passes: 0 exact, 1 network on gated
        faces, 2 exact with harvesting (see fvm_set_flux_mode)."""
        self._check(self.L.fvm_set_flux_mode(self.h, int(mode), ctypes.c_float(drho), ctypes.c_float(dp),
                                             ctypes.c_float(mach), ctypes.c_float(jmax), int(judge), int(hstride),
                                             int(hcap)), "fvm_set_flux_mode")

    def mlp_set_norm(self, mu_x, sd_x, mu_y, sd_y) -> None:
        """Standardisation of the network's inputs and outputs."""
        a = [np.ascontiguousarray(v, np.float32).ravel() for v in (mu_x, sd_x, mu_y, sd_y)]
        self._check(self.L.fvm_mlp_set_norm(self.h, *[_p(v) for v in a]), "fvm_mlp_set_norm")

    def learn_stats(self) -> dict:
        s = np.zeros(8)
        self._check(self.L.fvm_learn_stats(self.h, _p(s)), "fvm_learn_stats")
        return {"deferred": int(s[0]), "fallback": int(s[1]), "judged": int(s[2]),
                "judged_rel_l1": float(s[3] / s[4]) if s[4] > 0 else 0.0,
                "judged_mean_abs": float(s[3] / (7 * s[2])) if s[2] > 0 else 0.0, "judged_max_abs": float(s[5]),
                "positivity_fallback": int(s[6])}

    def harvest(self):
        """(X, Y) pairs harvested in mode 2 so far."""
        n = int(self.L.fvm_harvest_count(self.h))
        if n < 0:
            raise FvmError("fvm_harvest_count failed")
        X = np.zeros((n, 16), np.float32)
        Y = np.zeros((n, 8), np.float32)
        self._check(self.L.fvm_get_harvest(self.h, n, _p(X), _p(Y)), "fvm_get_harvest")
        return X, Y

    def mlp_get_weights(self) -> np.ndarray:
        out = np.zeros(MLP_NPARAM, np.float32)
        self._check(self.L.fvm_mlp_get_weights(self.h, _p(out)), "fvm_mlp_get_weights")
        return out

    def mlp_grad(self, X, T, wt=None):
        """(loss, gradient) of the mean-squared loss at the current parameters,
        from the training kernels."""
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        w = None if wt is None else np.ascontiguousarray(wt, np.float32)
        g = np.zeros(MLP_NPARAM, np.float32)
        loss = ctypes.c_float(0.0)
        self._check(self.L.fvm_mlp_grad(self.h, X.shape[0], _p(X), _p(T), _p(w), _p(g), ctypes.byref(loss)),
                    "fvm_mlp_grad")
        return float(loss.value), g

    def mlp_train(self, X, T, wt=None, batch=4096, steps=1000, lr=1e-3, seed=1) -> np.ndarray:
        """Adam training on the GPU from the current parameters; returns the
        minibatch losses."""
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        w = None if wt is None else np.ascontiguousarray(wt, np.float32)
        hist = np.zeros(max(steps, 1), np.float32)
        self._check(self.L.fvm_mlp_train(self.h, X.shape[0], _p(X), _p(T), _p(w), int(batch), int(steps),
                                         ctypes.c_float(lr), ctypes.c_ulonglong(seed), _p(hist)), "fvm_mlp_train")
        return hist[:steps]

    def autotune(self, shared=True, steps=3) -> dict:
        """Pick launch choices by timing trial steps (the state is restored)."""
        ch = np.zeros(4, np.int32)
        self._check(self.L.fvm_autotune(self.h, 1 if shared else 0, int(steps), _p(ch)), "fvm_autotune")
        return {"staged_limiter": int(ch[0]), "face_block": int(ch[1]), "cell_block": int(ch[2]),
                "cell2_block": int(ch[3])}

    def set_fused(self, max_cells) -> None:
        """Replayed individual-timestep steps involving at most max_cells
        cells run as one persistent kernel launch (0: never)."""
        self._check(self.L.fvm_set_fused(self.h, int(max_cells)), "fvm_set_fused")

    @property
    def fused_steps(self) -> int:
        """Steps the persistent rung kernel has run (as of the last run/step)."""
        return int(self.L.fvm_fused_step_count(self.h))

    def set_reduce(self, fn) -> None:
        """The reduction of the timestep minimum over ranks (MPI_Allreduce MIN
        of compute_timesteps, MPI/compute_timestep.cpp:101): fn(dt_min) ->
        the minimum over ranks, called on this thread inside steps and
        fvm_init_problem.  None removes it.  Steps with a reduction are eager
        (run() refuses)."""
        if fn is None:
            self._reduce_cb = None
            self._check(self.L.fvm_set_reduce(self.h, ctypes.cast(None, _lib.REDUCE_FN), None), "fvm_set_reduce")
            return

        def cb(_user, p):
            try:
                p[0] = float(fn(float(p[0])))
                return 0
            except Exception:  # reported by the library as a failed step
                return 1

        self._reduce_cb = _lib.REDUCE_FN(cb)  # kept alive while installed
        self._check(self.L.fvm_set_reduce(self.h, self._reduce_cb, None), "fvm_set_reduce")

    def set_halo(self, halo) -> None:
        """Marks the installed mesh's copies of other ranks' cells (a bool
        per cell; None: none); their timesteps stay out of the minimum."""
        h = None if halo is None else np.ascontiguousarray(np.asarray(halo) != 0, np.uint8)
        if h is not None and h.shape != (self.mesh.ncell,):
            raise ValueError("set_halo: one flag per cell")
        self._check(self.L.fvm_set_halo(self.h, _p(h)), "fvm_set_halo")

    def set_list_building(self, max_entries) -> None:
        """Partial steps whose active cells plus their links number at most
        max_entries build their lists from those cells' links instead of a
        pass over every face (-1: 1/256 of the mesh's cells plus links, at
        least 8192, the default; 0: never)."""
        self._check(self.L.fvm_set_list_building(self.h, int(max_entries)), "fvm_set_list_building")

    @property
    def incremental_steps(self) -> int:
        """Steps whose lists were built incrementally (as of the last run/step)."""
        return int(self.L.fvm_incremental_step_count(self.h))

    def set_tuning(self, staged_limiter, face_block, cell_block, cell2_block) -> None:
        """Set the launch choices the autotuner picks (see autotune)."""
        ch = np.array([staged_limiter, face_block, cell_block, cell2_block], np.int32)
        self._check(self.L.fvm_set_tuning(self.h, _p(ch)), "fvm_set_tuning")

    def clock(self):
        """(tsysU, dt_global, iteration): the scheduler clock after the last
        step (the reference's Scheduler::tsysU, system::dt_global and
        system::iteration)."""
        t = ctypes.c_ulonglong(0)
        dt = ctypes.c_double(0.0)
        it = ctypes.c_longlong(0)
        self._check(self.L.fvm_clock(self.h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(it)), "fvm_clock")
        return t.value, dt.value, it.value

    def dump_binary(self, path, idx=None, rmax=None) -> None:
        """Writes the current state as the reference's snapshot file
        (system::dump_binary, MPI/dump_binary.cpp); read it back with
        :func:`fvmhd3d_b200.snapshot.read_binary`.  idx (int32 particle ids)
        and rmax (float32 mesh search radii) default to the cell index and 0."""
        n = self.mesh.ncell
        i = None if idx is None else np.ascontiguousarray(idx, np.int32)
        r = None if rmax is None else np.ascontiguousarray(rmax, np.float32)
        for a in (i, r):
            if a is not None and a.shape != (n,):
                raise ValueError(f"expected {n} entries, got {a.shape}")
        self._check(self.L.fvm_dump_binary(self.h, os.fsencode(path), _p(i), _p(r)), "fvm_dump_binary")

    def set_state(self, vel=None, tlast=None, tend=None, rung=None, U=None, dU=None, wrec=None, tsys_ticks=0):
        conv = [None if a is None else np.ascontiguousarray(a, t) for a, t in
                ((vel, np.float64), (tlast, np.float64), (tend, np.float64), (rung, np.int32),
                 (U, np.float64), (dU, np.float64), (wrec, np.float64))]
        self._check(self.L.fvm_set_state(self.h, *[_p(a) for a in conv], ctypes.c_ulonglong(tsys_ticks)),
                    "fvm_set_state")

    STATE_ARRAYS = (("vel", np.float64, 3), ("tlast", np.float64, 1), ("tend", np.float64, 1),
                    ("rung", np.int32, 1), ("U", np.float64, 10), ("dU", np.float64, 14),
                    ("wrec", np.float64, 50))

    def step_host(self, state, shared=True, tsys_ticks=None) -> int:
        """One step on host-owned state (fvm_step_host): `state` maps vel,
        tlast, tend, rung, U, dU and wrec to C-contiguous arrays of the
        right type (pinned for the copies to overlap), read and then
        overwritten with the stepped state.  tsys_ticks defaults to the
        context's clock.  Returns the active cell count."""
        n = self.mesh.ncell
        for k, t, w in self.STATE_ARRAYS:
            a = state[k]
            if a.dtype != t or not a.flags["C_CONTIGUOUS"] or a.size != n * w:
                raise ValueError(f"step_host: {k} must be a C-contiguous {np.dtype(t).name} array of {n * w}")
        ticks = self.tsys_ticks if tsys_ticks is None else int(tsys_ticks)
        r = self.L.fvm_step_host(self.h, 1 if shared else 0, ctypes.c_ulonglong(ticks),
                                 *[_p(state[k]) for k, _, _ in self.STATE_ARRAYS])
        self._check(r, "fvm_step_host")
        return r

    def active_faces(self) -> np.ndarray:
        n = ctypes.c_int(0)
        self._check(self.L.fvm_get_active_faces(self.h, None, ctypes.byref(n)), "fvm_get_active_faces")
        ids = np.zeros(max(n.value, 1), np.int32)
        self._check(self.L.fvm_get_active_faces(self.h, _p(ids), ctypes.byref(n)), "fvm_get_active_faces")
        return ids[: n.value]

    def limited_wrec(self) -> np.ndarray:
        out = np.zeros((self.mesh.ncell, 50))
        self._check(self.L.fvm_get_limited_wrec(self.h, _p(out)), "fvm_get_limited_wrec")
        return out

    def dt_list(self) -> np.ndarray:
        out = np.zeros(self.mesh.ncell)
        self._check(self.L.fvm_get_dt_list(self.h, _p(out)), "fvm_get_dt_list")
        return out

    def step_dU(self) -> np.ndarray:
        out = np.zeros((self.mesh.ncell, 14))
        self._check(self.L.fvm_get_step_dU(self.h, _p(out)), "fvm_get_step_dU")
        return out

    def counters(self) -> np.ndarray:
        out = np.zeros(2, np.int64)
        self._check(self.L.fvm_get_counters(self.h, _p(out)), "fvm_get_counters")
        return out

    def compute_flux(self, wij, Wi, Wj, jbnd, normal):
        nf = Wi.shape[0]
        wij, Wi, Wj, normal = (np.ascontiguousarray(a, np.float64) for a in (wij, Wi, Wj, normal))
        jb = np.ascontiguousarray(jbnd, np.int32)
        psi, Bn, flux = np.zeros(nf), np.zeros(nf), np.zeros((nf, 10))
        self._check(self.L.fvm_compute_flux(self.h, nf, _p(wij), _p(Wi), _p(Wj), _p(jb), _p(normal),
                                            _p(psi), _p(Bn), _p(flux)), "fvm_compute_flux")
        return psi, Bn, flux

    def last_step_ms(self) -> float:
        return float(self.L.fvm_last_step_ms(self.h))

    @property
    def stream_ptr(self) -> int:
        """The context's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        return int(self.L.fvm_stream(self.h) or 0)

    def active_face_count(self) -> int:
        """Active faces of the last completed step (face-updates of that step)."""
        nf = ctypes.c_int(0)
        self._check(self.L.fvm_last_step_counts(self.h, None, ctypes.byref(nf)), "fvm_last_step_counts")
        return nf.value

    @property
    def launch_count(self) -> int:
        return int(self.L.fvm_launch_count(self.h))

    def fp64_peak(self) -> float:
        """Measured FP64 FMA throughput of the device, FLOP/s."""
        v = ctypes.c_double(0.0)
        self._check(self.L.fvm_fp64_peak(self.h, ctypes.byref(v)), "fvm_fp64_peak")
        return float(v.value)

    def set_profiling(self, on=True):
        self._check(self.L.fvm_set_profiling(self.h, int(bool(on))), "fvm_set_profiling")

    def kernel_times(self) -> dict:
        """{kernel class: (total ms, timed launches)} since set_profiling."""
        out = {}
        k = 0
        name = ctypes.c_char_p()
        ms = ctypes.c_double()
        calls = ctypes.c_longlong()
        while self.L.fvm_kernel_times(self.h, k, ctypes.byref(name), ctypes.byref(ms), ctypes.byref(calls)) == 1:
            out[name.value.decode()] = (ms.value, calls.value)
            k += 1
        return out
