"""ctypes front-ends for the two CPU checkers.  TEST INFRASTRUCTURE ONLY.

* :class:`RefSystem` drives ``_ref/libfvmref.so``: the reference's own MPI-tree
  hot path compiled from its sources with a one-rank harness
  (``ref_harness/ref_driver.cpp``).
* :class:`OracleSystem` drives ``_ref/liboracle.so``: the plain-C restatement
  in ``fvm_oracle.c``.

Both expose the same methods so tests can run them side by side and against
the CUDA path.  Only ``tests/``, ``__graft_entry__.smoke`` and the CPU
baseline leg of ``bench.py`` may use this module.
"""
from __future__ import annotations

import ctypes
import math
import os
import struct
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libfvmref.so")
ORACLE_SO = os.path.join(HERE, "_ref", "liboracle.so")


# The reference's MPI-tree sources, read where they lie (the Makefile's
# REF_DIR default); FVM_REF_DIR points the build elsewhere.
REF_DIR = os.environ.get("FVM_REF_DIR", "/root/reference/MPI")


def build(ref: bool = True) -> None:
    """Compile the checkers with oracle/Makefile (the reference build only when
    its sources are present)."""
    targets = ["oracle"]
    if ref and os.path.isdir(REF_DIR):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, f"REF_DIR={REF_DIR}"] + targets, check=True)


class _Params(ctypes.Structure):
    _fields_ = [
        ("gamma", ctypes.c_double),
        ("courant", ctypes.c_double),
        ("box", ctypes.c_double * 3),
        ("dtmax", ctypes.c_double),
        ("eos", ctypes.c_int),
        ("iso_GM", ctypes.c_double),
        ("iso_cfac", ctypes.c_double),
        ("static_mesh", ctypes.c_int),
    ]


SNAP_FIELDS = [
    ("wrec_after_limiter", np.float64, 50),
    ("U_after_update", np.float64, 10),
    ("dU_after_update", np.float64, 14),
    ("vel_after_pvel", np.float64, 3),
    ("rung_after_timestep", np.int32, 1),
    ("dt_after_timestep", np.float64, 1),
    ("wrec_after_update0", np.float64, 50),
    ("rung_after_update0", np.int32, 1),
    ("wrec_after_recon", np.float64, 50),
    ("active_faces", np.int32, 0),
    ("nactive_faces", np.int32, -1),
]


class _Snap(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name, _, _ in SNAP_FIELDS]


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _to_primitive(U, V):
    """FluidBase::to_primitive (MPI/Fluid.h:55-92) in double precision, the
    reference's operation order."""
    U = [float(u) for u in U]
    iM = 1.0 / U[0]
    iV = 1.0 / V
    W = [0.0] * 10
    W[0] = U[0] * iV
    W[1], W[2], W[3] = U[1] * iM, U[2] * iM, U[3] * iM
    W[5], W[6], W[7] = U[5] * iV, U[6] * iV, U[7] * iV
    W[8] = U[8] * iM
    W[9] = U[9] * iM
    W[4] = (U[4] * iV - 0.5 * (W[5] * W[5] + W[6] * W[6] + W[7] * W[7])
            - 0.5 * (W[1] * W[1] + W[2] * W[2] + W[3] * W[3]) * W[0])
    return W


def make_params(gamma=5.0 / 3.0, courant=0.4, box=(1.0, 1.0, 1.0), dtmax=1.0 / 64, eos=0,
                iso_GM=1.0, iso_cfac=0.05, static_mesh=False) -> _Params:
    p = _Params()
    p.gamma, p.courant = gamma, courant
    for a in range(3):
        p.box[a] = box[a]
    p.dtmax, p.eos, p.iso_GM, p.iso_cfac = dtmax, eos, iso_GM, iso_cfac
    p.static_mesh = 1 if static_mesh else 0
    return p


class _Base:
    prefix = ""
    so = ""
    off_dtype = np.int64

    def __init__(self, **params):
        if not os.path.exists(self.so):
            raise RuntimeError(f"{self.so} missing: build the checkers first")
        self.lib = ctypes.CDLL(self.so)
        f = self._fn
        f("create").restype = ctypes.c_void_p
        f("create").argtypes = [ctypes.POINTER(_Params)]
        f("time").restype = ctypes.c_double
        f("time").argtypes = [ctypes.c_void_p]
        for name in ("set_mesh", "init_problem", "step", "get_state", "compute_flux"):
            f(name).restype = ctypes.c_int
        self.params = make_params(**params)
        self.h = ctypes.c_void_p(f("create")(ctypes.byref(self.params)))
        self.mesh = None

    def _fn(self, name):
        return getattr(self.lib, self.prefix + name)

    def close(self):
        if self.h:
            self._fn("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_mesh(self, m):
        self.mesh = m
        self._keep = [np.ascontiguousarray(m.s1, np.int32), np.ascontiguousarray(m.s2, np.int32),
                      np.ascontiguousarray(m.n, np.float64), np.ascontiguousarray(m.centroid, np.float64),
                      np.ascontiguousarray(m.volume, np.float64),
                      np.ascontiguousarray(m.cell_centroid, np.float64),
                      np.ascontiguousarray(m.cell_face_off, self.off_dtype),
                      np.ascontiguousarray(m.cell_face_ids, np.int32)]
        rc = self._fn("set_mesh")(self.h, ctypes.c_int(m.ncell), ctypes.c_int(m.nface),
                                  *[_p(a) for a in self._keep])
        assert rc == 0

    def init_problem(self, W, bnd=None, rung_offset=0):
        m = self.mesh
        W = np.ascontiguousarray(W, np.float64)
        pos = np.ascontiguousarray(m.pos, np.float64)
        b = None if bnd is None else np.ascontiguousarray(bnd, np.int32)
        rc = self._fn("init_problem")(self.h, _p(W), _p(pos), _p(b), ctypes.c_int(rung_offset))
        assert rc == 0

    def step(self, shared=True, snap=False):
        n, nf = self.mesh.ncell, self.mesh.nface
        s = None
        out = {}
        if snap:
            s = _Snap()
            for name, dt, w in SNAP_FIELDS:
                if w == 0:
                    a = np.zeros(nf, dt)
                elif w == -1:
                    a = np.zeros(1, dt)
                else:
                    a = np.zeros((n, w) if w > 1 else n, dt)
                out[name] = a
                setattr(s, name, a.ctypes.data)
        nact = self._fn("step")(self.h, ctypes.c_int(1 if shared else 0), ctypes.byref(s) if s else None)
        if snap:
            out["active_faces"] = out["active_faces"][: int(out["nactive_faces"][0])]
            out["nactive"] = nact
            return out
        return nact

    @property
    def time(self):
        return self._fn("time")(self.h)

    def get_state(self):
        n = self.mesh.ncell
        st = dict(pos=np.zeros((n, 3)), vel=np.zeros((n, 3)), tlast=np.zeros(n), tend=np.zeros(n),
                  rung=np.zeros(n, np.int32), U=np.zeros((n, 10)), dU=np.zeros((n, 14)),
                  wrec=np.zeros((n, 50)))
        self._fn("get_state")(self.h, *[_p(st[k]) for k in ("pos", "vel", "tlast", "tend", "rung", "U", "dU", "wrec")])
        return st

    def get_motion(self):
        n = self.mesh.ncell
        out = dict(orig_pos=np.zeros((n, 3)), orig_vel=np.zeros((n, 3)), divb=np.zeros(n, np.float32))
        self._fn("get_motion")(self.h, _p(out["orig_pos"]), _p(out["orig_vel"]), _p(out["divb"]))
        return out

    def compute_flux(self, wij, Wi, Wj, jbnd, normal):
        nf = Wi.shape[0]
        wij, Wi, Wj, normal = (np.ascontiguousarray(a, np.float64) for a in (wij, Wi, Wj, normal))
        jb = np.ascontiguousarray(jbnd, np.int32)
        psi, Bn, flux = np.zeros(nf), np.zeros(nf), np.zeros((nf, 10))
        self._fn("compute_flux")(self.h, ctypes.c_int(nf), _p(wij), _p(Wi), _p(Wj), _p(jb), _p(normal),
                                 _p(psi), _p(Bn), _p(flux))
        return psi, Bn, flux


class RefSystem(_Base):
    """The reference's compiled hot path (one rank)."""
    prefix = "ref_"
    so = REF_SO
    off_dtype = np.int32

    def dump_binary(self, path):
        """The reference's own snapshot writer (MPI/dump_binary.cpp)."""
        self._fn("dump_binary")(self.h, ctypes.c_char_p(str(path).encode()))

    @property
    def tsys_ticks(self):
        f = self._fn("tsys_ticks")
        f.restype = ctypes.c_ulonglong
        return int(f(self.h))


class OracleSystem(_Base):
    """The plain-C restatement."""
    prefix = "fvo_"
    so = ORACLE_SO
    off_dtype = np.int64

    def clock(self):
        """(tsysU, dt_global, iteration) after the last step."""
        t = ctypes.c_ulonglong(0)
        dt = ctypes.c_double(0.0)
        it = ctypes.c_longlong(0)
        self._fn("clock")(self.h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(it))
        return t.value, dt.value, it.value

    def dump_binary_bytes(self, bnd=None, idx=None, rmax=None):
        """Restatement of system::dump_binary (MPI/dump_binary.cpp:5-99) for
        one rank over this oracle's state: returns the file's bytes."""
        p = self.params
        n = self.mesh.ncell
        st = self.get_state()
        mo = self.get_motion()
        tsys, dt_global, iteration = self.clock()
        vol = np.asarray(self.mesh.volume, np.float64)
        bnd = np.zeros(n, np.int32) if bnd is None else np.asarray(bnd, np.int32)
        out = [struct.pack("<4iQ", 80, 0, 1, 1, tsys),
               struct.pack("<3i2fi2fi", n, n, 3, self.time, dt_global, iteration, p.courant, p.gamma, -1),
               struct.pack("<6fi", 0.0, 0.0, 0.0, p.box[0], p.box[1], p.box[2], 80)]
        dt_tick = p.dtmax / float(1 << 31)
        for i in range(n):
            W = _to_primitive(st["U"][i], vol[i])
            pres = ((p.gamma - 1.0) * W[4] if p.gamma > 1.0 else W[4]) if p.eos == 0 else W[4]
            L = math.pow(vol[i] * 3.0 / 4.0 / math.pi, 1.0 / 3.0)
            dt = dt_tick * float(1 << (31 - int(st["rung"][i])))
            out.append(struct.pack(
                "<ii3f3f4fi3f3f5f3fi", 104, i if idx is None else int(idx[i]),
                *mo["orig_pos"][i], *mo["orig_vel"][i], W[0], W[4], pres,
                0.0 if rmax is None else float(rmax[i]), int(bnd[i]),
                W[1], W[2], W[3], W[5], W[6], W[7], dt, vol[i], W[8],
                L * float(mo["divb"][i]), W[9], 0.0, 0.0, 0.0, 104))
        return b"".join(out)

    def set_state(self, vel=None, tlast=None, tend=None, rung=None, U=None, dU=None, wrec=None, tsys_ticks=0):
        f = self._fn("set_state")
        conv = [None if a is None else np.ascontiguousarray(a, t) for a, t in
                ((vel, np.float64), (tlast, np.float64), (tend, np.float64), (rung, np.int32),
                 (U, np.float64), (dU, np.float64), (wrec, np.float64))]
        f(self.h, *[_p(a) for a in conv], ctypes.c_ulonglong(tsys_ticks))
