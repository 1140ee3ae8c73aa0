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
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libfvmref.so")
ORACLE_SO = os.path.join(HERE, "_ref", "liboracle.so")


def build(ref: bool = True) -> None:
    """Compile the checkers with oracle/Makefile (the reference build only when
    its sources are present)."""
    targets = ["oracle"]
    if ref and os.path.isdir("/root/reference/MPI"):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


class _Params(ctypes.Structure):
    _fields_ = [
        ("gamma", ctypes.c_double),
        ("courant", ctypes.c_double),
        ("box", ctypes.c_double * 3),
        ("dtmax", ctypes.c_double),
        ("eos", ctypes.c_int),
        ("iso_GM", ctypes.c_double),
        ("iso_cfac", ctypes.c_double),
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


def make_params(gamma=5.0 / 3.0, courant=0.4, box=(1.0, 1.0, 1.0), dtmax=1.0 / 64, eos=0,
                iso_GM=1.0, iso_cfac=0.05) -> _Params:
    p = _Params()
    p.gamma, p.courant = gamma, courant
    for a in range(3):
        p.box[a] = box[a]
    p.dtmax, p.eos, p.iso_GM, p.iso_cfac = dtmax, eos, iso_GM, iso_cfac
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


class OracleSystem(_Base):
    """The plain-C restatement."""
    prefix = "fvo_"
    so = ORACLE_SO
    off_dtype = np.int64

    def set_state(self, vel=None, tlast=None, tend=None, rung=None, U=None, dU=None, wrec=None, tsys_ticks=0):
        f = self._fn("set_state")
        conv = [None if a is None else np.ascontiguousarray(a, t) for a, t in
                ((vel, np.float64), (tlast, np.float64), (tend, np.float64), (rung, np.int32),
                 (U, np.float64), (dU, np.float64), (wrec, np.float64))]
        f(self.h, *[_p(a) for a in conv], ctypes.c_ulonglong(tsys_ticks))
