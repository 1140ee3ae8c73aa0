"""Host-side Voronoi mesh for periodic boxes.

The reference builds its moving Voronoi mesh with CGAL on the host
(MPI/build_mesh_active.cpp:121-851) and hands the fluid hot path two arrays:
``face_list`` (``Face{s1, s2, centroid, n}``, MPI/fvmhd3d.h:169-191) and
``cell_list`` (``Cell{Volume, centroid, ngb}``, MPI/fvmhd3d.h:221-249).  CGAL
is not available here, so :func:`build_periodic` computes the same mesh with
the project's own half-space clipping builder (``csrc/voronoi.cpp``), keeping
the reference's conventions:

* ``n`` is the area-weighted normal pointing from ``s1`` to ``s2``;
* ``centroid`` is stored in the periodic frame of ``s1``;
* a cell's face list is in face-creation order (faces first met by lower
  numbered cells come first), which fixes the active-face order.

Mesh construction is host work and is timed separately from the fluid path.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libfvmmesh.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing; run __graft_entry__.build()")
        lib = ctypes.CDLL(path)
        lib.fvm_mesh_build.restype = ctypes.c_void_p
        lib.fvm_mesh_build.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        lib.fvm_mesh_error.argtypes = [ctypes.c_void_p]
        lib.fvm_mesh_sizes.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.fvm_mesh_fetch.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 8
        lib.fvm_mesh_free.argtypes = [ctypes.c_void_p]
        _LIB = lib
    return _LIB


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


@dataclass
class Mesh:
    """Voronoi mesh in the reference's face/cell convention (see module doc)."""

    box: np.ndarray            # (3,) periodic box size
    pos: np.ndarray            # (ncell, 3) generator positions in [0, box)
    s1: np.ndarray             # (nface,) int32
    s2: np.ndarray             # (nface,) int32
    n: np.ndarray              # (nface, 3) area-weighted normal s1 -> s2
    centroid: np.ndarray       # (nface, 3) face centroid in the frame of s1
    volume: np.ndarray         # (ncell,)
    cell_centroid: np.ndarray  # (ncell, 3) in the frame of the generator
    cell_face_off: np.ndarray  # (ncell+1,) int64 CSR offsets
    cell_face_ids: np.ndarray  # (nlink,) int32 face ids per cell

    @property
    def ncell(self) -> int:
        return int(self.pos.shape[0])

    @property
    def nface(self) -> int:
        return int(self.s1.shape[0])

    def closure_error(self) -> np.ndarray:
        """|sum of outward area vectors| / V^(2/3) per cell (the reference's
        closure check, MPI/compute_update.cpp:307-320)."""
        acc = np.stack([np.bincount(self.s1, self.n[:, k], self.ncell) - np.bincount(self.s2, self.n[:, k], self.ncell)
                        for k in range(3)], axis=1)
        return np.linalg.norm(acc, axis=1) / self.volume ** (2.0 / 3.0)

    def save(self, path) -> None:
        """Write the mesh arrays to an uncompressed .npz (for processes that
        share one host-built mesh)."""
        np.savez(path, box=self.box, pos=self.pos, s1=self.s1, s2=self.s2, n=self.n, centroid=self.centroid,
                 volume=self.volume, cell_centroid=self.cell_centroid, cell_face_off=self.cell_face_off,
                 cell_face_ids=self.cell_face_ids)

    @staticmethod
    def load(path) -> "Mesh":
        z = np.load(path)
        return Mesh(z["box"], z["pos"], z["s1"], z["s2"], z["n"], z["centroid"], z["volume"], z["cell_centroid"],
                    z["cell_face_off"], z["cell_face_ids"])


def build_periodic(pos: np.ndarray, box, nthreads: int = 0) -> Mesh:
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    box = np.ascontiguousarray(np.broadcast_to(np.asarray(box, dtype=np.float64), (3,)))
    n = pos.shape[0]
    lib = _lib()
    h = lib.fvm_mesh_build(n, _ptr(pos), _ptr(box), int(nthreads))
    if not h:
        raise MemoryError("Voronoi build failed")
    try:
        err = lib.fvm_mesh_error(h)
        if err:
            raise RuntimeError(f"Voronoi build error flag {err}: 1 candidate search exhausted, 2 cell reaches the "
                               "bounding box, 4 a cell meets two periodic images of one neighbour (mesh too "
                               "coarse for the box)")
        nface = ctypes.c_int(0)
        nlink = ctypes.c_longlong(0)
        lib.fvm_mesh_sizes(h, ctypes.byref(nface), ctypes.byref(nlink))
        nf, nl = nface.value, nlink.value
        s1 = np.empty(nf, np.int32)
        s2 = np.empty(nf, np.int32)
        fn = np.empty((nf, 3))
        fc = np.empty((nf, 3))
        vol = np.empty(n)
        cc = np.empty((n, 3))
        off = np.empty(n + 1, np.int64)
        ids = np.empty(nl, np.int32)
        lib.fvm_mesh_fetch(h, _ptr(s1), _ptr(s2), _ptr(fn), _ptr(fc), _ptr(vol), _ptr(cc), _ptr(off), _ptr(ids))
    finally:
        lib.fvm_mesh_free(h)
    m = Mesh(box, pos, s1, s2, fn, fc, vol, cc, off, ids)
    # The mesh holds one face per cell pair (minimum image), so every cell
    # must be closed: a cell that meets two periodic images of a neighbour
    # (mesh too coarse for the box) shows up here.  Same bound as the
    # reference's check, MPI/compute_update.cpp:307-320.
    bad = np.nonzero(m.closure_error() >= 1e-10)[0]
    if bad.size:
        raise RuntimeError(f"Voronoi mesh not closed for {bad.size} cells (first {int(bad[0])}): the generators "
                           "are too coarse for the periodic box")
    return m


def jittered_lattice(nside: int, jitter: float = 0.1, seed: int = 1, box: float = 1.0) -> np.ndarray:
    """nside^3 generators on a cubic lattice in [0, box)^3, each moved by a
    uniform offset in [-jitter, +jitter] lattice spacings per axis (seeded).
    Ordered x fastest."""
    rng = np.random.default_rng(seed)
    h = box / nside
    idx = np.arange(nside, dtype=np.float64)
    z, y, x = np.meshgrid(idx, idx, idx, indexing="ij")
    p = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    p = (p + 0.5 + rng.uniform(-jitter, jitter, size=p.shape)) * h
    return np.mod(p, box)
