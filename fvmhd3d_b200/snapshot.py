"""The reference's snapshot file format (MPI/dump_binary.cpp,
MPI/read_binary.cpp), single rank.

The file is a sequence of Fortran-style records, each framed by its byte
count as an int32 before and after:

* a header of 20 words: myproc, nproc, nproc, tsysU (two uint32 words, low
  first), global_n, local_n, ndim=3, t_global (float), dt_global (float),
  iteration, courant (float), gamma (float), -1, domain rmin[3] and rmax[3]
  (float);
* one record of 26 words per cell: idx, orig_pos[3], orig_vel[3], DENS,
  ETHM, pressure, rmax, boundary (int), VELX..VELZ, BX..BZ, dt of the rung,
  volume, PSI, L*divB (L the radius of the sphere of the cell's volume),
  ENTR, J[3] (floats unless marked int).

:meth:`fvmhd3d_b200.System.dump_binary` writes it from the device state;
:func:`read_binary` reads it back into numpy arrays and
:func:`restart_inputs` turns a snapshot into the inputs of a new run the way
``system::read_binary`` does (positions and primitives from the file, the
clock at the file's tsysU).
"""
from __future__ import annotations

import numpy as np

HEADER_BYTES = 20 * 4
RECORD_BYTES = 26 * 4

HEADER_DTYPE = np.dtype([
    ("m0", "<i4"), ("myproc", "<i4"), ("nproc", "<i4"), ("nproc2", "<i4"), ("tsys", "<u8"),
    ("global_n", "<i4"), ("local_n", "<i4"), ("ndim", "<i4"), ("t_global", "<f4"), ("dt_global", "<f4"),
    ("iteration", "<i4"), ("courant", "<f4"), ("gamma", "<f4"), ("periodic", "<i4"),
    ("rmin", "<f4", 3), ("rmax", "<f4", 3), ("m1", "<i4"),
])

RECORD_DTYPE = np.dtype([
    ("m0", "<i4"), ("idx", "<i4"), ("pos", "<f4", 3), ("vel", "<f4", 3), ("dens", "<f4"), ("ethm", "<f4"),
    ("pres", "<f4"), ("rmax", "<f4"), ("boundary", "<i4"), ("velp", "<f4", 3), ("B", "<f4", 3),
    ("dt", "<f4"), ("volume", "<f4"), ("psi", "<f4"), ("Ldivb", "<f4"), ("entr", "<f4"), ("J", "<f4", 3),
    ("m1", "<i4"),
])

assert HEADER_DTYPE.itemsize == HEADER_BYTES + 8 and RECORD_DTYPE.itemsize == RECORD_BYTES + 8


class SnapshotError(ValueError):
    pass


def parse(buf) -> tuple[dict, np.ndarray]:
    """(header dict, structured record array) of a snapshot held in memory."""
    buf = memoryview(buf).cast("B")
    if len(buf) < HEADER_DTYPE.itemsize:
        raise SnapshotError(f"{len(buf)} bytes: shorter than the header")
    h = np.frombuffer(buf, HEADER_DTYPE, count=1)[0]
    if h["m0"] != HEADER_BYTES or h["m1"] != HEADER_BYTES:
        raise SnapshotError(f"bad header markers {h['m0']}, {h['m1']} (expected {HEADER_BYTES})")
    if h["ndim"] != 3:
        raise SnapshotError(f"ndim {h['ndim']} (expected 3)")
    n = int(h["local_n"])
    body = len(buf) - HEADER_DTYPE.itemsize
    if n < 0 or body != n * RECORD_DTYPE.itemsize:
        raise SnapshotError(f"{body} bytes of records for local_n={n} (expected {n * RECORD_DTYPE.itemsize}); "
                            "files of several ranks are not supported")
    rec = np.frombuffer(buf, RECORD_DTYPE, count=n, offset=HEADER_DTYPE.itemsize)
    if n and not ((rec["m0"] == RECORD_BYTES).all() and (rec["m1"] == RECORD_BYTES).all()):
        raise SnapshotError("bad record markers")
    header = {k: (h[k].copy() if h[k].shape else h[k].item()) for k in HEADER_DTYPE.names if k not in ("m0", "m1")}
    return header, rec


def read_binary(path) -> tuple[dict, np.ndarray]:
    """Reads a snapshot file written by the reference or by System.dump_binary."""
    with open(path, "rb") as f:
        return parse(f.read())


def primitives(rec: np.ndarray) -> np.ndarray:
    """(n, 10) primitive state of the records in the reference's Fluid order
    (DENS, VELX, VELY, VELZ, ETHM, BX, BY, BZ, PSI, ENTR), in float64."""
    W = np.zeros((rec.shape[0], 10))
    W[:, 0] = rec["dens"]
    W[:, 1:4] = rec["velp"]
    W[:, 4] = rec["ethm"]
    W[:, 5:8] = rec["B"]
    W[:, 8] = rec["psi"]
    W[:, 9] = rec["entr"]
    return W


def restart_inputs(header: dict, rec: np.ndarray, box) -> dict:
    """What system::read_binary (MPI/read_binary.cpp) rebuilds from a file:
    generator positions wrapped into the periodic box, primitives, boundary
    flags, particle ids and the clock (tsys ticks).  The positions feed the
    mesh builder, W/bnd feed System.init_problem."""
    box = np.broadcast_to(np.asarray(box, np.float64), (3,))
    pos = np.mod(rec["pos"].astype(np.float64), box)
    return dict(pos=pos, W=primitives(rec), bnd=rec["boundary"].astype(np.int32), idx=rec["idx"].copy(),
                rmax=rec["rmax"].copy(), tsys=int(header["tsys"]), t_global=float(header["t_global"]))
