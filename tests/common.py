"""Shared helpers for the parity tests."""
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libfvmref.so")
ORACLE_SO = os.path.join(ROOT, "oracle", "_ref", "liboracle.so")

# Tolerance of the plain FP64 GPU path against the FP64 oracle: per
# variable, max |gpu - oracle| over cells divided by max |oracle| over cells.
RTOL_FP64 = 1e-12


def maxrel(a, b, axis=0, scale=None):
    """Per-column max-norm relative error of a against b.  The denominator is
    max |b| over cells per column, or max |scale| when a subset of cells is
    compared (so that a column that is near zero on the subset is measured
    against its magnitude over the whole mesh)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.ndim == 1:
        a, b = a[:, None], b[:, None]
    ref = b if scale is None else np.asarray(scale, dtype=np.float64).reshape(-1, a.shape[1])
    den = np.abs(ref).max(axis=axis)
    den = np.where(den > 0, den, 1.0)
    return np.abs(a - b).max(axis=axis) / den


def setup_case(nside=8, problem="alfven", seed=1, noise=0.05, gamma=5.0 / 3.0):
    import fvmhd3d_b200 as F
    m = F.build_periodic(F.jittered_lattice(nside, 0.1, seed=seed), 1.0)
    W = getattr(F.problems, problem)(m.pos)
    if noise:
        W = F.problems.perturbed(W, noise, seed=seed + 100)
    return m, W


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GOLDEN_STEP_CASES = ["ref_alfven4_shared.npz", "ref_ot5_shared.npz", "ref_blast7_individual.npz",
                     "ref_blast8_individual.npz", "ref_disk4k_individual.npz",
                     "ref_disk4k_static_individual.npz"]


def golden_params(z):
    """System parameters of a fixture (ideal gas, unit box by default; the
    disk fixtures store gamma, courant, box, dtmax, eos, GM, cfac and, in
    the static-generator one, static_mesh)."""
    if "params" not in z:
        return {}
    p = z["params"]
    out = dict(gamma=float(p[0]), courant=float(p[1]), box=(float(p[2]), float(p[3]), float(p[4])),
               dtmax=float(p[5]), eos=int(p[6]), iso_GM=float(p[7]), iso_cfac=float(p[8]))
    if p.shape[0] > 9:
        out["static_mesh"] = bool(p[9])
    return out


def load_golden(name):
    """(mesh, fixture dict) of a golden fixture written by golden/make_golden.py."""
    from fvmhd3d_b200.mesh import Mesh
    z = dict(np.load(os.path.join(GOLDEN, name)))
    m = Mesh(z["box"], z["pos"], z["s1"], z["s2"], z["n"], z["centroid"], z["volume"], z["cell_centroid"],
             z["cell_face_off"], z["cell_face_ids"])
    return m, z
