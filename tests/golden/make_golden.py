"""Generates the golden fixtures in this directory from the reference's own
hot path (oracle/_ref/libfvmref.so, compiled from the reference's MPI-tree
sources by oracle/Makefile).

    make -C oracle ref && python tests/golden/make_golden.py

Each .npz holds the inputs (mesh arrays, initial primitives, flags) and the
reference's outputs, so the plain-C oracle and the CUDA path can be pinned
without the reference being present.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.pyoracle import RefSystem  # noqa: E402
import fvmhd3d_b200 as F  # noqa: E402


def mesh_arrays(m):
    return dict(box=m.box, pos=m.pos, s1=m.s1, s2=m.s2, n=m.n, centroid=m.centroid, volume=m.volume,
                cell_centroid=m.cell_centroid, cell_face_off=m.cell_face_off, cell_face_ids=m.cell_face_ids)


def finish(R, out, nact, faces, path):
    """Final state, generator motion, clock and the reference's own snapshot
    file (system::dump_binary) after the last step."""
    st = R.get_state()
    out.update({"out_" + k: v for k, v in st.items()})
    mo = R.get_motion()
    out.update({"out_" + k: v for k, v in mo.items()})
    out["out_time"] = np.float64(R.time)
    out["out_tsys"] = np.uint64(R.tsys_ticks)
    out["out_nactive"] = np.array(nact, np.int32)
    out["out_last_active_faces"] = faces[-1]
    tmp = path + ".dump.tmp"
    R.dump_binary(tmp)
    with open(tmp, "rb") as f:
        out["out_dump_binary"] = np.frombuffer(f.read(), np.uint8)
    os.unlink(tmp)
    np.savez_compressed(path, **out)


def run_case(name, nside, problem, shared, nsteps, seed, noise=0.05):
    m = F.build_periodic(F.jittered_lattice(nside, 0.1, seed=seed), 1.0)
    W = F.problems.perturbed(getattr(F.problems, problem)(m.pos), noise, seed=seed + 1)
    R = RefSystem()
    R.set_mesh(m)
    R.init_problem(W)
    out = dict(mesh_arrays(m), W=W, shared=np.int32(shared), nsteps=np.int32(nsteps))
    nact, faces = [], []
    for _ in range(nsteps):
        s = R.step(shared=bool(shared), snap=True)
        nact.append(s["nactive"])
        faces.append(s["active_faces"])
    finish(R, out, nact, faces, os.path.join(HERE, name))
    print(name, m.ncell, "cells", m.nface, "faces; active per step", nact)


def disk_case(name, n, nsteps, seed=3, static_mesh=False):
    """Keplerian disk, isothermal EOS, individual timesteps, with a DIOD sink;
    generators moving with the flow, or static (compute_pvel1 hook)."""
    pos, box = F.problems.disk_generators(n, seed=seed)
    m = F.build_periodic(pos, box)
    W, bnd = F.problems.disk(pos, box, r_sink=0.55)
    prm = dict(gamma=1.0, courant=0.4, box=tuple(box), dtmax=1.0 / 16, eos=1, iso_GM=1.0, iso_cfac=0.05,
               static_mesh=static_mesh)
    R = RefSystem(**prm)
    R.set_mesh(m)
    R.init_problem(W, bnd=bnd)
    out = dict(mesh_arrays(m), W=W, bnd=bnd, shared=np.int32(0), nsteps=np.int32(nsteps),
               params=np.array([prm["gamma"], prm["courant"], box[0], box[1], box[2], prm["dtmax"], 1.0, 1.0, 0.05,
                                float(static_mesh)]))
    nact, faces = [], []
    for _ in range(nsteps):
        s = R.step(shared=False, snap=True)
        nact.append(s["nactive"])
        faces.append(s["active_faces"])
    finish(R, out, nact, faces, os.path.join(HERE, name))
    print(name, m.ncell, "cells", m.nface, "faces,", int((bnd > 0).sum()), "DIOD cells; active per step", nact)


def flux_case(name, nface=256, seed=5):
    rng = np.random.default_rng(seed)
    Wi = np.zeros((nface, 10))
    Wj = np.zeros((nface, 10))
    for W in (Wi, Wj):
        W[:, 0] = rng.uniform(0.1, 3.0, nface)
        W[:, 1:4] = rng.normal(0, 1.0, (nface, 3))
        W[:, 4] = rng.uniform(0.05, 5.0, nface)
        W[:, 5:8] = rng.normal(0, 1.0, (nface, 3))
        W[:, 8] = rng.normal(0, 0.1, nface)
        W[:, 9] = rng.uniform(0.5, 2.0, nface)
    nrm = rng.normal(size=(nface, 3))
    nrm[:8] = [[0, 0, 1], [0, 0, -1], [1, 0, 0], [0, 1, 0], [0, -1, 0], [-1, 0, 0], [1, 1, 0], [0, 1, 1]]
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    wij = rng.normal(0, 1.0, (nface, 3))
    wij[:16] = 0.0
    jbnd = np.zeros(nface, np.int32)
    jbnd[nface // 2: nface // 2 + 32] = 1     # REFLECTING
    jbnd[nface // 2 + 32: nface // 2 + 64] = 3  # DIOD
    R = RefSystem()
    psi, Bn, flux = R.compute_flux(wij, Wi, Wj, jbnd, nrm)
    np.savez_compressed(os.path.join(HERE, name), wij=wij, Wi=Wi, Wj=Wj, jbnd=jbnd, normal=nrm,
                        psi=psi, Bn=Bn, flux=flux)
    print(name, nface, "faces")


if __name__ == "__main__":
    run_case("ref_alfven4_shared.npz", 4, "alfven", True, 3, seed=11)
    run_case("ref_blast7_individual.npz", 7, "blast", False, 14, seed=5, noise=0.2)
    run_case("ref_blast8_individual.npz", 8, "blast", False, 10, seed=12)
    run_case("ref_ot5_shared.npz", 5, "orszag_tang", True, 6, seed=13)
    disk_case("ref_disk4k_individual.npz", 4096, 12)
    disk_case("ref_disk4k_static_individual.npz", 4096, 16, seed=8, static_mesh=True)
    flux_case("ref_flux_kat.npz")
