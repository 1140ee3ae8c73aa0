"""Domain decomposition and halo exchange (fvmhd3d_b200/halo.py) across
ranks on the CPU with the gloo backend."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _mesh():
    import fvmhd3d_b200 as F
    return F.build_periodic(F.jittered_lattice(7, 0.1, seed=21), 1.0)


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from fvmhd3d_b200 import halo
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        m = _mesh()
        owner = halo.partition(m.pos, m.box, world)
        plan = halo.HaloPlan(m, owner, rank, depth=2)
        rng = np.random.default_rng(0)
        G = rng.normal(size=(m.ncell, 10))
        local = np.zeros((plan.cells.size, 10))
        local[:plan.nowned] = G[plan.owned]
        got = plan.exchange(local)
        ok_ex = bool(np.array_equal(got, G[plan.cells]))
        # every local cell contributes 1 + its global index to itself; after
        # collect, each owner holds the number of ranks that hold the cell
        C = np.zeros((plan.cells.size, 2))
        C[:, 0] = 1.0
        C[:, 1] = plan.cells
        back = plan.collect(C)
        out[rank] = (ok_ex, plan.owned.copy(), back[:plan.nowned].copy(), int(plan.halo.size))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_halo_exchange_and_collect(world):
    import torch.multiprocessing as mp
    from fvmhd3d_b200 import halo
    m = _mesh()
    owner = halo.partition(m.pos, m.box, world)
    assert np.bincount(owner).min() >= m.ncell // world - 1
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    holders = np.zeros(m.ncell)
    plans = [halo.HaloPlan(m, owner, r, depth=2) for r in range(world)]
    for p in plans:
        holders[p.cells] += 1
    owned_all = []
    for r in range(world):
        ok, owned, back, nhalo = out[r]
        assert ok, r
        assert nhalo > 0
        owned_all.append(owned)
        assert np.array_equal(back[:, 0], holders[owned])            # one contribution per holder
        assert np.array_equal(back[:, 1], holders[owned] * owned)     # summed exactly
    assert np.array_equal(np.sort(np.concatenate(owned_all)), np.arange(m.ncell))


def test_plan_local_faces_cover_owned_stencils():
    """Every face of an owned cell, and of a ring-1 cell, is local (depth 2):
    the limiter and flux of the owned cells see complete stencils."""
    from fvmhd3d_b200 import halo
    m = _mesh()
    owner = halo.partition(m.pos, m.box, 2)
    p = halo.HaloPlan(m, owner, 0, depth=2)
    local_faces = np.zeros(m.nface, bool)
    local_faces[p.faces] = True
    ring1 = set()
    for c in p.owned:
        for q in range(m.cell_face_off[c], m.cell_face_off[c + 1]):
            f = m.cell_face_ids[q]
            assert local_faces[f]
            ring1.add(int(m.s1[f]) if m.s2[f] == c else int(m.s2[f]))
    for c in ring1:
        for q in range(m.cell_face_off[c], m.cell_face_off[c + 1]):
            assert local_faces[m.cell_face_ids[q]]
