"""A run on a partitioned mesh (fvmhd3d_b200/halo.py `Domain`): each rank
steps its owned cells plus three rings of neighbour copies on its own
system, takes the timestep minimum over ranks through the system's
reduction (fvm_set_reduce; MPI/compute_timestep.cpp:101) and copies the
neighbour rows from their owners after every step
(MPI/distribute_work.cpp:367-724).  The owned cells must hold the bits of
the same steps on the whole mesh: their faces are listed in the same order
and every neighbour they read is exact.

Ranks are gloo processes.  The CPU tests step each domain with the oracle
(a timestep cap below every cell's CFL limit, so the minimum needs no
reduction); the GPU test steps each domain with the CUDA system on the one
GPU (the ranks' kernels never wait on one another: every exchange and the
reduction go through the host) on a blast whose CFL limit sets the step."""
import socket

import numpy as np
import pytest

from common import golden_params, load_golden, setup_case

KEYS = ("vel", "tlast", "tend", "rung", "U", "dU", "wrec")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case(nside):
    return setup_case(nside, "blast", seed=3, noise=0.02)


DISK = "ref_disk4k_individual.npz"


def _problem(case):
    """(mesh, W, boundary codes, system parameters) of a blast nside^3
    (an int) or of the Keplerian disk fixture with its sink cells."""
    if case == "disk":
        m, z = load_golden(DISK)
        return m, z["W"], z.get("bnd"), golden_params(z)
    m, W = _case(case)
    return m, W, None, {}


def _make(engine, params, precision):
    def make(m):
        if engine == "oracle":
            from oracle.pyoracle import OracleSystem
            s = OracleSystem(**params)
        else:
            import fvmhd3d_b200 as F
            s = F.System(precision=precision, **params)
        s.set_mesh(m)
        return s
    return make


def _worker(rank, world, port, case, nsteps, engine, dtmax, precision, depth, out):
    import torch.distributed as dist
    from fvmhd3d_b200 import halo
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        m, W, bnd, params = _problem(case)
        owner = halo.partition(m.pos, m.box, world)
        d = halo.Domain(m, owner, rank, _make(engine, dict(params, dtmax=dtmax), precision), depth=depth)
        d.init_problem(W, bnd=bnd)
        for _ in range(nsteps):
            d.step()
        owned, st = d.owned_state()
        out[rank] = (owned, st, d.sys.time, d.ticks, int(d.plan.halo.size), d.mesh.ncell)
    finally:
        dist.destroy_process_group()


def run_partitioned(world, case, nsteps, engine, dtmax, precision=0, depth=3):
    import torch.multiprocessing as mp
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), case, nsteps, engine, dtmax, precision, depth, out),
                       nprocs=world, join=True, start_method="spawn")
    return [out[r] for r in range(world)]


def assert_owned_bits(parts, whole, time, ticks, ncell):
    seen = np.zeros(ncell, bool)
    for owned, st, t, tk, nhalo, nloc in parts:
        assert nhalo > 0 and nloc < ncell  # each rank holds a proper part with copies
        assert t == time and tk == ticks
        seen[owned] = True
        for k in KEYS:
            a = np.asarray(whole[k]).reshape(ncell, -1)[owned]
            b = np.asarray(st[k]).reshape(len(owned), -1)
            assert np.array_equal(a, b), k
    assert seen.all()


def oracle_steps(case, nsteps, dtmax):
    from oracle.pyoracle import OracleSystem
    m, W, bnd, params = _problem(case)
    o = OracleSystem(**dict(params, dtmax=dtmax))
    o.set_mesh(m)
    o.init_problem(W, bnd=bnd)
    for _ in range(nsteps):
        o.step(shared=True)
    return m, o


def test_local_mesh_keeps_each_owned_cells_face_order():
    from fvmhd3d_b200 import halo
    m, _ = _case(12)
    owner = halo.partition(m.pos, m.box, 3)
    for owned_first in (True, False):
        p = halo.HaloPlan(m, owner, 1, depth=3, owned_first=owned_first)
        lm = halo.local_mesh(m, p)
        assert lm.ncell == p.cells.size and lm.nface == p.faces.size
        for lc in np.nonzero(~p.is_halo)[0]:
            c = p.cells[lc]
            g = m.cell_face_ids[m.cell_face_off[c]:m.cell_face_off[c + 1]]
            loc = lm.cell_face_ids[lm.cell_face_off[lc]:lm.cell_face_off[lc + 1]]
            assert np.array_equal(p.faces[loc], g)  # every face, in the same order
            assert np.array_equal(p.cells[lm.s1[loc]], m.s1[g]) and np.array_equal(p.cells[lm.s2[loc]], m.s2[g])
        # the copies in the outer ring miss faces
        h = p.is_halo
        assert (np.diff(lm.cell_face_off)[h] < np.diff(m.cell_face_off)[p.cells[h]]).any()
    assert np.array_equal(p.cells, np.sort(p.cells))


@pytest.mark.parametrize("world", [2, 3, 4])
def test_partitioned_oracle_steps_give_the_whole_mesh_bits(world):
    nside, nsteps, dtmax = 16, 3, 1e-4
    m, o = oracle_steps(nside, nsteps, dtmax)
    parts = run_partitioned(world, nside, nsteps, "oracle", dtmax)
    assert_owned_bits(parts, o.get_state(), o.time, o.clock()[0], m.ncell)


def test_partitioned_oracle_steps_on_the_disk_with_its_sink():
    """The Keplerian disk fixture (isothermal gas, moving generators, sink
    cells with boundary codes): the copies carry their boundary codes and the
    owned cells keep the whole mesh's bits."""
    nsteps, dtmax = 3, 0.0625 / 1024
    m, o = oracle_steps("disk", nsteps, dtmax)
    parts = run_partitioned(2, "disk", nsteps, "oracle", dtmax)
    assert_owned_bits(parts, o.get_state(), o.time, o.clock()[0], m.ncell)


def test_two_rings_are_not_enough():
    """The depth the exchange after each step needs: with two rings of
    copies some owned cell reads a neighbour the step left wrong."""
    nside, nsteps, dtmax = 16, 2, 1e-4
    m, o = oracle_steps(nside, nsteps, dtmax)
    whole = o.get_state()
    parts = run_partitioned(2, nside, nsteps, "oracle", dtmax, depth=2)
    assert any(not np.array_equal(np.asarray(whole[k])[owned], st[k]) for owned, st, *_ in parts for k in KEYS)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_partitioned_gpu_steps_give_the_whole_mesh_bits(precision):
    """Two ranks on the GPU with the timestep set by the CFL limit: the
    reduction hands every rank the whole mesh's minimum."""
    import fvmhd3d_b200 as F
    prec = F.FVM_PREC_FP32 if precision == "fp32" else F.FVM_PREC_FP64
    nside, nsteps, dtmax = 16, 4, 1.0 / 64
    m, W = _case(nside)
    s = F.System(dtmax=dtmax, precision=prec)
    s.set_mesh(m)
    s.init_problem(W)
    for _ in range(nsteps):
        s.step(shared=True)
    whole = s.get_state()
    assert whole["rung"].max() > 0  # the CFL limit, not the cap, sets the step
    parts = run_partitioned(2, nside, nsteps, "gpu", dtmax, precision=prec)
    assert_owned_bits(parts, whole, s.time, s.tsys_ticks, m.ncell)


@pytest.mark.gpu
def test_reduction_hook_contract():
    """The reduction is called once per step (and once by init_problem) with
    this system's minimum, its result is the step's, a failing reduction
    fails the step, and graph-replayed steps are refused while it is set."""
    import fvmhd3d_b200 as F
    m, W = _case(8)
    s = F.System()
    s.set_mesh(m)
    seen = []
    s.set_reduce(lambda v: (seen.append(v), v)[1])
    s.init_problem(W)
    assert len(seen) == 1
    s.step(shared=True)
    assert len(seen) == 2
    with pytest.raises(F.FvmError):
        s.run(1, shared=True)
    # a smaller minimum from another rank puts every cell on a finer rung
    r0 = s.get_state()["rung"].max()
    s.set_reduce(lambda v: v / 8.0)
    s.step(shared=True)
    assert s.get_state()["rung"].max() >= r0 + 2

    def boom(v):
        raise RuntimeError("peer lost")
    s.set_reduce(boom)
    with pytest.raises(F.FvmError):
        s.step(shared=True)
    s.set_reduce(None)
    s.set_halo(np.ones(m.ncell, bool))
    with pytest.raises(ValueError):
        s.set_halo(np.ones(3, bool))
