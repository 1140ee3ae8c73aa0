"""Domain decomposition and halo exchange for running one mesh on several
GPUs (the equivalent of the reference's distribute_particle_fluid_data /
collect_results, MPI/distribute_work.cpp:367-724).

Host logic over ``torch.distributed``: NCCL between GPUs (device tensors),
gloo on the CPU.  No multicast is used.

* :func:`partition` splits the cells into equal slabs along the longest box
  axis (the reference decomposes with a Peano-Hilbert domain tree; slabs keep
  the plan simple and balanced for the lattice workloads).
* :class:`HaloPlan` is one rank's view: its owned cells, `depth` rings of
  neighbour cells around them (the limiter of a ring-1 cell needs ring 2),
  the local numbering (owned first, then halo, in global order; or every
  local cell in global order), the local face list, and the per-peer send
  and receive lists.
* :class:`Domain` steps one rank's cells on its own system and exchanges
  the neighbour rows after each step.
* :meth:`HaloPlan.exchange` fills the halo rows of per-cell arrays from their
  owners (distribute_particle_fluid_data); :meth:`HaloPlan.collect` sends
  halo contributions back and adds them into the owners' rows
  (collect_results).
"""
from __future__ import annotations

import numpy as np

from .mesh import Mesh


def partition(pos, box, nranks: int) -> np.ndarray:
    """Owner rank of every cell: equal-count slabs along the longest axis."""
    pos = np.asarray(pos, np.float64)
    box = np.broadcast_to(np.asarray(box, np.float64), (3,))
    axis = int(np.argmax(box))
    order = np.argsort(pos[:, axis], kind="stable")
    owner = np.empty(pos.shape[0], np.int32)
    for r, chunk in enumerate(np.array_split(order, nranks)):
        owner[chunk] = r
    return owner


def _neighbours(mesh: Mesh):
    """CSR neighbour lists (from the cells' face lists)."""
    off = mesh.cell_face_off
    ids = mesh.cell_face_ids
    cells = np.repeat(np.arange(mesh.ncell), np.diff(off))
    s1, s2 = mesh.s1[ids], mesh.s2[ids]
    nb = np.where(s1 == cells, s2, s1)
    return off, nb


class HaloPlan:
    """Rank `rank`'s cells, halo rings and exchange lists."""

    def __init__(self, mesh: Mesh, owner: np.ndarray, rank: int, depth: int = 2, owned_first: bool = True):
        owner = np.asarray(owner, np.int32)
        self.rank = rank
        self.nranks = int(owner.max()) + 1
        off, nb = _neighbours(mesh)
        owned = np.nonzero(owner == rank)[0]
        inside = np.zeros(mesh.ncell, bool)
        inside[owned] = True
        ring = owned
        for _ in range(depth):
            cand = np.unique(np.concatenate([nb[off[c]:off[c + 1]] for c in ring])) if ring.size else ring
            ring = cand[~inside[cand]]
            inside[ring] = True
        halo = np.nonzero(inside & (owner != rank))[0]
        self.owned = owned
        self.halo = halo
        # local -> global: owned cells first, or every cell in global order
        self.cells = np.concatenate([owned, halo]) if owned_first else np.sort(np.concatenate([owned, halo]))
        self.local = np.full(mesh.ncell, -1, np.int64)      # global -> local
        self.local[self.cells] = np.arange(self.cells.size)
        self.nowned = owned.size
        self.is_halo = owner[self.cells] != rank             # per local cell
        # receive lists: my halo cells grouped by owner (in global order)
        self.recv = {s: halo[owner[halo] == s] for s in range(self.nranks) if s != rank}
        # send lists: my owned cells in each peer's halo, computed the same way
        # the peer computes its own halo
        self.send = {}
        for s in range(self.nranks):
            if s == rank:
                continue
            peer_inside = np.zeros(mesh.ncell, bool)
            peer_owned = np.nonzero(owner == s)[0]
            peer_inside[peer_owned] = True
            ring = peer_owned
            for _ in range(depth):
                cand = np.unique(np.concatenate([nb[off[c]:off[c + 1]] for c in ring])) if ring.size else ring
                ring = cand[~peer_inside[cand]]
                peer_inside[ring] = True
            self.send[s] = np.nonzero(peer_inside & (owner == rank))[0]
        # local faces: both sides in the local set
        keep = (self.local[mesh.s1] >= 0) & (self.local[mesh.s2] >= 0)
        self.faces = np.nonzero(keep)[0]

    # ---- exchange -----------------------------------------------------
    def _alltoall(self, send_rows, recv_counts, width, dtype, device, group):
        import torch
        import torch.distributed as dist
        peers = [s for s in range(self.nranks)]
        send_counts = [send_rows[s].shape[0] * width if s != self.rank else 0 for s in peers]
        rc = [recv_counts[s] * width if s != self.rank else 0 for s in peers]
        parts = [torch.as_tensor(np.ascontiguousarray(send_rows[s]).ravel(), device=device)
                 if s != self.rank else torch.empty(0, dtype=dtype, device=device) for s in peers]
        send = torch.cat(parts) if parts else torch.empty(0, dtype=dtype, device=device)
        recv = torch.empty(sum(rc), dtype=dtype, device=device)
        dist.all_to_all_single(recv, send, output_split_sizes=rc, input_split_sizes=send_counts, group=group)
        out, o = {}, 0
        for s in peers:
            out[s] = recv[o:o + rc[s]]
            o += rc[s]
        return out

    def exchange(self, local_rows, group=None, device="cpu"):
        """Fill the halo rows of `local_rows` (n_local x k, local numbering)
        from the owners' owned rows; returns the updated array."""
        import torch
        a = np.array(local_rows, copy=True)
        width = int(np.prod(a.shape[1:])) if a.ndim > 1 else 1
        rows = {s: a[self.local[self.send[s]]].reshape(-1, width) for s in self.send}
        counts = {s: self.recv[s].size for s in self.recv}
        tdt = torch.from_numpy(a[:0]).dtype
        got = self._alltoall(rows, counts, width, tdt, device, group)
        for s, idx in self.recv.items():
            if idx.size:
                a[self.local[idx]] = got[s].cpu().numpy().reshape((idx.size,) + a.shape[1:])
        return a

    def collect(self, local_rows, group=None, device="cpu"):
        """Add the halo rows' contributions into their owners' rows (the
        reverse exchange); halo rows are zeroed.  Returns the updated array."""
        import torch
        a = np.array(local_rows, copy=True)
        width = int(np.prod(a.shape[1:])) if a.ndim > 1 else 1
        rows = {s: a[self.local[self.recv[s]]].reshape(-1, width) for s in self.recv}
        counts = {s: self.send[s].size for s in self.send}
        tdt = torch.from_numpy(a[:0]).dtype
        got = self._alltoall(rows, counts, width, tdt, device, group)
        for s, idx in self.send.items():
            if idx.size:
                np.add.at(a, self.local[idx], got[s].cpu().numpy().reshape((idx.size,) + a.shape[1:]))
        a[self.is_halo] = 0
        return a


# ---- one rank's domain -------------------------------------------------------

STATE_KEYS = ("vel", "tlast", "tend", "rung", "U", "dU", "wrec")


def local_mesh(mesh: Mesh, plan: HaloPlan) -> Mesh:
    """The rank's mesh: its cells (`plan.cells`, local numbering) and the
    faces between them, in the whole mesh's face order.  Each cell lists its
    local faces in the order the whole mesh lists them, so an owned cell
    (every face local) adds its face sums in the same order: the same bits.
    A plan numbered in global order also keeps the order in which a walk
    over the cells meets the faces (the reference's active-face list,
    MPI/iterate.cpp:58-113, and the face loops that scatter along it)."""
    cells, f = plan.cells, plan.faces
    fmap = np.full(mesh.nface, -1, np.int64)
    fmap[f] = np.arange(f.size)
    off = np.asarray(mesh.cell_face_off, np.int64)
    starts, lens = off[cells], off[cells + 1] - off[cells]
    first = np.concatenate([[0], np.cumsum(lens)[:-1]])
    at = np.repeat(starts - first, lens) + np.arange(int(lens.sum()))
    lf = fmap[np.asarray(mesh.cell_face_ids)[at]]
    keep = lf >= 0
    counts = np.bincount(np.repeat(np.arange(cells.size), lens)[keep], minlength=cells.size)
    loc = plan.local
    return Mesh(np.asarray(mesh.box), np.ascontiguousarray(mesh.pos[cells]),
                loc[mesh.s1[f]].astype(np.int32), loc[mesh.s2[f]].astype(np.int32),
                np.ascontiguousarray(mesh.n[f]), np.ascontiguousarray(mesh.centroid[f]),
                np.ascontiguousarray(mesh.volume[cells]), np.ascontiguousarray(mesh.cell_centroid[cells]),
                np.concatenate([[0], np.cumsum(counts)]).astype(np.int64), lf[keep].astype(np.int32))


def _ticks(s) -> int:
    """The system clock (Scheduler::tsysU) of a system object."""
    return int(s.tsys_ticks) if hasattr(s, "tsys_ticks") else int(s.clock()[0])


class Domain:
    """One rank's part of a run on a partitioned mesh (iterate_step across
    ranks, MPI/iterate.cpp:115-247): its owned cells plus `depth` rings of
    neighbour copies as the mesh of its own system, numbered in global
    order, the state the host keeps, and after each step the copy of the
    neighbour rows from their owners (`HaloPlan.exchange`).

    Steps are global (shared timestep): every rank takes the minimum over
    ranks of its owned cells' timesteps through the system's reduction
    (fvm_set_reduce), so all ranks step with the one dt of the whole mesh.

    Depth: a pass that reads neighbours leaves the outermost ring of copies
    wrong.  Within a step the slope limiter, the corrector flux, the
    timestep, the predictor flux and the reconstruction's gradient read
    neighbours; the corrected state is right on rings 0 .. depth-2, the
    predicted state and the reconstruction on rings 0 .. depth-3, so three
    rings keep every owned cell exact until the exchange refreshes the
    copies.

    `make_system(mesh)` returns a system with the mesh installed (a
    :class:`~fvmhd3d_b200.system.System`, or any object with its
    init_problem / set_state / step / get_state methods and its clock)."""

    def __init__(self, mesh: Mesh, owner, rank: int, make_system, group=None, depth: int = 3, device="cpu"):
        self.plan = HaloPlan(mesh, owner, rank, depth=depth, owned_first=False)
        self.mesh = local_mesh(mesh, self.plan)
        self.group, self.device = group, device
        self.sys = make_system(self.mesh)
        self.state = None
        self.ticks = 0

    @property
    def nowned(self) -> int:
        return self.plan.nowned

    def _min(self, v: float) -> float:
        import torch
        import torch.distributed as dist
        t = torch.tensor([v], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
        return float(t[0])

    def init_problem(self, W, bnd=None, rung_offset=0) -> None:
        """The initial state of the rank's cells from the whole mesh's
        primitives W (and boundary codes)."""
        cells = self.plan.cells
        s = self.sys
        if hasattr(s, "set_halo"):
            s.set_halo(self.plan.is_halo)
            s.set_reduce(self._min)
        s.init_problem(np.ascontiguousarray(np.asarray(W)[cells]), bnd=None if bnd is None else np.asarray(bnd)[cells],
                       rung_offset=rung_offset)
        st = s.get_state()
        self.state = {k: np.ascontiguousarray(st[k]) for k in STATE_KEYS}
        self.ticks = _ticks(s)

    def step(self) -> int:
        """One global step on every rank, then the exchange of the neighbour
        rows.  Returns the rank's owned cell count (every cell steps)."""
        s, h = self.sys, self.state
        if hasattr(s, "step_host"):
            s.step_host(h, shared=True, tsys_ticks=self.ticks)
        else:
            s.set_state(tsys_ticks=self.ticks, **h)
            s.step(shared=True)
            st = s.get_state()
            for k in STATE_KEYS:
                h[k] = np.ascontiguousarray(np.asarray(st[k]).reshape(h[k].shape), h[k].dtype)
        self.ticks = _ticks(s)
        for k in STATE_KEYS:
            h[k] = np.ascontiguousarray(self.plan.exchange(h[k], self.group, self.device))
        return self.nowned

    def owned_state(self):
        """The owned cells' global indices and their state rows."""
        own = ~self.plan.is_halo
        return self.plan.cells[own], {k: v[own].copy() for k, v in self.state.items()}
