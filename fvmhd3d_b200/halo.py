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
  the local numbering (owned first, then halo, in global order), the local
  face list, and the per-peer send and receive lists.
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

    def __init__(self, mesh: Mesh, owner: np.ndarray, rank: int, depth: int = 2):
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
        self.cells = np.concatenate([owned, halo])          # local -> global
        self.local = np.full(mesh.ncell, -1, np.int64)      # global -> local
        self.local[self.cells] = np.arange(self.cells.size)
        self.nowned = owned.size
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
        a[self.nowned:] = 0
        return a
