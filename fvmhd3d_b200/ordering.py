"""Space-filling-curve ordering of the local cells, the equivalent of the
reference's ``system::sort_local_data`` (MPI/sort_local_data.cpp:17-55),
which sorts the local particles and their U, dU and Wrec rows by
Peano-Hilbert key every time the data are redistributed
(MPI/distribute_data.cpp:236).

Cells that are close in space then sit close in memory, so the neighbour
gathers of the limiter, the reconstruction and the face kernels hit L2 rather
than HBM.  The key is the Hilbert index of the position quantised to
``bits`` bits per axis on the box's longest side, computed with Skilling's
transpose algorithm (J. Skilling, "Programming the Hilbert curve", AIP Conf.
Proc. 707, 381 (2004)).  The curve's orientation need not match the
reference's tables: the order only changes memory locality and the order in
which adjust_timesteps visits sites, and the oracle is always run on the same
ordered input.
"""
from __future__ import annotations

import numpy as np

BITS_PER_DIMENSION = 21  # 3 x 21 = 63 bits of key


def hilbert_keys(cells: np.ndarray, bits: int = BITS_PER_DIMENSION) -> np.ndarray:
    """Hilbert index (uint64) of integer cell coordinates (n x 3, each in
    [0, 2^bits))."""
    if not 1 <= bits <= BITS_PER_DIMENSION:
        raise ValueError(f"bits must be in [1, {BITS_PER_DIMENSION}]")
    X = [np.asarray(cells[:, i], dtype=np.uint64).copy() for i in range(3)]
    one = np.uint64(1)
    # inverse undo of the excess work (axes -> transposed Hilbert index)
    q = one << np.uint64(bits - 1)
    while q > one:
        p = q - one
        for i in range(3):
            hit = (X[i] & q) != 0
            # bit set: invert the low bits of X[0]; clear: exchange them with X[i]
            t = np.where(hit, np.uint64(0), (X[0] ^ X[i]) & p)
            X[0] = np.where(hit, X[0] ^ p, X[0] ^ t)
            if i:
                X[i] = X[i] ^ t
        q >>= one
    # Gray encode
    for i in range(1, 3):
        X[i] ^= X[i - 1]
    t = np.zeros_like(X[0])
    q = one << np.uint64(bits - 1)
    while q > one:
        t = np.where((X[2] & q) != 0, t ^ (q - one), t)
        q >>= one
    for i in range(3):
        X[i] ^= t
    # interleave: the most significant bit of X[0], X[1], X[2], then the next
    key = np.zeros_like(X[0])
    for b in range(bits - 1, -1, -1):
        for i in range(3):
            key = (key << one) | ((X[i] >> np.uint64(b)) & one)
    return key


def sort_local_data(pos, box, bits: int = BITS_PER_DIMENSION) -> np.ndarray:
    """Permutation that orders the cells at `pos` (n x 3) along the Hilbert
    curve over the box (a scalar or three side lengths; positions are taken
    modulo the box).  Apply it to the generators and every per-cell array
    (``pos[order]``, ``W[order]``, ``bnd[order]``) before building the mesh,
    as the reference reorders ptcl_local, U_local, dU_local and Wrec_local."""
    pos = np.asarray(pos, dtype=np.float64)
    if pos.ndim != 2 or pos.shape[1] != 3:
        raise ValueError("pos must be n x 3")
    box = np.broadcast_to(np.asarray(box, dtype=np.float64), (3,))
    lo = pos.min(axis=0) if pos.size else np.zeros(3)
    # cubic cells on the longest side, as the reference scales by the domain's
    # largest extent
    size = float(box.max())
    scale = float(1 << bits) / size
    x = np.mod(pos - lo, box)
    c = np.clip(np.floor(x * scale), 0, (1 << bits) - 1).astype(np.uint64)
    return np.argsort(hilbert_keys(c, bits), kind="stable")
