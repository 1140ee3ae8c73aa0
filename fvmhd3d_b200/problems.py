"""Seeded synthetic initial conditions for the benchmark workloads.

Each generator returns primitive states ``W`` (ncell x 10, the reference's
``Fluid`` primitive order DENS, VELX, VELY, VELZ, ETHM, BX, BY, BZ, PSI, ENTR,
MPI/Fluid.h:21-32) for the generator positions of a mesh.  ``ETHM`` is the
thermal energy density P/(gamma-1) and ``ENTR`` the entropy function
(gamma-1) ETHM / rho^gamma (MPI/set_problem.cpp:127-131).

The reference ships no datasets; these stand in for its problem files
(``alfven.cpp``, ``blast.cpp``, ``MPI/set_problem.cpp`` Orszag-Tang) with the
shapes and sizes of the benchmark configurations.
"""
from __future__ import annotations

import numpy as np

NVAR = 10
DENS, VELX, VELY, VELZ, ETHM, BX, BY, BZ, PSI, ENTR = range(10)


def _finish(W: np.ndarray, pres: np.ndarray, gamma: float) -> np.ndarray:
    W[:, ETHM] = pres / (gamma - 1.0)
    W[:, PSI] = 0.0
    W[:, ENTR] = (gamma - 1.0) * W[:, ETHM] / W[:, DENS] ** gamma
    return W


def alfven(pos: np.ndarray, gamma: float = 5.0 / 3.0, amp: float = 0.1) -> np.ndarray:
    """Circularly polarised Alfven wave travelling along the (1,1,1) diagonal
    of the unit periodic cube: rho=1, P=0.1, B0=1 along the diagonal,
    transverse velocity and field of amplitude ``amp``.  The wave vector is
    2*pi*(1,1,1), the longest wavelength along the diagonal that is periodic
    in the unit cube (box diagonal / 3)."""
    n = pos.shape[0]
    e = np.ones(3) / np.sqrt(3.0)
    e1 = np.array([1.0, -1.0, 0.0]) / np.sqrt(2.0)
    e2 = np.cross(e, e1)
    phase = 2.0 * np.pi * (pos[:, 0] + pos[:, 1] + pos[:, 2])
    dv = amp * (np.outer(np.cos(phase), e1) + np.outer(np.sin(phase), e2))
    W = np.zeros((n, NVAR))
    W[:, DENS] = 1.0
    W[:, VELX:VELZ + 1] = dv
    W[:, BX:BZ + 1] = e[None, :] * 1.0 - dv  # dB = -sqrt(rho) dv: wave along +B0
    return _finish(W, np.full(n, 0.1), gamma)


def blast(pos: np.ndarray, gamma: float = 5.0 / 3.0, box: float = 1.0) -> np.ndarray:
    """MHD blast wave: rho=1, P=0.1 with P=100 inside r<0.1 of the box centre,
    uniform B=(1,1,0)/sqrt(2), at rest."""
    n = pos.shape[0]
    r = np.linalg.norm(pos - 0.5 * box, axis=1)
    W = np.zeros((n, NVAR))
    W[:, DENS] = 1.0
    W[:, BX] = 1.0 / np.sqrt(2.0)
    W[:, BY] = 1.0 / np.sqrt(2.0)
    pres = np.where(r < 0.1 * box, 100.0, 0.1)
    return _finish(W, pres, gamma)


def orszag_tang(pos: np.ndarray, gamma: float = 5.0 / 3.0) -> np.ndarray:
    """3D Orszag-Tang-type vortex in the unit periodic cube."""
    x, y, z = pos[:, 0], pos[:, 1], pos[:, 2]
    n = pos.shape[0]
    W = np.zeros((n, NVAR))
    W[:, DENS] = 25.0 / (36.0 * np.pi)
    W[:, VELX] = -np.sin(2 * np.pi * y)
    W[:, VELY] = np.sin(2 * np.pi * x)
    W[:, VELZ] = 0.1 * np.sin(2 * np.pi * z)
    b0 = 1.0 / np.sqrt(4.0 * np.pi)
    W[:, BX] = -b0 * np.sin(2 * np.pi * y)
    W[:, BY] = b0 * np.sin(4 * np.pi * x)
    return _finish(W, np.full(n, 5.0 / (12.0 * np.pi)), gamma)


def perturbed(W: np.ndarray, rel: float = 0.05, seed: int = 7) -> np.ndarray:
    """Seeded multiplicative noise on density/pressure and additive noise on
    velocity and field; used by parity tests to reach every solver branch."""
    rng = np.random.default_rng(seed)
    W = W.copy()
    n = W.shape[0]
    W[:, DENS] *= 1.0 + rel * rng.uniform(-1, 1, n)
    W[:, ETHM] *= 1.0 + rel * rng.uniform(-1, 1, n)
    W[:, VELX:VELZ + 1] += rel * rng.uniform(-1, 1, (n, 3))
    W[:, BX:BZ + 1] += rel * rng.uniform(-1, 1, (n, 3))
    return W


def disk_generators(n_total: int, seed: int = 3, box=(6.0, 6.0, 1.5), frac_bg: float = 0.125):
    """Generators of the Keplerian-disk workload in the periodic box
    [-box/2, box/2) centred on the disk: a fraction 1 - frac_bg sampled with
    surface density proportional to 1/r on 0.5 < r < 2 (so r is uniform) and
    a Gaussian vertical profile of scale height H = 0.1 r, the rest a
    jittered lattice padding the whole box.  Positions stay centred on the
    origin because the isothermal EOS depends on |x| (the mesh and the fluid
    path only use positions modulo the box)."""
    rng = np.random.default_rng(seed)
    box = np.asarray(box, dtype=np.float64)
    n_bg = int(round(n_total * frac_bg))
    # background lattice with the box's aspect ratio
    nz = max(2, int(round((n_bg * box[2] ** 2 / (box[0] * box[1])) ** (1.0 / 3.0))))
    nxy = max(2, int(round(np.sqrt(n_bg / nz))))
    n_bg = nxy * nxy * nz
    ix, iy, iz = np.meshgrid(np.arange(nxy), np.arange(nxy), np.arange(nz), indexing="ij")
    h = box / np.array([nxy, nxy, nz])
    bg = (np.stack([ix.ravel(), iy.ravel(), iz.ravel()], 1) + 0.5 + rng.uniform(-0.1, 0.1, (n_bg, 3))) * h - box / 2
    n_d = n_total - n_bg
    r = rng.uniform(0.5, 2.0, n_d)
    phi = rng.uniform(0.0, 2 * np.pi, n_d)
    z = np.clip(rng.normal(0.0, 0.1 * r), -0.45 * box[2], 0.45 * box[2])
    disk = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    pos = np.concatenate([disk, bg])
    return np.mod(pos + box / 2, box) - box / 2, box


def disk(pos: np.ndarray, box, GM: float = 1.0, cfac: float = 0.05, beta: float = 400.0,
         rho_bg: float = 1e-3, noise: float = 0.01, seed: int = 4, r_sink: float = 0.3):
    """Keplerian disk with a weak vertical field on generators from
    disk_generators: rho = max(Sigma(r)/(sqrt(2 pi) H) exp(-z^2/2H^2), rho_bg)
    with Sigma = 1/r, isothermal P = rho cs^2 with cs = cfac v_K(|x|),
    v = v_K azimuthal inside 0.5 < r < 2 plus `noise` relative random
    velocity, B_z with plasma beta = 2P/B^2.  Returns (W, bnd): cells
    with |x| < r_sink are DIOD boundary cells (the reference's inner sink,
    MPI/problems/mri_disk3d.cpp:762-765)."""
    rng = np.random.default_rng(seed)
    x = np.asarray(pos, dtype=np.float64)
    R = np.hypot(x[:, 0], x[:, 1])
    rr = np.linalg.norm(x, axis=1)
    H = 0.1 * np.maximum(R, 0.5)
    sigma = np.where((R > 0.5) & (R < 2.0), 1.0 / np.maximum(R, 1e-3), 0.0)
    rho = np.maximum(sigma / (np.sqrt(2 * np.pi) * H) * np.exp(-0.5 * (x[:, 2] / H) ** 2), rho_bg)
    cs2 = GM / np.maximum(rr, 1e-3) * cfac ** 2
    pres = rho * cs2
    vk = np.sqrt(GM / np.maximum(R, 0.3))
    inside = (R > 0.5) & (R < 2.0)
    n = x.shape[0]
    W = np.zeros((n, NVAR))
    W[:, DENS] = rho
    W[:, VELX] = np.where(inside, -vk * x[:, 1] / np.maximum(R, 1e-9), 0.0)
    W[:, VELY] = np.where(inside, vk * x[:, 0] / np.maximum(R, 1e-9), 0.0)
    W[:, VELX:VELZ + 1] += noise * vk[:, None] * rng.uniform(-1, 1, (n, 3))
    W[:, ETHM] = pres          # isothermal: ETHM = P (MPI/problems/mri_disk3d.cpp:377-380)
    W[:, BZ] = np.sqrt(2.0 * pres / beta)
    W[:, PSI] = 0.0
    W[:, ENTR] = 1.0
    bnd = np.where(rr < r_sink, 3, 0).astype(np.int32)  # DIOD
    return W, bnd
