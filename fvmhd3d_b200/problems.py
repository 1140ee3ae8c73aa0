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
