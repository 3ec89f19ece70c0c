"""Seeded synthetic particle lattices for tests and benchmarks.

The reference publishes no benchmark dataset; its workloads are N-body particle
lattices.  ``zeldovich`` builds one: a Lagrangian lattice ``q = (idx + 1/2) L/n``
displaced by the Zel'dovich field of a Gaussian random density with
``P(k) ~ k^-2``, scaled to a stated rms displacement in lattice cells, wrapped
into the periodic box ``[0, L)^3``.  Velocities are ``10 psi`` rounded through
float32 (the workload's stated velocity precision) and returned as float64.
"""
from __future__ import annotations

import numpy as np


def zeldovich(n: int, rms_cells: float, seed: int, box: float = 100.0, wrap: bool = True):
    """Return ``pos, vel`` as float64 arrays of shape (n, n, n, 3); with
    ``wrap=False`` the positions are left unwrapped (an open lattice)."""
    rng = np.random.default_rng(seed)
    white = rng.standard_normal((n, n, n))
    wk = np.fft.rfftn(white)
    kx = np.fft.fftfreq(n) * n
    kz = np.fft.rfftfreq(n) * n
    KX, KY, KZ = np.meshgrid(kx, kx, kz, indexing="ij")
    k2 = KX * KX + KY * KY + KZ * KZ
    k2[0, 0, 0] = 1.0
    delta = wk / np.sqrt(k2)  # amplitude sqrt(P(k)) with P ~ k^-2
    delta[0, 0, 0] = 0.0
    psi = np.empty((n, n, n, 3))
    for a, K in enumerate((KX, KY, KZ)):
        psi[..., a] = np.fft.irfftn(1j * K * delta / k2, s=(n, n, n), axes=(0, 1, 2))
    rms = np.sqrt(np.mean(np.sum(psi * psi, axis=-1)))
    if rms > 0:
        psi *= rms_cells * (box / n) / rms
    idx = (np.arange(n) + 0.5) * (box / n)
    q = np.stack(np.meshgrid(idx, idx, idx, indexing="ij"), axis=-1)
    pos = np.mod(q + psi, box) if wrap else q + psi
    vel = (10.0 * psi).astype(np.float32).astype(np.float64)
    return np.ascontiguousarray(pos), np.ascontiguousarray(vel)


def lattice(n: int, box: float = 100.0):
    """The undisplaced lattice (every particle at a cell centre)."""
    idx = (np.arange(n) + 0.5) * (box / n)
    return np.ascontiguousarray(np.stack(np.meshgrid(idx, idx, idx, indexing="ij"), axis=-1))
