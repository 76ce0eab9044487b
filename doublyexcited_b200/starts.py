"""Seeded start vectors for GPLMR.

The reference builds its start vectors from a He+ block Lanczos run and a
product-orbital subspace diagonalisation (doublyexcited.F90:137-190) or reads
them from an eigenvector file.  Reproducible benchmarks and tests use seeded
complex-Gaussian blocks instead: entries (N(0,1) + i N(0,1))/sqrt(2) from
numpy's PCG64, exchange-symmetrised in (p,q) -- X <- (X + X^T)/sqrt(2) for
singlets, (X - X^T)/sqrt(2) for triplets -- and normalised per column.
"""
from __future__ import annotations

import math

import numpy as np


def seeded_start(m: int, nev: int, seed: int, spin: str = "singlet") -> np.ndarray:
    """(m*m, nev) complex128 block in the reference layout (Fortran order)."""
    if spin not in ("singlet", "triplet"):
        raise ValueError("spin must be 'singlet' or 'triplet'")
    rng = np.random.Generator(np.random.PCG64(seed))
    out = np.empty((m * m, nev), np.complex128, order="F")
    sgn = 1.0 if spin == "singlet" else -1.0
    for j in range(nev):
        z = (rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m))) / math.sqrt(2.0)
        z = (z + sgn * z.T) / math.sqrt(2.0)
        col = z.reshape(-1, order="F")
        out[:, j] = col / np.linalg.norm(col)
    return out
