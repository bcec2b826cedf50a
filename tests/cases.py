"""Seeded test populations for the parity tests (small grids the oracle finishes in seconds)."""
from __future__ import annotations

import numpy as np

from gell_b200.cells import CELL_DTYPE, live_cells, uniform_ball


def ball_cells(N: int, length: float, n: int, seed: int, radius_frac: float = 0.35,
               dead_frac: float = 0.05, outside: int = 8, phases: bool = False) -> np.ndarray:
    """n cells uniform in a ball at the grid centre, with a few dead cells (sign = 0) and a few
    cells outside the grid (negative, beyond the far face, and in (-len, 0), which the reference's
    truncating bin lookup puts in bin 0)."""
    rng = np.random.Generator(np.random.Philox(seed + 1))
    L = N * length
    c = uniform_ball(n, radius_frac * L, L / 2, seed, length, N)
    c["oldforce"] = rng.normal(0, 0.5, (n, 3)).astype(np.float32)
    dead = rng.random(n) < dead_frac
    c["sign"][dead] = 0
    if phases:
        c["phase"] = rng.choice([0, 0, 0, 1, 2, 3, 4, 5], n)
        c["cell_clock"] = rng.choice(np.array([0, 6, 150, 774, 780], np.float32), n)
    k = min(outside, n)
    idx = rng.choice(n, k, replace=False)
    bad = np.array([[-3.0, L / 2, L / 2], [L + 2.0, L / 2, L / 2], [L / 2, -0.5 * length, L / 2],
                    [L / 2, L / 2, L - 1e-3], [-length - 1.0, 1.0, 1.0], [L / 2, L * 2, 0.0],
                    [0.0, 0.0, 0.0], [L - 0.01, L - 0.01, L - 0.01]], np.float32)
    c["pos"][idx] = bad[:k]
    return c


def one_per_voxel(N: int, length: float, seed: int, lo: int, hi: int) -> np.ndarray:
    """One cell at the centre of every voxel of the cube [lo, hi)^3: each voxel's uptake is a
    single term, so the uptake map does not depend on summation order."""
    rng = np.random.Generator(np.random.Philox(seed))
    g = np.arange(lo, hi)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    pos = (np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1) + 0.5) * length
    c = live_cells(pos, rng.uniform(4, 6, len(pos)), length, N)
    c["phase"] = rng.choice([-1, 0, 1, 2, 3, 4, 5], len(c))
    return c


def random_field(N: int, seed: int, lo: float = 5.0, hi: float = 40.0) -> np.ndarray:
    rng = np.random.Generator(np.random.Philox(seed))
    return rng.uniform(lo, hi, N ** 3).astype(np.float32)


def canonical(cells: np.ndarray) -> np.ndarray:
    """Cells sorted by the bytes of their records (for comparing sets appended in any order)."""
    raw = np.ascontiguousarray(cells).view(np.uint8).reshape(len(cells), CELL_DTYPE.itemsize)
    order = np.lexsort(raw.T[::-1])
    return cells[order]
