"""Host-side cell records: the 72-byte layout of the reference's ``struct Cell``
(include/Cells.cuh:9-47), as a numpy dtype, plus helpers to build synthetic spheroids.

Field offsets: sign@0 (bool), mesh_idx@4, pos@8, force@20, oldforce@32, r@44, V@48, Vf@52,
Vcs@56, Vns@60, phase@64, cell_clock@68.
"""
from __future__ import annotations

import numpy as np

CELL_DTYPE = np.dtype(
    [
        ("sign", "u1"),
        ("_pad", "u1", (3,)),
        ("mesh_idx", "<i4"),
        ("pos", "<f4", (3,)),
        ("force", "<f4", (3,)),
        ("oldforce", "<f4", (3,)),
        ("r", "<f4"),
        ("V", "<f4"),
        ("Vf", "<f4"),
        ("Vcs", "<f4"),
        ("Vns", "<f4"),
        ("phase", "<i4"),
        ("cell_clock", "<f4"),
    ]
)
assert CELL_DTYPE.itemsize == 72

# V = r^3 / 0.23873241 keeps Cell::Radius_update (include/Cells.cuh:69-71) consistent with r.
RADIUS_COEF = 0.23873241
# Initial compartment split of include/Initialization.cuh:35-37 (Vf:Vns:Vcs = 1871:135:489).
_SPLIT = np.array([1871.0, 135.0, 489.0]) / (1871.0 + 135.0 + 489.0)


def empty_cells(n: int) -> np.ndarray:
    """n records with the reference's default member values (include/Cells.cuh:10-33)."""
    c = np.zeros(n, dtype=CELL_DTYPE)
    c["sign"] = 0
    c["mesh_idx"] = -1
    c["pos"] = -1.0
    c["r"] = -1.0
    c["V"] = -1.0
    c["Vf"] = -1.0
    c["Vcs"] = -1.0
    c["Vns"] = -1.0
    c["phase"] = -1
    c["cell_clock"] = 0.0
    return c


def live_cells(pos: np.ndarray, radii: np.ndarray, voxel_length: float, voxel_num: int,
               phase: np.ndarray | None = None, clock: np.ndarray | None = None) -> np.ndarray:
    """Quiescent live cells at `pos` (n,3) with radii `radii`; V from r, compartments split in
    the reference's initial ratio, mesh_idx of the voxel holding each cell."""
    n = len(pos)
    c = empty_cells(n)
    c["sign"] = 1
    c["pos"] = pos.astype(np.float32)
    c["force"] = 0.0
    c["oldforce"] = 0.0
    r = radii.astype(np.float32)
    c["r"] = r
    V = (r.astype(np.float64) ** 3 / RADIUS_COEF).astype(np.float32)
    c["V"] = V
    c["Vf"] = (V * _SPLIT[0]).astype(np.float32)
    c["Vns"] = (V * _SPLIT[1]).astype(np.float32)
    c["Vcs"] = (V * _SPLIT[2]).astype(np.float32)
    c["phase"] = 0 if phase is None else phase
    c["cell_clock"] = 0.0 if clock is None else clock
    ijk = (c["pos"] / np.float32(voxel_length)).astype(np.int32)
    c["mesh_idx"] = ijk[:, 0] + ijk[:, 1] * voxel_num + ijk[:, 2] * voxel_num * voxel_num
    return c


def _radii(rng: np.random.Generator, n: int) -> np.ndarray:
    return np.clip(rng.normal(5.0, 0.5, n), 4.0, 6.0)


def uniform_ball(n: int, radius: float, center: float, seed: int, voxel_length: float,
                 voxel_num: int) -> np.ndarray:
    """n cells uniform in a ball (rejection sampling from a Philox stream), radii N(5, 0.5)
    clipped to [4, 6] um.  The small plain-method workload: 10,000 cells, r = 150 um."""
    rng = np.random.Generator(np.random.Philox(seed))
    pts = np.empty((0, 3))
    while len(pts) < n:
        q = rng.uniform(-1.0, 1.0, size=(2 * n, 3))
        q = q[(q * q).sum(1) < 1.0]
        pts = np.concatenate([pts, q])
    pts = center + radius * pts[:n]
    return live_cells(pts, _radii(rng, n), voxel_length, voxel_num)


def lattice_spheroid(n: int, center: float, seed: int, voxel_length: float, voxel_num: int,
                     volume_fraction: float = 0.6, mean_radius: float = 5.0) -> np.ndarray:
    """The n sites of a cubic lattice closest to `center`, jittered by U(+-0.1 a), where the
    lattice spacing a = (4/3 pi r^3 / volume_fraction)^(1/3) packs cells of the mean radius at
    the given volume fraction.  The large plain-method workload: 10^6 cells, radius ~590 um."""
    rng = np.random.Generator(np.random.Philox(seed))
    a = (4.0 / 3.0 * np.pi * mean_radius ** 3 / volume_fraction) ** (1.0 / 3.0)
    m = int(np.ceil((3.0 * n / (4.0 * np.pi)) ** (1.0 / 3.0))) + 3
    g = np.arange(-m, m + 1, dtype=np.float64)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    d2 = X * X + Y * Y + Z * Z
    flat = np.argsort(d2.ravel(), kind="stable")[:n]
    pts = np.stack([X.ravel()[flat], Y.ravel()[flat], Z.ravel()[flat]], 1) * a
    pts += rng.uniform(-0.1 * a, 0.1 * a, size=pts.shape)
    pts += center
    return live_cells(pts, _radii(rng, n), voxel_length, voxel_num)


def seed_ki67_states(c: np.ndarray, seed: int) -> np.ndarray:
    """Spread cells over the Ki-67 phases so that a run of a few biology steps divides and
    removes cells (a population that starts all quiescent has almost no events for hundreds of
    minutes: the premitotic phase lasts 780 min).  Seeded draws (Philox): 60% quiescent, 15%
    premitotic with clocks U[0, 780), 10% postmitotic with clocks U[0, 150), 5% each apoptotic,
    early necrotic and late necrotic; a third of the dead cells have cytoplasm already below the
    removal threshold (Vcs 20 um^3)."""
    rng = np.random.Generator(np.random.Philox(seed))
    n = len(c)
    ph = rng.choice(np.array([0, 1, 2, 3, 4, 5], np.int32), n, p=[0.60, 0.15, 0.10, 0.05, 0.05, 0.05])
    clock = np.zeros(n, np.float32)
    clock[ph == 1] = rng.uniform(0.0, 780.0, int((ph == 1).sum())).astype(np.float32)
    clock[ph == 2] = rng.uniform(0.0, 150.0, int((ph == 2).sum())).astype(np.float32)
    c["phase"] = ph
    c["cell_clock"] = clock
    dead = np.flatnonzero(ph >= 3)
    low = dead[rng.random(len(dead)) < 1.0 / 3.0]
    c["Vcs"][low] = np.float32(20.0)
    return c
