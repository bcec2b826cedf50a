"""Generate tests/golden/host_ref.npz from the reference's own host-callable functions.

The reference's Morton code, bin lookup and Cell model are `__host__ __device__` functions
(include/BasicFunctions.cuh:60-66,111-137, include/Cells.cuh:69-223).  oracle/ref_harness.cu
compiles them from the unmodified reference headers (oracle/Makefile target `ref`); this script
calls them on the CPU over a seeded grid of inputs and stores inputs and outputs, so the CPU test
suite can pin the oracle against the reference without the reference present.

Run from the repository root after `make -C oracle ref`:  python tests/golden/make_golden_host.py
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from gell_b200.cells import CELL_DTYPE  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "host_ref.npz")


def load(name: str) -> ctypes.CDLL:
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", f"libgellref_{name}.so"))
    P = ctypes.c_void_p
    lib.gref_morton.argtypes = [ctypes.c_int] * 3
    lib.gref_morton.restype = ctypes.c_int
    lib.gref_find_mesh.argtypes = [P, P]
    lib.gref_inside.argtypes = [ctypes.c_int] * 3
    lib.gref_o2_consume.argtypes = [P]
    lib.gref_o2_consume.restype = ctypes.c_float
    lib.gref_volume_update.argtypes = [P]
    lib.gref_phase_update.argtypes = [P, ctypes.c_float, ctypes.c_float]
    lib.gref_phase_update.restype = ctypes.c_int
    lib.gref_radius_update.argtypes = [P]
    lib.gref_build_params.argtypes = [P, P]
    return lib


def params(lib) -> tuple[np.ndarray, np.ndarray]:
    i4 = np.zeros(4, np.int32)
    f4 = np.zeros(4, np.float32)
    lib.gref_build_params(i4.ctypes.data, f4.ctypes.data)
    return i4, f4


def cell_grid(rng: np.random.Generator, n: int) -> np.ndarray:
    c = np.zeros(n, CELL_DTYPE)
    c["sign"] = 1
    c["mesh_idx"] = -1
    c["phase"] = rng.integers(-1, 6, n)
    V = rng.uniform(800.0, 6000.0, n).astype(np.float32)
    # include the thresholds the model tests: V >= 2*Default_V, Vcs <= 24.4
    V[:50] = np.float32(4988.0)
    c["V"] = V
    c["Vf"] = (V * rng.uniform(0.0, 0.9, n)).astype(np.float32)
    c["Vns"] = (V * rng.uniform(0.0, 0.1, n)).astype(np.float32)
    c["Vcs"] = (V * rng.uniform(0.0, 0.3, n)).astype(np.float32)
    c["Vcs"][50:100] = np.float32(24.4)
    c["r"] = rng.uniform(4.0, 8.0, n).astype(np.float32)
    clocks = np.array([0, 6, 144, 150, 774, 780, 786, 1000], np.float32)
    c["cell_clock"] = rng.choice(clocks, n)
    c["pos"] = rng.uniform(0, 1000, (n, 3)).astype(np.float32)
    return c


def main() -> None:
    rng = np.random.Generator(np.random.Philox(2024))
    ref25 = load("default")   # Voxel_length 25, Voxel_num 100
    ref10 = load("t32")       # Voxel_length 10, Voxel_num 32
    out: dict[str, np.ndarray] = {}
    for tag, lib in (("l25", ref25), ("l10", ref10)):
        i4, f4 = params(lib)
        out[f"{tag}_params_i"] = i4
        out[f"{tag}_params_f"] = f4

    # Morton codes: corners, edges and a random sample of the 10-bit cube
    ijk = np.concatenate([
        np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1023, 1023, 1023], [511, 512, 513]]),
        rng.integers(0, 1024, (20000, 3)),
        rng.integers(0, 64, (2000, 3)),
    ]).astype(np.int32)
    out["morton_ijk"] = ijk
    out["morton"] = np.array([ref25.gref_morton(int(a), int(b), int(c)) for a, b, c in ijk], np.int32)

    # Find_Mesh / Check_Inside for both voxel lengths, including negative positions that the
    # truncating conversion maps to bin 0
    pos = np.concatenate([
        rng.uniform(-30.0, 2600.0, (5000, 3)),
        np.array([[-0.5, -24.9, 0.0], [25.0, 50.0, 2475.0], [2499.99, 2500.0, 1e-7], [-25.0, 10.0, 9.99]]),
        (rng.integers(0, 101, (500, 3)) * 25.0),
        (rng.integers(0, 101, (500, 3)) * 10.0),
    ]).astype(np.float32)
    out["mesh_pos"] = pos
    for tag, lib in (("l25", ref25), ("l10", ref10)):
        res = np.zeros((len(pos), 3), np.int32)
        ins = np.zeros(len(pos), np.int32)
        for n in range(len(pos)):
            p = np.ascontiguousarray(pos[n])
            o = np.zeros(3, np.int32)
            lib.gref_find_mesh(p.ctypes.data, o.ctypes.data)
            res[n] = o
            ins[n] = lib.gref_inside(int(o[0]), int(o[1]), int(o[2]))
        out[f"mesh_ijk_{tag}"] = res
        out[f"mesh_inside_{tag}"] = ins

    # Cell model: O2_consume, Volume_update, Phase_update_ki67adv, Radius_update
    cells = cell_grid(rng, 6000)
    out["model_in"] = cells.view(np.uint8).reshape(len(cells), 72)
    for tag, lib in (("l25", ref25), ("l10", ref10)):
        out[f"o2_consume_{tag}"] = np.array(
            [lib.gref_o2_consume(cells[n:n + 1].ctypes.data) for n in range(len(cells))], np.float32)
    vol = cells.copy()
    for n in range(len(vol)):
        lib_c = vol[n:n + 1]
        ref25.gref_volume_update(lib_c.ctypes.data)
    out["volume_out"] = vol.view(np.uint8).reshape(len(vol), 72)

    rnd = rng.choice(np.array([1e-7, 1e-4, 5e-4, 1e-3, 1.2e-3, 2e-3, 0.01, 0.5, 1.0], np.float32), len(cells))
    o2 = rng.choice(np.array([0.0, 2.4, 2.5, 3.0, 4.9, 5.0, 5.1, 7.5, 9.9, 10.0, 10.1, 38.0], np.float32),
                    len(cells))
    rnd[:2000] = rng.uniform(0, 0.004, 2000).astype(np.float32)
    o2[:2000] = rng.uniform(0, 12, 2000).astype(np.float32)
    ph = cells.copy()
    ret = np.zeros(len(ph), np.int32)
    for n in range(len(ph)):
        ret[n] = ref25.gref_phase_update(ph[n:n + 1].ctypes.data, float(rnd[n]), float(o2[n]))
    out["phase_rand"] = rnd
    out["phase_o2"] = o2
    out["phase_out"] = ph.view(np.uint8).reshape(len(ph), 72)
    out["phase_ret"] = ret

    rad = cells.copy()
    for n in range(len(rad)):
        ref25.gref_radius_update(rad[n:n + 1].ctypes.data)
    out["radius_out"] = rad["r"].copy()

    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
