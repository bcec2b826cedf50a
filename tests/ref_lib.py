"""ctypes access to the reference's own kernels, built from its unmodified sources by
`make -C oracle ref` into oracle/_ref/libgellref_<set>.so (see oracle/ref_harness.cu).

Test infrastructure only.  Each library is one parameter set of the reference (Voxel_num,
Voxel_length, Max_Cell_num and the substrate constants are compile-time there):
  default  N=100, 25 um voxels, 2M cells, oxygen     t32/t32d  N=32, 10 um, 65536 cells, oxygen/drug
  c1       N=100, 10 um, 2M cells, oxygen            c2/c2d    N=400, 10 um, 2M cells, oxygen/drug
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from gell_b200.cells import CELL_DTYPE

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")

P = ctypes.c_void_p
_libs: dict[str, ctypes.CDLL] = {}


def available(name: str) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libgellref_{name}.so"))


def lib(name: str) -> ctypes.CDLL:
    if name not in _libs:
        L = ctypes.CDLL(os.path.join(REF_DIR, f"libgellref_{name}.so"))
        L.gref_build_params.argtypes = [P, P]
        L.gref_create.argtypes = [ctypes.c_float] * 3
        L.gref_create.restype = P
        for f in ("gref_destroy", "gref_fm_update", "gref_prelod", "gref_birth", "gref_death", "gref_count"):
            getattr(L, f).argtypes = [P]
            getattr(L, f).restype = ctypes.c_int
        L.gref_set_cells.argtypes = [P, P, ctypes.c_int]
        L.gref_get_cells.argtypes = [P, P, ctypes.c_int]
        L.gref_get_keys.argtypes = [P, P, ctypes.c_int]
        L.gref_get_se.argtypes = [P, P, P]
        L.gref_lodsolver.argtypes = [P, ctypes.c_int]
        for f in ("gref_get_field", "gref_set_field", "gref_get_rate", "gref_set_rate"):
            getattr(L, f).argtypes = [P, P]
        L.gref_get_ef.argtypes = [P, P, P]
        L.gref_savecsv_cell.argtypes = [P, ctypes.c_int, ctypes.c_char_p]
        L.gref_init_sphere.argtypes = [ctypes.c_uint, ctypes.c_int, P]
        L.gref_savecsv_mesh.argtypes = [P, ctypes.c_char_p]
        L.gref_savecsv_meshslice.argtypes = [P, ctypes.c_char_p]
        L.gref_volume_update_device.argtypes = [P, ctypes.c_int]
        L.gref_volume_update_device.restype = ctypes.c_int
        for f in ("gref_time_fm", "gref_time_prelod", "gref_time_lod"):
            getattr(L, f).argtypes = [P, ctypes.c_int, ctypes.c_int]
            getattr(L, f).restype = ctypes.c_float
        _libs[name] = L
    return _libs[name]


class RefSim:
    """The reference's Mesh_struct, MechanicsMesh_struct, device_vector<Cell> and RNG states."""

    def __init__(self, name: str, conc: float, D: float, decay: float):
        self.L = lib(name)
        i4 = np.zeros(4, np.int32)
        f4 = np.zeros(4, np.float32)
        self.L.gref_build_params(i4.ctypes.data, f4.ctypes.data)
        self.N, self.cap = int(i4[0]), int(i4[1])
        self.length = float(f4[0])
        self.h = self.L.gref_create(conc, D, decay)
        if not self.h:
            raise RuntimeError("reference set-up failed")

    def close(self):
        if self.h:
            self.L.gref_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_cells(self, cells: np.ndarray):
        c = np.ascontiguousarray(cells, CELL_DTYPE)
        assert self.L.gref_set_cells(self.h, c.ctypes.data, len(c)) == 0

    def cells(self) -> np.ndarray:
        n = self.L.gref_count(self.h)
        out = np.zeros(max(n, 1), CELL_DTYPE)
        assert self.L.gref_get_cells(self.h, out.ctypes.data, n) == 0
        return out[:n]

    def count(self) -> int:
        return self.L.gref_count(self.h)

    def fm_update(self):
        assert self.L.gref_fm_update(self.h) == 0

    def keys(self) -> np.ndarray:
        n = self.count()
        out = np.zeros(max(n, 1), np.int32)
        assert self.L.gref_get_keys(self.h, out.ctypes.data, n) == 0
        return out[:n]

    def se(self):
        s = np.zeros(self.N ** 3, np.int32)
        e = np.zeros(self.N ** 3, np.int32)
        assert self.L.gref_get_se(self.h, s.ctypes.data, e.ctypes.data) == 0
        return s, e

    def prelod(self):
        assert self.L.gref_prelod(self.h) == 0

    def lodsolver(self, k: int):
        assert self.L.gref_lodsolver(self.h, k) == 0

    def field(self) -> np.ndarray:
        out = np.zeros(self.N ** 3, np.float32)
        assert self.L.gref_get_field(self.h, out.ctypes.data) == 0
        return out

    def set_field(self, f: np.ndarray):
        f = np.ascontiguousarray(f, np.float32)
        assert self.L.gref_set_field(self.h, f.ctypes.data) == 0

    def rate(self) -> np.ndarray:
        out = np.zeros(self.N ** 3, np.float32)
        assert self.L.gref_get_rate(self.h, out.ctypes.data) == 0
        return out

    def set_rate(self, r: np.ndarray):
        r = np.ascontiguousarray(r, np.float32)
        assert self.L.gref_set_rate(self.h, r.ctypes.data) == 0

    def ef(self):
        E = np.zeros(self.N, np.float32)
        Fv = np.zeros(self.N, np.float32)
        assert self.L.gref_get_ef(self.h, E.ctypes.data, Fv.ctypes.data) == 0
        return E, Fv

    def birth(self) -> int:
        return self.L.gref_birth(self.h)

    def death(self) -> int:
        return self.L.gref_death(self.h)

    def savecsv_mesh(self, path):
        assert self.L.gref_savecsv_mesh(self.h, os.fsencode(path)) == 0

    def savecsv_meshslice(self, path):
        assert self.L.gref_savecsv_meshslice(self.h, os.fsencode(path)) == 0

    def time_fm(self, warm, iters):
        return self.L.gref_time_fm(self.h, warm, iters)

    def time_prelod(self, warm, iters):
        return self.L.gref_time_prelod(self.h, warm, iters)

    def time_lod(self, warm, iters):
        return self.L.gref_time_lod(self.h, warm, iters)
