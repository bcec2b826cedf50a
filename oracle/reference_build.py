"""ctypes access to the reference's own kernels, built from its unmodified sources by
`make -C oracle ref` into oracle/_ref/libgellref_<set>.so (see oracle/ref_harness.cu).

Test infrastructure only: loaded by the tests and by bench.py's reference arm, never by the
gell_b200 package.  Each library is one parameter set of the reference (Voxel_num, Voxel_length,
Max_Cell_num and the substrate constants are compile-time there):
  default  N=100, 25 um voxels, 2M cells, oxygen     t32/t32d  N=32, 10 um, 65536 cells, oxygen/drug
  c1       N=100, 10 um, 2M cells, oxygen            c2/c2d    N=400, 10 um, 2M cells, oxygen/drug
  c3/c3d   N=600, 10 um, 4M cells, oxygen/drug       c5        N=256, 10 um, 400k cells, oxygen
"""
from __future__ import annotations

import contextlib
import ctypes
import os
import sys

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
        L.gref_cells_ptr.argtypes = [P]
        L.gref_cells_ptr.restype = P
        L.gref_prelod_ptr.argtypes = [P, P, ctypes.c_int]
        L.gref_prelod_ptr.restype = ctypes.c_int
        L.gref_event_create.restype = P
        L.gref_event_record.argtypes = [P]
        L.gref_event_record.restype = ctypes.c_int
        L.gref_event_elapsed_ms.argtypes = [P, P]
        L.gref_event_elapsed_ms.restype = ctypes.c_float
        L.gref_event_destroy.argtypes = [P]
        L.gref_sync.restype = ctypes.c_int
        L.gref_host_alloc.argtypes = [ctypes.c_size_t]
        L.gref_host_alloc.restype = P
        L.gref_host_free.argtypes = [P]
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
        with quiet_stdout():
            self.h = self.L.gref_create(conc, D, decay)
        if not self.h:
            raise RuntimeError("reference set-up failed")

    def close(self):
        if self.h:
            with quiet_stdout():
                self.L.gref_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_cells(self, cells: np.ndarray):
        c = np.ascontiguousarray(cells, CELL_DTYPE)
        assert self.L.gref_set_cells(self.h, c.ctypes.data, len(c)) == 0

    def get_cells_into(self, out: np.ndarray):
        """Copy the current cells into `out` (len == count), e.g. a pinned host buffer."""
        assert out.dtype == CELL_DTYPE and out.flags.c_contiguous and len(out) == self.count()
        assert self.L.gref_get_cells(self.h, out.ctypes.data, len(out)) == 0

    def cells_ptr(self) -> int:
        return self.L.gref_cells_ptr(self.h)

    def prelod_on(self, other: "RefSim"):
        """PreLOD of this build's substrate on the cells of `other` (same device)."""
        assert self.L.gref_prelod_ptr(self.h, other.cells_ptr(), other.count()) == 0

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


class RefEvent:
    """A CUDA event on the legacy default stream, recorded through a reference build."""

    def __init__(self, name: str):
        self.L = lib(name)
        self.e = self.L.gref_event_create()
        if not self.e:
            raise RuntimeError("cudaEventCreate failed")

    def record(self):
        assert self.L.gref_event_record(self.e) == 0

    def elapsed_ms(self, end: "RefEvent") -> float:
        ms = self.L.gref_event_elapsed_ms(self.e, end.e)
        assert ms >= 0.0
        return float(ms)

    def close(self):
        if self.e:
            self.L.gref_event_destroy(self.e)
            self.e = None


class PinnedCells:
    """`n` cell records in page-locked host memory (cudaMallocHost through a reference build)."""

    def __init__(self, name: str, n: int):
        self.L = lib(name)
        self.p = self.L.gref_host_alloc(n * CELL_DTYPE.itemsize)
        if not self.p:
            raise RuntimeError("cudaMallocHost failed")
        buf = (ctypes.c_uint8 * (n * CELL_DTYPE.itemsize)).from_address(self.p)
        self.cells = np.frombuffer(buf, dtype=CELL_DTYPE, count=n)

    def close(self):
        if self.p:
            self.cells = None
            self.L.gref_host_free(self.p)
            self.p = None


@contextlib.contextmanager
def quiet_stdout():
    """Send what the reference prints on stdout (its constructors report allocations) to stderr,
    so that a caller's own stdout stays clean."""
    libc = ctypes.CDLL(None)
    sys.stdout.flush()
    libc.fflush(None)
    saved = os.dup(1)
    os.dup2(2, 1)
    try:
        yield
    finally:
        libc.fflush(None)
        os.dup2(saved, 1)
        os.close(saved)


def host_available(name: str) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libgellref_host_{name}.so"))


_host_libs: dict[str, ctypes.CDLL] = {}


def host_lib(name: str) -> ctypes.CDLL:
    if name not in _host_libs:
        L = ctypes.CDLL(os.path.join(REF_DIR, f"libgellref_host_{name}.so"))
        L.gref_build_params.argtypes = [P, P]
        L.gref_create.argtypes = [ctypes.c_float] * 3
        L.gref_create.restype = P
        for f in ("gref_destroy", "gref_fm_update", "gref_prelod", "gref_count"):
            getattr(L, f).argtypes = [P]
            getattr(L, f).restype = ctypes.c_int
        for f in ("gref_set_cells", "gref_get_cells"):
            getattr(L, f).argtypes = [P, P, ctypes.c_int]
            getattr(L, f).restype = ctypes.c_int
        L.gref_cells_ptr.argtypes = [P]
        L.gref_cells_ptr.restype = P
        L.gref_prelod_ptr.argtypes = [P, P, ctypes.c_int]
        L.gref_lodsolver.argtypes = [P, ctypes.c_int]
        for f in ("gref_get_field", "gref_set_field"):
            getattr(L, f).argtypes = [P, P]
        L.gref_threads.restype = ctypes.c_int
        _host_libs[name] = L
    return _host_libs[name]


class HostRefSim:
    """The reference's FM and LOD kernel bodies compiled for the host (oracle/ref_host_harness.cpp,
    OpenMP over each launch's threads): Mesh_struct, MechanicsMesh_struct and the cells."""

    def __init__(self, name: str, conc: float, D: float, decay: float):
        self.L = host_lib(name)
        i4 = np.zeros(4, np.int32)
        f4 = np.zeros(4, np.float32)
        self.L.gref_build_params(i4.ctypes.data, f4.ctypes.data)
        self.N, self.cap, self.threads = int(i4[0]), int(i4[1]), int(i4[3])
        with quiet_stdout():
            self.h = self.L.gref_create(conc, D, decay)
        if not self.h:
            raise RuntimeError("host reference set-up failed")

    def close(self):
        if self.h:
            with quiet_stdout():
                self.L.gref_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def count(self) -> int:
        return self.L.gref_count(self.h)

    def set_cells(self, cells: np.ndarray):
        c = np.ascontiguousarray(cells, CELL_DTYPE)
        assert self.L.gref_set_cells(self.h, c.ctypes.data, len(c)) == 0

    def cells(self) -> np.ndarray:
        n = self.count()
        out = np.zeros(max(n, 1), CELL_DTYPE)
        assert self.L.gref_get_cells(self.h, out.ctypes.data, n) == 0
        return out[:n]

    def fm_update(self):
        self.L.gref_fm_update(self.h)

    def prelod(self):
        self.L.gref_prelod(self.h)

    def prelod_on(self, other: "HostRefSim"):
        self.L.gref_prelod_ptr(self.h, self.L.gref_cells_ptr(other.h), other.count())

    def lodsolver(self, k: int):
        self.L.gref_lodsolver(self.h, k)

    def field(self) -> np.ndarray:
        out = np.zeros(self.N ** 3, np.float32)
        self.L.gref_get_field(self.h, out.ctypes.data)
        return out

    def set_field(self, f: np.ndarray):
        f = np.ascontiguousarray(f, np.float32)
        self.L.gref_set_field(self.h, f.ctypes.data)
