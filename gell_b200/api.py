"""Python mirror of the gell_b200 C ABI (include/gell.h).

The reference drives its hot path from a C++ host loop through member functions of
MechanicsMesh_struct and Mesh_struct and two free functions (include/FMkernel.cuh:181,
include/LODkernel.cuh:270,280, include/PDkernel.cuh:88,100).  `Simulation` exposes the same
operations under the same names (FM_update, PreLOD, LODsolver, CellBirth_kernel,
CellDeath_kernel) on top of the C ABI, for tests, benchmarks and Python callers; C and C++ callers
use include/gell.h or include/gell_compat.hpp directly.

The compute path is the CUDA library gell_b200/libgell_b200.so; there is no other implementation,
and constructing a Simulation fails loudly when that library is missing or no GPU is visible.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

from .cells import CELL_DTYPE

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libgell_b200.so")

GELL_OK = 0
STATUS_NAMES = {
    0: "GELL_OK", -1: "GELL_ERR_INVALID_ARG", -2: "GELL_ERR_CAPACITY", -3: "GELL_ERR_CUDA",
    -4: "GELL_ERR_NO_DEVICE", -5: "GELL_ERR_TIMEOUT", -6: "GELL_ERR_STATE",
    -7: "GELL_ERR_UNSUPPORTED", -8: "GELL_ERR_ALLOC",
}
GELL_RNG_XORWOW, GELL_RNG_PHILOX = 0, 1
GELL_DUMP_KEYS, GELL_DUMP_PERM, GELL_DUMP_SE, GELL_DUMP_RATE, GELL_DUMP_EF = 1, 2, 3, 4, 5

F = ctypes.c_float
D = ctypes.c_double
I32 = ctypes.c_int32
P = ctypes.c_void_p


class GellParams(ctypes.Structure):
    """struct gell_params (include/gell.h)."""
    _fields_ = [
        ("voxel_num", I32), ("voxel_length", F), ("max_cell_num", I32),
        ("mechanics_dt", F), ("diffusion_dt", F), ("biology_dt", F),
        ("ccca", F), ("cccr", F), ("ra_ratio", D), ("cc_max_dist", F),
        ("dead_uptake_factor", F), ("default_v", F),
        ("o2_prolif_thres", F), ("o2_prolif_sat", F), ("o2_necrosis_thres", F),
        ("o2_necrosis_max", F),
        ("necrosis_rate", D), ("apoptosis_rate", D), ("proliferation_rate", D),
        ("duration_pre2post", F), ("duration_post2q", F),
        ("o2_substrate", I32), ("rng_mode", I32), ("mech_mode", I32), ("_reserved0", I32),
        ("seed", ctypes.c_uint64),
    ]


class GellProfileRecord(ctypes.Structure):
    """struct gell_profile_record (include/gell.h)."""
    _fields_ = [("name", ctypes.c_char * 40), ("launches", ctypes.c_int32), ("total_ms", ctypes.c_float)]


class GellSubstrate(ctypes.Structure):
    """struct gell_substrate (include/gell.h)."""
    _fields_ = [("boundary", F), ("diffusion", F), ("decay", F), ("uptake", F), ("init", F)]


@dataclass
class Substrate:
    boundary: float
    diffusion: float
    decay: float
    uptake: float
    init: float


def oxygen() -> Substrate:
    """Oxygen as the reference defines it (include/Definitions.h:21-24)."""
    return Substrate(boundary=38.0, diffusion=1e5, decay=0.1, uptake=-10.0, init=38.0)


def drug() -> Substrate:
    """The second substrate of the large plain-method workload: D 5e4, decay 0.05, boundary 1,
    uptake 1 per min; starts at its boundary value like oxygen does."""
    return Substrate(boundary=1.0, diffusion=5e4, decay=0.05, uptake=-1.0, init=1.0)


class GellError(RuntimeError):
    def __init__(self, status: int, what: str, detail: str = ""):
        self.status = status
        super().__init__(f"{what}: {STATUS_NAMES.get(status, status)}" + (f" ({detail})" if detail else ""))


_lib = None


def load_library() -> ctypes.CDLL:
    """Load gell_b200/libgell_b200.so (built by `make -C gell_b200/csrc`)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C gell_b200/csrc` "
                          "(the CUDA library is the only implementation of the hot path)")
    L = ctypes.CDLL(LIB_PATH)
    L.gell_params_default.argtypes = [P]
    L.gell_params_default.restype = None
    L.gell_substrate_oxygen.argtypes = [P]
    L.gell_substrate_oxygen.restype = None
    L.gell_create.argtypes = [P, P]
    L.gell_destroy.argtypes = [P]
    L.gell_set_stream.argtypes = [P, P]
    L.gell_substrate_add.argtypes = [P, P, P]
    L.gell_cells_import.argtypes = [P, P, ctypes.c_int, ctypes.c_int]
    L.gell_cells_export.argtypes = [P, P, ctypes.c_int, P, ctypes.c_int]
    L.gell_cell_count.argtypes = [P, P]
    L.gell_cells_import_async.argtypes = [P, P, ctypes.c_int]
    L.gell_cells_export_async.argtypes = [P, P, ctypes.c_int, P]
    L.gell_wait_transfers.argtypes = [P]
    L.gell_run_mechanics.argtypes = [P, ctypes.c_int, ctypes.c_int]
    L.gell_write_cells_csv.argtypes = [P, ctypes.c_int, ctypes.c_char_p]
    L.gell_save_cells_csv.argtypes = [P, ctypes.c_char_p]
    L.gell_save_field_csv.argtypes = [P, ctypes.c_int, ctypes.c_char_p]
    L.gell_save_field_slice_csv.argtypes = [P, ctypes.c_int, ctypes.c_char_p]
    L.gell_checkpoint_save.argtypes = [P, ctypes.c_char_p]
    L.gell_checkpoint_load.argtypes = [P, ctypes.c_char_p]
    L.gell_reference_spheroid.argtypes = [P, ctypes.c_int, ctypes.c_float, ctypes.c_uint32, P]
    L.gell_ensemble_create.argtypes = [P, ctypes.c_int, P]
    L.gell_ensemble_destroy.argtypes = [P]
    L.gell_ensemble_configure.argtypes = [P, ctypes.c_int, ctypes.c_int]
    L.gell_ensemble_run_mechanics.argtypes = [P, ctypes.c_int, ctypes.c_int]
    L.gell_ensemble_tune.argtypes = [P, ctypes.c_int, P, P, P]
    L.gell_ensemble_sync.argtypes = [P]
    L.gell_ensemble_set_batched.argtypes = [P, ctypes.c_int]
    L.gell_ensemble_get_batched.argtypes = [P, P]
    L.gell_field_import.argtypes = [P, ctypes.c_int, P, ctypes.c_int]
    L.gell_field_export.argtypes = [P, ctypes.c_int, P, ctypes.c_int]
    L.gell_fm_update.argtypes = [P]
    L.gell_prelod.argtypes = [P, ctypes.c_int]
    L.gell_lod_solver.argtypes = [P, ctypes.c_int, ctypes.c_int]
    L.gell_cell_birth.argtypes = [P, P]
    L.gell_cell_death.argtypes = [P, P]
    L.gell_mechanics_step.argtypes = [P, ctypes.c_int]
    L.gell_sync.argtypes = [P]
    L.gell_debug_dump.argtypes = [P, ctypes.c_int, ctypes.c_int, P, ctypes.c_size_t]
    L.gell_status_string.argtypes = [ctypes.c_int]
    L.gell_status_string.restype = ctypes.c_char_p
    L.gell_last_error.argtypes = [P]
    L.gell_last_error.restype = ctypes.c_char_p
    L.gell_abi_version.restype = ctypes.c_int
    L.gell_profile_enable.argtypes = [P, ctypes.c_int]
    L.gell_profile_read.argtypes = [P, P, ctypes.c_int, P, ctypes.c_int]
    L.gell_launch_count.argtypes = [P, P]
    L.gell_set_option.argtypes = [P, ctypes.c_int, ctypes.c_int64]
    L.gell_selftest_timeout.argtypes = [P, ctypes.c_int]
    L.gell_selftest_division.argtypes = [P, ctypes.c_int64, ctypes.c_uint64, P]
    L.gell_surrogate_weight_count.argtypes = []
    L.gell_surrogate_weight_count.restype = ctypes.c_longlong
    L.gell_surrogate_load.argtypes = [P, ctypes.c_int, P, ctypes.c_longlong, ctypes.c_int, ctypes.c_float,
                                      ctypes.c_float]
    L.gell_lod_surrogate.argtypes = [P, ctypes.c_int, P, P]
    L.gell_surrogate_infer.argtypes = [P, ctypes.c_int]
    L.gell_surrogate_run_layers.argtypes = [P, ctypes.c_int, ctypes.c_int]
    L.gell_surrogate_read.argtypes = [P, ctypes.c_int, ctypes.c_int, P, ctypes.c_longlong]
    L.gell_surrogate_train_init.argtypes = [P, ctypes.c_int, P, ctypes.c_longlong, ctypes.c_int, ctypes.c_float]
    L.gell_surrogate_train_pair.argtypes = [P, ctypes.c_int, ctypes.c_float, P]
    L.gell_surrogate_train_read.argtypes = [P, ctypes.c_int, ctypes.c_int, P, ctypes.c_longlong]
    for name in ("gell_create", "gell_destroy", "gell_set_stream", "gell_substrate_add",
                 "gell_cells_import", "gell_cells_export", "gell_cell_count", "gell_field_import",
                 "gell_field_export", "gell_fm_update", "gell_prelod", "gell_lod_solver",
                 "gell_cell_birth", "gell_cell_death", "gell_mechanics_step", "gell_sync",
                 "gell_debug_dump", "gell_profile_enable", "gell_profile_read", "gell_launch_count",
                 "gell_selftest_division", "gell_set_option", "gell_selftest_timeout", "gell_cells_import_async",
                 "gell_cells_export_async", "gell_wait_transfers", "gell_run_mechanics",
                 "gell_write_cells_csv", "gell_save_cells_csv", "gell_save_field_csv",
                 "gell_save_field_slice_csv", "gell_checkpoint_save", "gell_checkpoint_load",
                 "gell_reference_spheroid", "gell_ensemble_create", "gell_ensemble_destroy",
                 "gell_ensemble_configure", "gell_ensemble_run_mechanics", "gell_ensemble_tune",
                 "gell_ensemble_sync", "gell_ensemble_set_batched", "gell_ensemble_get_batched", "gell_surrogate_load", "gell_lod_surrogate", "gell_surrogate_infer",
                 "gell_surrogate_run_layers", "gell_surrogate_read", "gell_surrogate_train_init",
                 "gell_surrogate_train_pair", "gell_surrogate_train_read"):
        getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def default_params(**overrides) -> GellParams:
    """The reference's compile-time parameter set (include/Definitions.h), with overrides."""
    p = GellParams()
    load_library().gell_params_default(ctypes.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(f"gell_params has no field {k}")
        setattr(p, k, v)
    return p


def _ptr(a) -> int:
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data
    return int(a.data_ptr())  # torch tensor


class Simulation:
    """One gell context: cells, substrates and the hot path on the current CUDA device."""

    def __init__(self, params: GellParams | None = None, **overrides):
        self.lib = load_library()
        self.params = params if params is not None else default_params(**overrides)
        h = P()
        self._check(self.lib.gell_create(ctypes.byref(self.params), ctypes.byref(h)), "gell_create", None)
        self.h = h
        self.N = self.params.voxel_num
        self.nsub = 0

    # -- plumbing
    def _check(self, st: int, what: str, h=-1):
        if st != GELL_OK:
            handle = self.h if h == -1 else h
            detail = self.lib.gell_last_error(handle).decode() if handle else ""
            raise GellError(st, what, detail)

    def close(self):
        if getattr(self, "h", None):
            self.lib.gell_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream) -> None:
        """Use a torch.cuda.Stream (or raw cudaStream_t int) for every later call."""
        raw = getattr(stream, "cuda_stream", stream)
        self._check(self.lib.gell_set_stream(self.h, P(raw)), "gell_set_stream")

    def sync(self) -> None:
        self._check(self.lib.gell_sync(self.h), "gell_sync")

    # -- state
    def add_substrate(self, s: Substrate) -> int:
        c = GellSubstrate(s.boundary, s.diffusion, s.decay, s.uptake, s.init)
        idx = ctypes.c_int()
        self._check(self.lib.gell_substrate_add(self.h, ctypes.byref(c), ctypes.byref(idx)),
                    "gell_substrate_add")
        self.nsub += 1
        return idx.value

    def import_cells(self, cells, on_device: bool = False) -> None:
        n = len(cells) if isinstance(cells, np.ndarray) else cells.shape[0] // CELL_DTYPE.itemsize
        if isinstance(cells, np.ndarray) and cells.dtype != CELL_DTYPE:
            raise TypeError("cells must have gell_b200.CELL_DTYPE")
        self._check(self.lib.gell_cells_import(self.h, P(_ptr(cells) if n else 0), n, int(on_device)),
                    "gell_cells_import")

    def export_cells(self, out: np.ndarray | None = None) -> np.ndarray:
        n = self.count()
        if out is None:
            out = np.zeros(max(n, 1), CELL_DTYPE)
        cnt = ctypes.c_int()
        self._check(self.lib.gell_cells_export(self.h, P(_ptr(out)), len(out), ctypes.byref(cnt), 0),
                    "gell_cells_export")
        return out[:cnt.value]

    def import_cells_async(self, cells: np.ndarray) -> None:
        """Queued import from host memory (pinned for overlap); `cells` must stay unchanged until
        the transfer has finished (sync(), or wait_transfers() in stream order)."""
        if cells.dtype != CELL_DTYPE:
            raise TypeError("cells must have gell_b200.CELL_DTYPE")
        n = len(cells)
        self._check(self.lib.gell_cells_import_async(self.h, P(_ptr(cells) if n else 0), n),
                    "gell_cells_import_async")

    def export_cells_async(self, out: np.ndarray) -> int:
        """Queued export into host memory `out`; valid after sync().  Returns the count."""
        cnt = ctypes.c_int()
        self._check(self.lib.gell_cells_export_async(self.h, P(_ptr(out)), len(out), ctypes.byref(cnt)),
                    "gell_cells_export_async")
        return cnt.value

    def run_mechanics(self, steps: int, substeps: int = 10) -> None:
        """`steps` mechanics steps (FM_update, PreLOD, `substeps` LOD substeps each), pairs of them
        replayed from a captured CUDA graph; queued, no host synchronisation."""
        self._check(self.lib.gell_run_mechanics(self.h, steps, substeps), "gell_run_mechanics")

    # -- snapshots and checkpoints
    def save_cells_csv(self, path: str) -> None:
        self._check(self.lib.gell_save_cells_csv(self.h, os.fsencode(path)), "gell_save_cells_csv")

    def save_field_csv(self, sub: int, path: str) -> None:
        self._check(self.lib.gell_save_field_csv(self.h, sub, os.fsencode(path)), "gell_save_field_csv")

    def save_field_slice_csv(self, sub: int, path: str) -> None:
        self._check(self.lib.gell_save_field_slice_csv(self.h, sub, os.fsencode(path)), "gell_save_field_slice_csv")

    def checkpoint_save(self, path: str) -> None:
        self._check(self.lib.gell_checkpoint_save(self.h, os.fsencode(path)), "gell_checkpoint_save")

    def checkpoint_load(self, path: str) -> None:
        self._check(self.lib.gell_checkpoint_load(self.h, os.fsencode(path)), "gell_checkpoint_load")

    def wait_transfers(self) -> None:
        """Make the context's stream wait for every queued transfer (the host does not block)."""
        self._check(self.lib.gell_wait_transfers(self.h), "gell_wait_transfers")

    def export_cells_device(self, out_tensor) -> int:
        """Write the cells as 72-byte records into a CUDA uint8 tensor; returns the count."""
        cnt = ctypes.c_int()
        cap = out_tensor.numel() // CELL_DTYPE.itemsize
        self._check(self.lib.gell_cells_export(self.h, P(_ptr(out_tensor)), cap, ctypes.byref(cnt), 1),
                    "gell_cells_export")
        return cnt.value

    def count(self) -> int:
        n = ctypes.c_int()
        self._check(self.lib.gell_cell_count(self.h, ctypes.byref(n)), "gell_cell_count")
        return n.value

    def set_field(self, sub: int, field: np.ndarray) -> None:
        f = np.ascontiguousarray(field, np.float32).reshape(-1)
        if f.size != self.N ** 3:
            raise ValueError("field must hold N^3 values")
        self._check(self.lib.gell_field_import(self.h, sub, P(f.ctypes.data), 0), "gell_field_import")

    def field(self, sub: int) -> np.ndarray:
        out = np.zeros(self.N ** 3, np.float32)
        self._check(self.lib.gell_field_export(self.h, sub, P(out.ctypes.data), 0), "gell_field_export")
        return out

    # -- the reference's entry points
    def FM_update(self) -> None:
        self._check(self.lib.gell_fm_update(self.h), "gell_fm_update")

    def PreLOD(self, sub: int = -1) -> None:
        self._check(self.lib.gell_prelod(self.h, sub), "gell_prelod")

    def LODsolver(self, substeps: int = 1, sub: int = -1) -> None:
        self._check(self.lib.gell_lod_solver(self.h, sub, substeps), "gell_lod_solver")

    def CellBirth_kernel(self) -> int:
        n = ctypes.c_int()
        self._check(self.lib.gell_cell_birth(self.h, ctypes.byref(n)), "gell_cell_birth")
        return n.value

    def CellDeath_kernel(self) -> int:
        n = ctypes.c_int()
        self._check(self.lib.gell_cell_death(self.h, ctypes.byref(n)), "gell_cell_death")
        return n.value

    def mechanics_step(self, substeps: int = 10) -> None:
        self._check(self.lib.gell_mechanics_step(self.h, substeps), "gell_mechanics_step")

    # -- profiling
    def profile(self, on: bool = True) -> None:
        self._check(self.lib.gell_profile_enable(self.h, int(on)), "gell_profile_enable")

    def profile_read(self, reset: bool = True) -> dict[str, tuple[int, float]]:
        """{kernel: (launches, total device ms)} since the last reset (synchronises)."""
        recs = (GellProfileRecord * 64)()
        cnt = ctypes.c_int()
        self._check(self.lib.gell_profile_read(self.h, recs, 64, ctypes.byref(cnt), int(reset)),
                    "gell_profile_read")
        return {recs[i].name.decode(): (recs[i].launches, recs[i].total_ms) for i in range(cnt.value)}

    def selftest_division(self, samples: int, seed: int = 1) -> int:
        """Mismatches of the sweeps' division against IEEE division over random operands."""
        m = ctypes.c_int64()
        self._check(self.lib.gell_selftest_division(self.h, samples, seed, ctypes.byref(m)),
                    "gell_selftest_division")
        return m.value

    def selftest_timeout(self, polls: int = 1000) -> int:
        """Run the bounded-wait give-up path; returns the status (GELL_ERR_TIMEOUT = -5 expected)."""
        return self.lib.gell_selftest_timeout(self.h, polls)

    def set_exact_chain(self, on: bool = True) -> None:
        """Run every LOD back-substitution group on the exact division chain (same results)."""
        self._check(self.lib.gell_set_option(self.h, 1, int(bool(on))), "gell_set_option")

    def set_sweep_warps(self, warps: int) -> None:
        """Line tiles per CTA of the LOD sweeps (0 = as many as fit; the ring sweeps use twice as many
        warps); results do not change."""
        self._check(self.lib.gell_set_option(self.h, 3, int(warps)), "gell_set_option")

    def set_sweep_ring(self, on=True) -> None:
        """LOD sweeps as ring kernels (more warps per SM, same results): True/1, or 2..8 = at most
        that many group slots per warp; False/0 = whole line tiles; -1 = automatic (the default)."""
        self._check(self.lib.gell_set_option(self.h, 5, int(on)), "gell_set_option")

    def set_sweep_ring_lag(self, lag: int) -> None:
        """Result stores a ring-sweep warp lets run before refilling a stored slot (0 = default)."""
        self._check(self.lib.gell_set_option(self.h, 7, int(lag)), "gell_set_option")

    def set_lod_streams(self, on: bool = True) -> None:
        """Each substrate's LOD substeps on a stream of its own (same results)."""
        self._check(self.lib.gell_set_option(self.h, 10, int(bool(on))), "gell_set_option")

    def set_sweep_l2hint(self, on: bool = True) -> None:
        """The ring sweeps' L2 eviction priorities (same results)."""
        self._check(self.lib.gell_set_option(self.h, 6, int(bool(on))), "gell_set_option")

    def set_conv_ring(self, on: bool = True) -> None:
        """The surrogate's convolutions with (default) or without the row ring along y."""
        self._check(self.lib.gell_set_option(self.h, 4, int(bool(on))), "gell_set_option")

    def launch_count(self) -> int:
        v = ctypes.c_int64()
        self._check(self.lib.gell_launch_count(self.h, ctypes.byref(v)), "gell_launch_count")
        return v.value

    # -- learned surrogate of one substrate's LOD
    def surrogate_load(self, sub: int, weights: np.ndarray, substeps: int = 50, rate_scale: float = 0.1,
                       threshold: float = 1e-3, input_kind: int = 0) -> None:
        """Load the operator's weights (gell_surrogate_weight_count() floats, conv3d order); input_kind
        is the form the weights were trained for (GELL_OPT_SURROGATE_INPUT: 0 field, 1 one-substep change)."""
        self._check(self.lib.gell_set_option(self.h, 9, int(input_kind)), "gell_set_option")
        w = np.ascontiguousarray(weights, np.float32).reshape(-1)
        self._check(self.lib.gell_surrogate_load(self.h, sub, P(w.ctypes.data), w.size, substeps, rate_scale,
                                                 threshold), "gell_surrogate_load")

    def lod_surrogate(self, sub: int) -> tuple[bool, float]:
        """One judged surrogate step; returns (accepted, judge residual)."""
        acc = ctypes.c_int()
        r = ctypes.c_float()
        self._check(self.lib.gell_lod_surrogate(self.h, sub, ctypes.byref(acc), ctypes.byref(r)),
                    "gell_lod_surrogate")
        return bool(acc.value), float(r.value)

    def surrogate_infer(self, sub: int) -> None:
        self._check(self.lib.gell_surrogate_infer(self.h, sub), "gell_surrogate_infer")

    def surrogate_run_layers(self, sub: int, layers: int) -> None:
        self._check(self.lib.gell_surrogate_run_layers(self.h, sub, layers), "gell_surrogate_run_layers")

    def surrogate_read(self, sub: int, which: int) -> np.ndarray:
        """which 0: input planes, 1: h, 2: t as float32 [C][N^3]; 3: the output field [N^3]."""
        n3 = self.N ** 3
        if which == 3:
            P_ = (self.N + 3) // 4 * 4
            raw = np.zeros(P_ * self.N * self.N, np.float32)
            self._check(self.lib.gell_surrogate_read(self.h, sub, 3, P(raw.ctypes.data), raw.nbytes),
                        "gell_surrogate_read")
            return raw.reshape(self.N, self.N, P_)[:, :, :self.N].reshape(-1).copy()
        planes = 2 if which == 0 else 4
        raw = np.zeros(planes * n3 * 8, np.uint16)
        self._check(self.lib.gell_surrogate_read(self.h, sub, which, P(raw.ctypes.data), raw.nbytes),
                    "gell_surrogate_read")
        f = (raw.astype(np.uint32) << 16).view(np.float32).reshape(planes, n3, 8)
        return f.transpose(0, 2, 1).reshape(planes * 8, n3).copy()

    def surrogate_train_init(self, sub: int, weights: np.ndarray, substeps: int = 50, rate_scale: float = 0.1,
                             input_kind: int = 0) -> None:
        self._check(self.lib.gell_set_option(self.h, 9, int(input_kind)), "gell_set_option")
        w = np.ascontiguousarray(weights, np.float32).reshape(-1)
        self._check(self.lib.gell_surrogate_train_init(self.h, sub, P(w.ctypes.data), w.size, substeps, rate_scale),
                    "gell_surrogate_train_init")

    def surrogate_train_pair(self, sub: int, lr: float, want_loss: bool = True) -> float | None:
        """One training pair from the current state (see gell_surrogate_train_pair)."""
        loss = ctypes.c_float()
        self._check(self.lib.gell_surrogate_train_pair(self.h, sub, lr, ctypes.byref(loss) if want_loss else None),
                    "gell_surrogate_train_pair")
        return float(loss.value) if want_loss else None

    def surrogate_train_read(self, sub: int, which: int) -> np.ndarray:
        """which 0: master weights, 1: last gradient, 2: last target field (N^3)."""
        if which == 2:
            P_ = (self.N + 3) // 4 * 4
            raw = np.zeros(P_ * self.N * self.N, np.float32)
            self._check(self.lib.gell_surrogate_train_read(self.h, sub, 2, P(raw.ctypes.data), raw.size),
                        "gell_surrogate_train_read")
            return raw.reshape(self.N, self.N, P_)[:, :, :self.N].reshape(-1).copy()
        out = np.zeros(self.lib.gell_surrogate_weight_count(), np.float32)
        self._check(self.lib.gell_surrogate_train_read(self.h, sub, which, P(out.ctypes.data), out.size),
                    "gell_surrogate_train_read")
        return out

    # -- parity support
    def _dump(self, what: int, arg: int, dtype, count: int) -> np.ndarray:
        out = np.zeros(max(count, 1), dtype)
        self._check(self.lib.gell_debug_dump(self.h, what, arg, P(out.ctypes.data), out.nbytes),
                    "gell_debug_dump")
        return out[:count]

    def dump_keys(self) -> np.ndarray:
        return self._dump(GELL_DUMP_KEYS, 0, np.int32, self.count())

    def dump_perm(self) -> np.ndarray:
        return self._dump(GELL_DUMP_PERM, 0, np.int32, self.count())

    def dump_se(self) -> tuple[np.ndarray, np.ndarray]:
        se = self._dump(GELL_DUMP_SE, 0, np.int32, 2 * self.N ** 3)
        return se[:self.N ** 3], se[self.N ** 3:]

    def dump_rate(self, sub: int) -> np.ndarray:
        return self._dump(GELL_DUMP_RATE, sub, np.float32, self.N ** 3)

    def dump_ef(self, sub: int) -> tuple[np.ndarray, np.ndarray]:
        ef = self._dump(GELL_DUMP_EF, sub, np.float32, 2 * self.N)
        return ef[:self.N], ef[self.N:]


def write_cells_csv(cells: np.ndarray, path: str) -> None:
    """The reference's savecsv_cell format for host records (no GPU needed)."""
    if cells.dtype != CELL_DTYPE:
        raise TypeError("cells must have gell_b200.CELL_DTYPE")
    c = np.ascontiguousarray(cells)
    st = load_library().gell_write_cells_csv(P(c.ctypes.data if len(c) else 0), len(c), os.fsencode(path))
    if st != GELL_OK:
        raise GellError(st, "gell_write_cells_csv")


def reference_spheroid(n: int, cell_radius: float = 8.4, seed: int = 1, **param_overrides) -> np.ndarray:
    """The reference's initial tumour (Cell_sphere_Initialization) for the given parameters."""
    p = default_params(**param_overrides)
    out = np.zeros(max(n, 1), CELL_DTYPE)
    st = load_library().gell_reference_spheroid(ctypes.byref(p), n, cell_radius, seed, P(out.ctypes.data))
    if st != GELL_OK:
        raise GellError(st, "gell_reference_spheroid")
    return out[:n]


class Ensemble:
    """Independent simulations stepped together (gell_ensemble_*): pairs of mechanics steps of all
    members replay one CUDA graph whose parallel branches run the members side by side."""

    def __init__(self, members: list[Simulation]):
        self.lib = load_library()
        self.members = list(members)
        arr = (P * len(members))(*[m.h for m in members])
        h = P()
        st = self.lib.gell_ensemble_create(arr, len(members), ctypes.byref(h))
        if st != GELL_OK:
            raise GellError(st, "gell_ensemble_create")
        self.h = h

    def _check(self, st: int, what: str) -> None:
        if st != GELL_OK:
            raise GellError(st, what)

    def configure(self, branches: int, sweep_warps: int = 0) -> None:
        self._check(self.lib.gell_ensemble_configure(self.h, branches, sweep_warps), "gell_ensemble_configure")

    def run_mechanics(self, steps: int, substeps: int = 10) -> None:
        self._check(self.lib.gell_ensemble_run_mechanics(self.h, steps, substeps), "gell_ensemble_run_mechanics")

    def tune(self, substeps: int = 10) -> tuple[int, int, int]:
        """Returns (steps taken by every member, best branch count, best sweep tile width)."""
        t, b, w = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.gell_ensemble_tune(self.h, substeps, ctypes.byref(t), ctypes.byref(b), ctypes.byref(w)),
                    "gell_ensemble_tune")
        return t.value, b.value, w.value

    def set_batched(self, on: bool = True) -> None:
        """LOD substeps of all members as one launch per sweep (same results)."""
        self._check(self.lib.gell_ensemble_set_batched(self.h, int(bool(on))), "gell_ensemble_set_batched")

    def batched(self) -> bool:
        v = ctypes.c_int()
        self._check(self.lib.gell_ensemble_get_batched(self.h, ctypes.byref(v)), "gell_ensemble_get_batched")
        return bool(v.value)

    def sync(self) -> None:
        self._check(self.lib.gell_ensemble_sync(self.h), "gell_ensemble_sync")

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.gell_ensemble_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
