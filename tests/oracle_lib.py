"""ctypes access to oracle/libgell_oracle.so (the C restatement of the reference's hot path).

Test infrastructure: used by the tests, by __graft_entry__.smoke() and by bench.py's CPU
baseline, always as the checker, never as the code under measurement.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "libgell_oracle.so")

P = ctypes.c_void_p
I = ctypes.c_int
F = ctypes.c_float

GO_VOL_HOST, GO_VOL_DEVICE, GO_VOL_DEVICE_FUSED, GO_VOL_DEVICE_SWAP, GO_VOL_DEVICE_SWAP_FUSED = 0, 1, 2, 3, 4
GO_VOL_DEVICE_REF = 5


class GoParams(ctypes.Structure):
    _fields_ = [
        ("N", ctypes.c_int32), ("len", ctypes.c_float), ("cap", ctypes.c_int32),
        ("mech_dt", F), ("diff_dt", F), ("bio_dt", F),
        ("ccca", F), ("cccr", F), ("ra_ratio", ctypes.c_double), ("cc_max_dist", F),
        ("dead_factor", F), ("default_v", F),
        ("o2_pt", F), ("o2_ps", F), ("o2_nt", F), ("o2_nm", F),
        ("necrosis_rate", ctypes.c_double), ("apoptosis_rate", ctypes.c_double),
        ("prolif_rate", ctypes.c_double),
        ("dur_pre2post", F), ("dur_post2q", F),
    ]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", ORACLE_DIR, "libgell_oracle.so"], check=True,
                           stdout=subprocess.DEVNULL)
        L = ctypes.CDLL(LIB_PATH)
        L.go_params_reference.argtypes = [P]
        L.go_morton.argtypes = [I, I, I]
        L.go_morton.restype = I
        L.go_find_mesh.argtypes = [P, F, P]
        L.go_inside.argtypes = [I, I, I, I]
        L.go_inside.restype = I
        L.go_mesh_init.argtypes = [I, F, F, F, F, P, P]
        L.go_mesh_init_f64.argtypes = [I, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, P, P]
        L.go_lod_substep.argtypes = [P, P, P, P, I, F, F]
        L.go_lod_substep_f64.argtypes = [P, P, P, P, I, ctypes.c_double, ctypes.c_double]
        L.go_thomas_line.argtypes = [P, ctypes.c_long, P, P, I, F]
        L.go_uptake.argtypes = [P, F, F, F]
        L.go_uptake.restype = F
        L.go_prelod.argtypes = [P, I, I, F, F, F, P]
        L.go_update_keys.argtypes = [P, I, P, P]
        L.go_stable_sort.argtypes = [P, P, I, P]
        L.go_cell_list.argtypes = [P, I, P, P, P]
        L.go_force.argtypes = [P, I, P, P, P]
        L.go_update_keys.argtypes = [P, I, P, P]
        L.go_stable_sort.argtypes = [P, P, I, P]
        L.go_cell_list.argtypes = [P, I, P, P, P]
        L.go_force_move_f64.argtypes = [P, I, P, P, P, P, P]
        L.go_force_one.argtypes = [P, I, P, P, P, P]
        L.go_move.argtypes = [P, I, P]
        L.go_fm_update.argtypes = [P, I, P, P, P, P, P]
        L.go_volume_update.argtypes = [P]
        L.go_volume_update_mode.argtypes = [P, I]
        L.go_set_volume_mode.argtypes = [I]
        L.go_volume_update_modes.argtypes = [P, I, I]
        L.go_radius_update.argtypes = [P]
        L.go_phase_update.argtypes = [P, F, F, P]
        L.go_phase_update.restype = I
        L.go_random_vect.argtypes = [F, F, P]
        L.go_philox4x32_10.argtypes = [P, P, P]
        L.go_u01.argtypes = [ctypes.c_uint32]
        L.go_u01.restype = F
        L.go_birth_philox.argtypes = [P, I, P, P, ctypes.c_uint64, ctypes.c_uint32]
        L.go_birth_philox.restype = I
        L.go_birth_draws.argtypes = [P, I, P, P, P, P, P]
        L.go_birth_draws.restype = I
        L.go_death.argtypes = [P, I]
        L.go_death.restype = I
        L.go_set_threads.argtypes = [I]
        L.go_get_threads.restype = I
        _lib = L
    return _lib


def params(**kw) -> GoParams:
    p = GoParams()
    lib().go_params_reference(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def ptr(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def mesh_init(N, length, D, decay, dt):
    E = np.zeros(N, np.float32)
    Fv = np.zeros(N, np.float32)
    lib().go_mesh_init(N, length, D, decay, dt, ptr(E), ptr(Fv))
    return E, Fv


def mesh_init_f64(N, length, D, decay, dt):
    E = np.zeros(N, np.float64)
    Fv = np.zeros(N, np.float64)
    lib().go_mesh_init_f64(N, length, D, decay, dt, ptr(E), ptr(Fv))
    return E, Fv


def lod_substeps(p, rate, E, Fv, N, dt, boundary, k):
    p = np.ascontiguousarray(p, np.float32).copy()
    rate = np.ascontiguousarray(rate, np.float32)
    for _ in range(k):
        lib().go_lod_substep(ptr(p), ptr(rate), ptr(E), ptr(Fv), N, dt, boundary)
    return p


def lod_substeps_f64(p, rate, N, length, D, decay, dt, boundary, k):
    E, Fv = mesh_init_f64(N, length, D, decay, dt)
    p = np.ascontiguousarray(p, np.float64).copy()
    rate = np.ascontiguousarray(rate, np.float64)
    for _ in range(k):
        lib().go_lod_substep_f64(ptr(p), ptr(rate), ptr(E), ptr(Fv), N, dt, boundary)
    return p


def prelod(cells, N, length, coef, dead_factor=0.1):
    rate = np.zeros(N * N * N, np.float32)
    lib().go_prelod(ptr(cells), len(cells), N, length, coef, dead_factor, ptr(rate))
    return rate


def fm_update(cells, P: GoParams):
    """One FM_update in place; returns (keys, perm, s, e)."""
    n = len(cells)
    NNN = P.N ** 3
    keys = np.zeros(max(n, 1), np.int32)
    perm = np.zeros(max(n, 1), np.int32)
    s = np.zeros(NNN, np.int32)
    e = np.zeros(NNN, np.int32)
    lib().go_fm_update(ptr(cells), n, ctypes.byref(P), ptr(keys), ptr(perm), ptr(s), ptr(e))
    return keys[:n], perm[:n], s, e


def force_move_f64(cells, P: GoParams):
    """The cells sorted as FM_update sorts them, and the FP64 force and moved position of each
    live one: (sorted cells, force[n,3], pos[n,3])."""
    c = np.ascontiguousarray(cells).copy()
    n = len(c)
    NNN = P.N ** 3
    keys = np.zeros(max(n, 1), np.int32)
    perm = np.zeros(max(n, 1), np.int32)
    s = np.zeros(NNN, np.int32)
    e = np.zeros(NNN, np.int32)
    lib().go_update_keys(ptr(c), n, ctypes.byref(P), ptr(keys))
    lib().go_stable_sort(ptr(c), ptr(keys), n, ptr(perm))
    lib().go_cell_list(ptr(c), n, ctypes.byref(P), ptr(s), ptr(e))
    f = np.zeros((max(n, 1), 3), np.float64)
    q = np.zeros((max(n, 1), 3), np.float64)
    lib().go_force_move_f64(ptr(c), n, ctypes.byref(P), ptr(s), ptr(e), ptr(f), ptr(q))
    return c, f[:n], q[:n]


def force_one(cells, i, P, s, e):
    out = np.zeros(3, np.float32)
    lib().go_force_one(ptr(cells), i, ctypes.byref(P), ptr(s), ptr(e), ptr(out))
    return out


def philox(ctr, key):
    c = np.asarray(ctr, np.uint32)
    k = np.asarray(key, np.uint32)
    o = np.zeros(4, np.uint32)
    lib().go_philox4x32_10(ptr(c), ptr(k), ptr(o))
    return o


def birth_philox(cells, n, P, field, seed, step):
    return lib().go_birth_philox(ptr(cells), n, ctypes.byref(P), ptr(field), seed, step)


def death(cells, n):
    return lib().go_death(ptr(cells), n)
