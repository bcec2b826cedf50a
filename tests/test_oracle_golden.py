"""Pin the oracle against the reference's own host-callable functions.

tests/golden/host_ref.npz holds inputs and outputs of the reference's Morton_encode, Find_Mesh,
Check_Inside, Cell::O2_consume, Cell::Volume_update, Cell::Phase_update_ki67adv and
Cell::Radius_update (include/BasicFunctions.cuh, include/Cells.cuh), compiled from the unmodified
reference sources and run on the CPU by tests/golden/make_golden_host.py.  Bit-exact comparisons.
"""
import ctypes
import os

import numpy as np
import pytest

import oracle_lib as ol
from gell_b200.cells import CELL_DTYPE

GOLD = os.path.join(os.path.dirname(__file__), "golden", "host_ref.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def cells_of(raw):
    return np.ascontiguousarray(raw).view(CELL_DTYPE).reshape(-1).copy()


def test_reference_build_parameters(gold):
    # default build: Voxel_num 100, Voxel_length 25, Max_Cell_num 2M, sizeof(Cell) 72
    assert list(gold["l25_params_i"][:3]) == [100, 2000000, 72]
    assert gold["l25_params_f"][0] == 25.0
    assert gold["l10_params_f"][0] == 10.0


def test_morton_bit_exact(gold):
    L = ol.lib()
    got = np.array([L.go_morton(int(a), int(b), int(c)) for a, b, c in gold["morton_ijk"]], np.int32)
    np.testing.assert_array_equal(got, gold["morton"])


@pytest.mark.parametrize("tag,length,N", [("l25", 25.0, 100), ("l10", 10.0, 32)])
def test_find_mesh_and_inside(gold, tag, length, N):
    L = ol.lib()
    pos = gold["mesh_pos"]
    got = np.zeros((len(pos), 3), np.int32)
    ins = np.zeros(len(pos), np.int32)
    for n in range(len(pos)):
        p = np.ascontiguousarray(pos[n])
        o = np.zeros(3, np.int32)
        L.go_find_mesh(p.ctypes.data, length, o.ctypes.data)
        got[n] = o
        ins[n] = L.go_inside(int(o[0]), int(o[1]), int(o[2]), N)
    np.testing.assert_array_equal(got, gold[f"mesh_ijk_{tag}"])
    np.testing.assert_array_equal(ins, gold[f"mesh_inside_{tag}"])


@pytest.mark.parametrize("tag,length", [("l25", 25.0), ("l10", 10.0)])
def test_o2_consume(gold, tag, length):
    L = ol.lib()
    cells = cells_of(gold["model_in"])
    got = np.array([L.go_uptake(cells[n:n + 1].ctypes.data, -10.0, length, 0.1)
                    for n in range(len(cells))], np.float32)
    np.testing.assert_array_equal(got.view(np.uint32), gold[f"o2_consume_{tag}"].view(np.uint32))


def test_volume_update_host_semantics(gold):
    """The reference's host build rounds every operation: the oracle's GO_VOL_HOST mode."""
    L = ol.lib()
    cells = cells_of(gold["model_in"])
    for n in range(len(cells)):
        L.go_volume_update_mode(cells[n:n + 1].ctypes.data, ol.GO_VOL_HOST)
    ref = cells_of(gold["volume_out"])
    np.testing.assert_array_equal(cells.view(np.uint8), ref.view(np.uint8))


def test_volume_update_device_semantics_close(gold):
    """The fused device sequence differs from the host build by at most a few ulp."""
    L = ol.lib()
    cells = cells_of(gold["model_in"])
    for n in range(len(cells)):
        L.go_volume_update_mode(cells[n:n + 1].ctypes.data, ol.GO_VOL_DEVICE_REF)
    ref = cells_of(gold["volume_out"])
    for f in ("V", "Vf", "Vcs", "Vns", "r"):
        np.testing.assert_allclose(cells[f], ref[f], rtol=2e-6, atol=1e-4)


def test_phase_update_bit_exact(gold):
    L = ol.lib()
    P = ol.params()
    cells = cells_of(gold["model_in"])
    ret = np.zeros(len(cells), np.int32)
    for n in range(len(cells)):
        ret[n] = L.go_phase_update(cells[n:n + 1].ctypes.data, float(gold["phase_rand"][n]),
                                   float(gold["phase_o2"][n]), ctypes.byref(P))
    ref = cells_of(gold["phase_out"])
    np.testing.assert_array_equal(ret, gold["phase_ret"])
    np.testing.assert_array_equal(cells.view(np.uint8), ref.view(np.uint8))
    # the grid reaches every branch of the Ki-67 state machine
    assert ret.sum() > 0
    assert set(np.unique(ref["phase"])) >= {-1, 0, 1, 2, 3, 4, 5}
    assert (ref["sign"] == 0).sum() > 0


def test_radius_update(gold):
    L = ol.lib()
    cells = cells_of(gold["model_in"])
    for n in range(len(cells)):
        L.go_radius_update(cells[n:n + 1].ctypes.data)
    np.testing.assert_array_equal(cells["r"].view(np.uint32), gold["radius_out"].view(np.uint32))
