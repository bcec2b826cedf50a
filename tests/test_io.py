"""Snapshots and initialisation on the CPU against the reference's own host code (built from its
sources by oracle/Makefile): the initial spheroid of Cell_sphere_Initialization and the cell CSV of
savecsv_cell must be identical."""
import numpy as np
import pytest

import ref_lib
from cases import ball_cells

gb = pytest.importorskip("gell_b200")

FLOATS = ("pos", "force", "oldforce", "r", "V", "Vf", "Vcs", "Vns", "cell_clock")


@pytest.mark.skipif(not ref_lib.available("default"), reason="reference build oracle/_ref missing")
@pytest.mark.parametrize("seed,n", [(1, 2347), (5, 500)])
def test_reference_spheroid_matches_reference_initialization(seed, n):
    # the default build has the reference's own parameters: 100^3 voxels of 25 um
    ours = gb.reference_spheroid(n, 8.4, seed, voxel_num=100, voxel_length=25.0)
    ref = np.zeros(n, gb.CELL_DTYPE)
    assert ref_lib.lib("default").gref_init_sphere(seed, n, ref.ctypes.data) == 0
    for f in ("sign", "mesh_idx", "phase"):
        np.testing.assert_array_equal(ours[f], ref[f], err_msg=f)
    for f in FLOATS:
        np.testing.assert_array_equal(ours[f].view(np.uint32), ref[f].view(np.uint32), err_msg=f)


@pytest.mark.skipif(not ref_lib.available("default"), reason="reference build oracle/_ref missing")
def test_cells_csv_matches_savecsv_cell(tmp_path):
    cells = ball_cells(32, 10.0, 3000, seed=51, dead_frac=0.2)
    cells["phase"] = np.random.default_rng(0).integers(-1, 6, len(cells))
    a, b = tmp_path / "ours.csv", tmp_path / "ref.csv"
    gb.write_cells_csv(cells, str(a))
    assert ref_lib.lib("default").gref_savecsv_cell(cells.ctypes.data, len(cells), str(b).encode()) == 0
    assert a.read_bytes() == b.read_bytes()
    assert a.read_text().splitlines()[0] == "Index,Sign,Phase,x,y,z,r,V,Vns,Vcs"
