"""Field snapshots against the reference's savecsv_mesh / savecsv_meshslice, and checkpoint/resume:
a run interrupted by gell_checkpoint_save and continued in a new context from gell_checkpoint_load
must give exactly the cells and fields of the uninterrupted run."""
import numpy as np
import pytest

import ref_lib
from cases import ball_cells, random_field
from gell_b200.cells import CELL_DTYPE

pytestmark = pytest.mark.gpu

gb = pytest.importorskip("gell_b200")


def raw(c):
    return np.ascontiguousarray(c).view(np.uint8).reshape(len(c), CELL_DTYPE.itemsize)


@pytest.mark.skipif(not ref_lib.available("t32"), reason="reference build oracle/_ref missing")
def test_field_csv_matches_reference(tmp_path):
    field = random_field(32, seed=61)
    with ref_lib.RefSim("t32", 38.0, 1e5, 0.1) as ref, \
            gb.Simulation(voxel_num=32, voxel_length=10.0, max_cell_num=ref.cap) as sim:
        ref.set_field(field)
        sim.add_substrate(gb.oxygen())
        sim.set_field(0, field)
        ref.savecsv_mesh(str(tmp_path / "ref_mesh.csv"))
        sim.save_field_csv(0, str(tmp_path / "mesh.csv"))
        assert (tmp_path / "mesh.csv").read_bytes() == (tmp_path / "ref_mesh.csv").read_bytes()
        ref.savecsv_meshslice(str(tmp_path / "ref_slice.csv"))
        sim.save_field_slice_csv(0, str(tmp_path / "slice.csv"))
        assert (tmp_path / "slice.csv").read_bytes() == (tmp_path / "ref_slice.csv").read_bytes()


def test_cells_csv_of_context_equals_host_writer(tmp_path):
    cells = ball_cells(32, 10.0, 2000, seed=62)
    with gb.Simulation(voxel_num=32, voxel_length=10.0, max_cell_num=65536) as sim:
        sim.import_cells(cells)
        sim.FM_update()
        sim.save_cells_csv(str(tmp_path / "a.csv"))
        gb.write_cells_csv(sim.export_cells(), str(tmp_path / "b.csv"))
        assert (tmp_path / "a.csv").read_bytes() == (tmp_path / "b.csv").read_bytes()


def eventful(n, seed):
    c = ball_cells(32, 10.0, n, seed, radius_frac=0.3, outside=0)
    return gb.seed_ki67_states(c, seed)


def make(rng_mode):
    sim = gb.Simulation(voxel_num=32, voxel_length=10.0, max_cell_num=65536, rng_mode=rng_mode, seed=77)
    sim.add_substrate(gb.oxygen())
    sim.add_substrate(gb.drug())
    return sim


def segment(sim):
    sim.run_mechanics(3, 4)
    sim.CellBirth_kernel()
    sim.run_mechanics(2, 4)
    sim.CellDeath_kernel()


@pytest.mark.parametrize("rng_mode", [gb.GELL_RNG_XORWOW, gb.GELL_RNG_PHILOX])
def test_checkpoint_resume_is_bit_exact(tmp_path, rng_mode):
    cells = eventful(6000, 63)
    path = str(tmp_path / "run.ckpt")
    with make(rng_mode) as a:
        a.set_field(0, random_field(32, seed=64))
        a.set_field(1, random_field(32, seed=65, lo=0.0, hi=1.0))
        a.import_cells(cells)
        segment(a)
        a.checkpoint_save(path)
        segment(a)
        segment(a)
        a.sync()
        ref = (raw(a.export_cells()), a.field(0), a.field(1))
    with make(rng_mode) as b:
        b.checkpoint_load(path)
        segment(b)
        segment(b)
        b.sync()
        got = (raw(b.export_cells()), b.field(0), b.field(1))
    assert len(ref[0]) == len(got[0]) and len(ref[0]) != len(cells)
    np.testing.assert_array_equal(got[0], ref[0])
    for x, y in zip(got[1:], ref[1:]):
        np.testing.assert_array_equal(x.view(np.uint32), y.view(np.uint32))


def test_checkpoint_refuses_other_parameters(tmp_path):
    path = str(tmp_path / "run.ckpt")
    with make(gb.GELL_RNG_PHILOX) as a:
        a.import_cells(eventful(500, 66))
        a.checkpoint_save(path)
    with gb.Simulation(voxel_num=33, voxel_length=10.0, max_cell_num=65536, rng_mode=gb.GELL_RNG_PHILOX,
                       seed=77) as b:
        b.add_substrate(gb.oxygen())
        b.add_substrate(gb.drug())
        with pytest.raises(gb.GellError) as e:
            b.checkpoint_load(path)
        assert e.value.status == -6
