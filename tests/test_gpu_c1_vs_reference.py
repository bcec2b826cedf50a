"""The small plain-method workload end to end against the reference's own CUDA build.

100^3 voxels of 10 um, oxygen (boundary 38, D 1e5, decay 0.1, uptake 10), 10^4 cells uniform in a
ball of 150 um at the centre (seed 0), five mechanics steps of FM_update, PreLOD and 10 LOD substeps
each, run by the reference's facades (built from its sources with these parameters) and by
gell_b200.  The cells must agree bit for bit (mechanics has no order-dependent sums); the field
within 1e-5 relative, because both sum the uptake of several cells per voxel with float atomics.
"""
import numpy as np
import pytest

import ref_lib

pytestmark = pytest.mark.gpu

gb = pytest.importorskip("gell_b200")


@pytest.mark.skipif(not ref_lib.available("c1"), reason="reference build oracle/_ref missing")
def test_five_mechanics_steps_match_the_reference_build():
    N, length, steps = 100, 10.0, 5
    cells = gb.cells.uniform_ball(10_000, 150.0, N * length / 2, 0, length, N)
    with ref_lib.RefSim("c1", 38.0, 1e5, 0.1) as ref, \
            gb.Simulation(voxel_num=N, voxel_length=length, max_cell_num=ref.cap) as sim:
        assert ref.N == N
        ref.set_cells(cells)
        sim.add_substrate(gb.oxygen())
        sim.import_cells(cells)
        for _ in range(steps):
            ref.fm_update()
            ref.prelod()
            ref.lodsolver(10)
            sim.FM_update()
            sim.PreLOD()
            sim.LODsolver(10)
        got, exp = sim.export_cells(), ref.cells()
        assert len(got) == len(exp)
        for f in ("sign", "mesh_idx", "phase"):
            np.testing.assert_array_equal(got[f], exp[f], err_msg=f)
        for f in ("pos", "oldforce", "r", "V"):
            np.testing.assert_array_equal(got[f].view(np.uint32), exp[f].view(np.uint32), err_msg=f)
        gf, ef = sim.field(0), ref.field()
        same = np.mean(gf.view(np.uint32) == ef.view(np.uint32))
        print(f"field voxels bit-identical with the reference build after {steps} steps: {same:.6f}")
        np.testing.assert_allclose(gf, ef, rtol=1e-5, atol=0)


@pytest.mark.skipif(not (ref_lib.available("c2") and ref_lib.available("c2d")),
                    reason="reference build oracle/_ref missing")
def test_large_workload_whole_steps_match_the_reference_build():
    """The large plain-method workload (400^3, oxygen + drug, the bench's 10^6-cell lattice
    spheroid), three whole steps (FM_update, PreLOD of both substrates, 10 LODsolver substeps of
    both) through the reference's facades and through gell_b200's graph-driven step loop: the cells'
    integer fields, radii and volumes bit for bit, positions and forces within 1e-5 relative, both
    fields within 1e-5 relative (float-atomic uptake sums, as in the reference)."""
    N, length, steps = 400, 10.0, 3
    cells = gb.lattice_spheroid(1_000_000, N * length / 2, 0, length, N)
    with ref_lib.RefSim("c2", 38.0, 1e5, 0.1) as o2, ref_lib.RefSim("c2d", 1.0, 5e4, 0.05) as drug, \
            gb.Simulation(voxel_num=N, voxel_length=length, max_cell_num=o2.cap) as sim:
        o2.set_cells(cells)
        sim.add_substrate(gb.oxygen())
        sim.add_substrate(gb.drug())
        sim.import_cells(cells)
        for _ in range(steps):
            o2.fm_update()
            o2.prelod()
            drug.prelod_on(o2)
            o2.lodsolver(10)
            drug.lodsolver(10)
        sim.run_mechanics(steps, 10)
        got, exp = sim.export_cells(), o2.cells()
        assert len(got) == len(exp)
        for f in ("sign", "mesh_idx", "phase"):
            np.testing.assert_array_equal(got[f], exp[f], err_msg=f)
        for f in ("r", "V"):
            np.testing.assert_array_equal(got[f].view(np.uint32), exp[f].view(np.uint32), err_msg=f)
        same = np.mean(np.all(got["pos"].view(np.uint32) == exp["pos"].view(np.uint32), 1))
        print(f"positions bit-identical with the reference build: {same:.6f}")
        np.testing.assert_allclose(got["pos"], exp["pos"], rtol=1e-5, atol=0)
        live = got["sign"] == 1
        fscale = np.abs(exp["oldforce"][live]).max()
        np.testing.assert_allclose(got["oldforce"][live], exp["oldforce"][live], rtol=1e-5, atol=1e-5 * fscale)
        for sub, ref in ((0, o2), (1, drug)):
            gf, ef = sim.field(sub), ref.field()
            same = np.mean(gf.view(np.uint32) == ef.view(np.uint32))
            print(f"substrate {sub}: voxels bit-identical with the reference build after {steps} steps: {same:.6f}")
            np.testing.assert_allclose(gf, ef, rtol=1e-5, atol=0)
