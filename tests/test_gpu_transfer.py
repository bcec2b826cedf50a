"""Queued host transfers of the cells (gell_cells_import_async / gell_cells_export_async).

They run on a transfer stream ordered after the last work that used the cells, so a step driven
through them must give exactly the cells that the synchronous import/export give, and an export
queued before the LOD substeps must hold the cells as FM_update and PreLOD left them.
"""
import numpy as np
import pytest

from cases import ball_cells, random_field
from gell_b200.cells import CELL_DTYPE

pytestmark = pytest.mark.gpu

gb = pytest.importorskip("gell_b200")
torch = pytest.importorskip("torch")


def raw(c):
    return np.ascontiguousarray(c).view(np.uint8).reshape(len(c), CELL_DTYPE.itemsize)


def pinned(n):
    return torch.empty(n * CELL_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True).numpy().view(CELL_DTYPE)


def run(cells, field, steps, queued):
    N, length = 32, 10.0
    outs = []
    with gb.Simulation(voxel_num=N, voxel_length=length, max_cell_num=65536) as sim:
        sim.add_substrate(gb.oxygen())
        sim.set_field(0, field)
        host = pinned(len(cells))
        host[:] = cells
        for _ in range(steps):
            if queued:
                sim.import_cells_async(host)
            else:
                sim.import_cells(host)
            sim.FM_update()
            sim.PreLOD()
            sim.LODsolver(5)
            if queued:
                sim.export_cells_async(host)
            else:
                host[:sim.count()] = sim.export_cells()
            if queued:
                sim.sync()
            outs.append(host.copy())
        outs.append(sim.field(0))
    return outs


def test_queued_transfers_match_synchronous_ones():
    cells = ball_cells(32, 10.0, 5000, seed=31)
    field = random_field(32, seed=4)
    a = run(cells, field, 4, queued=False)
    b = run(cells, field, 4, queued=True)
    for x, y in zip(a[:-1], b[:-1]):
        np.testing.assert_array_equal(raw(x), raw(y))
    np.testing.assert_array_equal(a[-1].view(np.uint32), b[-1].view(np.uint32))


def test_queued_steps_without_host_sync():
    """Several steps with no host synchronisation in between: every import waits for the export
    before it (same host buffer) and every FM_update for its import."""
    cells = ball_cells(32, 10.0, 5000, seed=32)
    field = random_field(32, seed=5)
    ref = run(cells, field, 3, queued=False)[-2]
    N, length = 32, 10.0
    with gb.Simulation(voxel_num=N, voxel_length=length, max_cell_num=65536) as sim:
        sim.add_substrate(gb.oxygen())
        sim.set_field(0, field)
        host = pinned(len(cells))
        host[:] = cells
        for _ in range(3):
            sim.import_cells_async(host)
            sim.FM_update()
            sim.PreLOD()
            sim.LODsolver(5)
            sim.export_cells_async(host)
        sim.sync()
        np.testing.assert_array_equal(raw(host), raw(ref))
