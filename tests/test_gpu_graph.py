"""gell_run_mechanics: mechanics steps replayed from a captured CUDA graph.

Replaying must give exactly what the same steps give when launched one by one (cells and fields
bit for bit), including after the cell count changes (the graph is captured again), and it must
count the kernels it replays.
"""
import numpy as np
import pytest

from cases import ball_cells, random_field
from gell_b200.cells import CELL_DTYPE

pytestmark = pytest.mark.gpu

gb = pytest.importorskip("gell_b200")


def raw(c):
    return np.ascontiguousarray(c).view(np.uint8).reshape(len(c), CELL_DTYPE.itemsize)


def make(cells, N=32):
    sim = gb.Simulation(voxel_num=N, voxel_length=10.0, max_cell_num=65536)
    sim.add_substrate(gb.oxygen())
    sim.add_substrate(gb.drug())
    sim.set_field(0, random_field(N, seed=3))
    sim.set_field(1, random_field(N, seed=4, lo=0.0, hi=1.0))
    sim.import_cells(cells)
    return sim


def state(sim):
    return raw(sim.export_cells()), sim.field(0).view(np.uint32), sim.field(1).view(np.uint32)


@pytest.mark.parametrize("steps", [1, 2, 3, 7])
def test_graph_replay_matches_eager_steps(steps):
    cells = ball_cells(32, 10.0, 4000, seed=41, radius_frac=0.3)
    with make(cells) as a, make(cells) as b:
        for _ in range(steps):
            a.mechanics_step(4)
        b.run_mechanics(steps, 4)
        b.sync()
        for x, y in zip(state(a), state(b)):
            np.testing.assert_array_equal(x, y)


def test_graph_recaptured_when_cells_change():
    cells = ball_cells(32, 10.0, 4000, seed=42, radius_frac=0.3, dead_frac=0.2)
    with make(cells) as a, make(cells) as b:
        for _ in range(5):
            a.mechanics_step(3)
        a.CellDeath_kernel()
        for _ in range(6):
            a.mechanics_step(3)
        b.run_mechanics(5, 3)
        b.CellDeath_kernel()
        b.run_mechanics(6, 3)
        b.sync()
        assert a.count() == b.count() < len(cells)
        for x, y in zip(state(a), state(b)):
            np.testing.assert_array_equal(x, y)


def test_graph_replay_counts_its_kernels():
    cells = ball_cells(32, 10.0, 3000, seed=43)
    with make(cells) as a, make(cells) as b:
        a.mechanics_step(2)
        b.mechanics_step(2)
        l0 = a.launch_count()
        for _ in range(6):
            a.mechanics_step(2)
        l1 = b.launch_count()
        b.run_mechanics(6, 2)
        b.sync()
        assert b.launch_count() - l1 == a.launch_count() - l0
