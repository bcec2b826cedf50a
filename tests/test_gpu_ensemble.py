"""Ensembles (gell_ensemble_*): independent simulations of different sizes stepped together through
one CUDA graph of parallel branches must give exactly what each gives when stepped alone, before
and after the tuner and across birth and death (which re-captures the graph)."""
import numpy as np
import pytest

from cases import ball_cells, random_field
from gell_b200.cells import CELL_DTYPE

pytestmark = pytest.mark.gpu

gb = pytest.importorskip("gell_b200")

SIZES = [(32, 1500), (40, 3000), (48, 800), (56, 5000), (64, 2500)]


def raw(c):
    return np.ascontiguousarray(c).view(np.uint8).reshape(len(c), CELL_DTYPE.itemsize)


def member(i, N, n):
    sim = gb.Simulation(voxel_num=N, voxel_length=10.0, max_cell_num=65536, rng_mode=gb.GELL_RNG_PHILOX, seed=100 + i)
    D = 5e4 + 3e4 * i
    sim.add_substrate(gb.Substrate(boundary=38.0, diffusion=D, decay=0.1, uptake=-(5.0 + 3.0 * i), init=38.0))
    sim.set_field(0, random_field(N, seed=200 + i))
    cells = gb.seed_ki67_states(ball_cells(N, 10.0, n, seed=300 + i, radius_frac=0.3, outside=0), 400 + i)
    sim.import_cells(cells)
    return sim


def state(sim):
    return raw(sim.export_cells()), sim.field(0).view(np.uint32)


def members():
    return [member(i, N, n) for i, (N, n) in enumerate(SIZES)]


def test_ensemble_matches_members_stepped_alone():
    alone = members()
    for m in alone:
        for _ in range(5):
            m.mechanics_step(4)
    together = members()
    with gb.Ensemble(together) as ens:
        ens.configure(branches=3, sweep_warps=2)
        ens.run_mechanics(5, 4)
        ens.sync()
    for a, b in zip(alone, together):
        for x, y in zip(state(a), state(b)):
            np.testing.assert_array_equal(x, y)
        assert a.launch_count() == b.launch_count()
    for m in alone + together:
        m.close()


def test_ensemble_across_birth_and_death_and_tuning():
    alone = members()
    together = members()
    with gb.Ensemble(together) as ens:
        taken, branches, warps = ens.tune(3)
        assert taken >= 3 and 1 <= branches <= len(SIZES) and warps in (0, 1, 2)
        for m in alone:
            for _ in range(taken):
                m.mechanics_step(3)
        for _ in range(2):
            for a, b in zip(alone, together):
                a.CellBirth_kernel()
                b.CellBirth_kernel()
            for a in alone:
                for _ in range(4):
                    a.mechanics_step(3)
            ens.run_mechanics(4, 3)
            for a, b in zip(alone, together):
                a.CellDeath_kernel()
                b.CellDeath_kernel()
        ens.sync()
    for a, b in zip(alone, together):
        assert a.count() == b.count()
        for x, y in zip(state(a), state(b)):
            np.testing.assert_array_equal(x, y)
    for m in alone + together:
        m.close()


def test_batched_lod_matches_members_stepped_alone():
    """gell_ensemble_set_batched: the LOD substeps of all members as one launch per sweep over a
    work list of every member's line tiles.  Members of 1 to 7 groups per line (N = 32 .. 200), one
    with two substrates, so consecutive tiles of a warp differ in length; across birth and death."""
    sizes = [(32, 1500), (48, 800), (100, 6000), (131, 9000), (200, 20000), (64, 2500)]

    def make():
        ms = [member(i, N, n) for i, (N, n) in enumerate(sizes)]
        ms[2].add_substrate(gb.drug())
        return ms

    alone, together = make(), make()
    with gb.Ensemble(together) as ens:
        ens.configure(branches=4, sweep_warps=0)
        ens.set_batched(True)
        assert ens.batched()
        for a in alone:
            for _ in range(5):
                a.mechanics_step(4)
        ens.run_mechanics(5, 4)
        for a, b in zip(alone, together):
            a.CellBirth_kernel()
            b.CellBirth_kernel()
        for a in alone:
            for _ in range(4):
                a.mechanics_step(4)
        ens.run_mechanics(4, 4)
        for a, b in zip(alone, together):
            a.CellDeath_kernel()
            b.CellDeath_kernel()
        ens.sync()
    for a, b in zip(alone, together):
        assert a.count() == b.count()
        np.testing.assert_array_equal(raw(a.export_cells()), raw(b.export_cells()))
        np.testing.assert_array_equal(a.field(0).view(np.uint32), b.field(0).view(np.uint32))
    np.testing.assert_array_equal(alone[2].field(1).view(np.uint32), together[2].field(1).view(np.uint32))
    for m in alone + together:
        m.close()


def test_batched_steps_with_empty_and_substrate_free_members():
    """Batched steps (every member's mechanics and LOD as one launch per kernel) when a member holds
    no cells (its uptake map is still cleared) and another has no substrate (no uptake map, no LOD):
    each member gives what it gives stepped alone, across birth and death."""
    def make():
        ms = [member(0, 40, 2000), member(1, 48, 3000), member(2, 56, 4000)]
        empty = gb.Simulation(voxel_num=44, voxel_length=10.0, max_cell_num=65536, rng_mode=gb.GELL_RNG_PHILOX,
                              seed=77)
        empty.add_substrate(gb.oxygen())
        empty.set_field(0, random_field(44, seed=78))
        bare = gb.Simulation(voxel_num=36, voxel_length=10.0, max_cell_num=65536, rng_mode=gb.GELL_RNG_PHILOX,
                             seed=79)
        bare.import_cells(gb.seed_ki67_states(ball_cells(36, 10.0, 1500, seed=80, radius_frac=0.3, outside=0), 81))
        return ms + [empty, bare]

    alone, together = make(), make()
    with gb.Ensemble(together) as ens:
        ens.configure(branches=2, sweep_warps=0)
        ens.set_batched(True)
        for a in alone:
            for _ in range(4):
                a.mechanics_step(3)
        ens.run_mechanics(4, 3)
        for a, b in zip(alone, together):
            a.CellBirth_kernel()
            b.CellBirth_kernel()
        for a in alone:
            for _ in range(3):
                a.mechanics_step(3)
        ens.run_mechanics(3, 3)
        for a, b in zip(alone, together):
            a.CellDeath_kernel()
            b.CellDeath_kernel()
        ens.sync()
    for i, (a, b) in enumerate(zip(alone, together)):
        assert a.count() == b.count(), i
        np.testing.assert_array_equal(raw(a.export_cells()), raw(b.export_cells()))
        if i < 4:
            np.testing.assert_array_equal(a.field(0).view(np.uint32), b.field(0).view(np.uint32))
    assert together[3].count() == 0
    for m in alone + together:
        m.close()
