"""The ring variant of the LOD sweeps (GELL_OPT_SWEEP_RING) against the oracle, bit for bit.

The ring kernels keep only a few group slots per warp: the forward elimination records the running
value entering each group and frees the slot, and the back substitution loads the lower groups a
second time and recomputes their forward values from that checkpoint.  The grid edges below cover
a line of one group (N <= 32), lines with fewer groups than slots (every group resident), ragged
last groups (N = 37, 131), the uniform-group path (N >= 100), the size of the large workload
(N = 400, 13 groups) and a line longer than any ring (N = 600, 19 groups), each with two
substrates, uptake lines and several substeps.  Fields must equal the oracle's
(include/LODkernel.cuh:24-136) and the line-tile kernels' bit for bit."""
import numpy as np
import pytest

import oracle_lib as ol
from cases import one_per_voxel, random_field

pytestmark = pytest.mark.gpu

gb = pytest.importorskip("gell_b200")


def bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


def run(N, cells, field, k, ring, exact=False, warps=0, hint=False, lag=0):
    length = 10.0
    with gb.Simulation(voxel_num=N, voxel_length=length, max_cell_num=max(65536, len(cells) + 1024)) as sim:
        sim.add_substrate(gb.oxygen())
        sim.add_substrate(gb.drug())
        sim.set_sweep_ring(ring)
        sim.set_sweep_l2hint(hint)
        sim.set_sweep_ring_lag(lag)
        sim.set_exact_chain(exact)
        if warps:
            sim.set_sweep_warps(warps)
        sim.set_field(0, field)
        sim.set_field(1, field * np.float32(0.03))
        sim.import_cells(cells)
        sim.PreLOD()
        sim.LODsolver(k)
        return sim.field(0), sim.field(1)


def oracle(N, cells, field, k):
    out = []
    for sub, s in enumerate((gb.oxygen(), gb.drug())):
        rate = ol.prelod(cells, N, 10.0, s.uptake)
        E, F = ol.mesh_init(N, 10.0, s.diffusion, s.decay, 0.01)
        start = field if sub == 0 else field * np.float32(0.03)
        out.append(ol.lod_substeps(start, rate, E, F, N, 0.01, s.boundary, k))
    return out


@pytest.mark.parametrize("N,k", [(16, 2), (32, 3), (37, 3), (64, 2), (100, 3), (131, 2), (200, 2)])
def test_ring_sweeps_bit_exact(N, k):
    cells = one_per_voxel(N, 10.0, seed=N + 3, lo=N // 4, hi=N // 4 + N // 2)
    field = random_field(N, seed=N)
    got = run(N, cells, field, k, ring=True)
    exp = oracle(N, cells, field, k)
    for sub in range(2):
        assert bits_equal(got[sub], exp[sub]), f"N={N} substrate {sub}"


@pytest.mark.parametrize("N", [100, 160])
def test_ring_exact_chain_and_fewer_warps_give_the_same_fields(N):
    cells = one_per_voxel(N, 10.0, seed=5, lo=N // 3, hi=N // 3 + N // 3)
    field = random_field(N, seed=9)
    base = run(N, cells, field, 2, ring=False)
    for exact, warps in ((False, 1), (True, 0), (False, 2)):
        got = run(N, cells, field, 2, ring=True, exact=exact, warps=warps)
        for sub in range(2):
            assert bits_equal(got[sub], base[sub]), (exact, warps, sub)


@pytest.mark.parametrize("N", [400, 600])
def test_ring_sweeps_full_size_vs_oracle(N):
    """The sizes of the large and the birth/death workloads: 13 and 19 groups per line."""
    lo, hi = (150, 250) if N == 400 else (250, 350)
    cells = one_per_voxel(N, 10.0, seed=N, lo=lo, hi=hi)
    rng = np.random.Generator(np.random.Philox(N + 1))
    field = rng.uniform(10.0, 38.0, N ** 3).astype(np.float32)
    got = run(N, cells, field, 2, ring=True)
    exp = oracle(N, cells, field, 2)
    for sub in range(2):
        assert bits_equal(got[sub], exp[sub]), f"N={N} substrate {sub}"


@pytest.mark.parametrize("N", [131, 400])
def test_ring_slot_counts_and_l2_hints_give_the_same_fields(N):
    """Rings of 2, 3 and 5 slots (more groups loaded twice), with and without the L2 priorities,
    with 1 to 4 result stores in flight per warp."""
    cells = one_per_voxel(N, 10.0, seed=N + 11, lo=N // 3, hi=N // 3 + N // 4)
    field = random_field(N, seed=N + 12)
    exp = oracle(N, cells, field, 2)
    for ring, hint, lag in ((2, False, 1), (3, True, 2), (5, False, 4), (1, True, 1), (1, False, 2), (4, False, 3)):
        got = run(N, cells, field, 2, ring=ring, hint=hint, lag=lag)
        for sub in range(2):
            assert bits_equal(got[sub], exp[sub]), (N, ring, hint, lag, sub)


@pytest.mark.parametrize("N,ring", [(131, 0), (400, 0), (600, 1)])
def test_a_stream_per_substrate_gives_the_same_fields(N, ring):
    """GELL_OPT_LOD_STREAMS: each substrate's substeps on a stream of its own, eagerly and replayed
    from the step graph (gell_run_mechanics), bit for bit the single-stream fields."""
    lo, hi = N // 3, N // 3 + N // 6
    cells = one_per_voxel(N, 10.0, seed=N + 31, lo=lo, hi=hi)
    rng = np.random.Generator(np.random.Philox(N + 32))
    field = rng.uniform(10.0, 38.0, N ** 3).astype(np.float32)
    out = []
    for streams in (False, True):
        with gb.Simulation(voxel_num=N, voxel_length=10.0, max_cell_num=len(cells) + 1024) as sim:
            sim.add_substrate(gb.oxygen())
            sim.add_substrate(gb.drug())
            sim.set_sweep_ring(ring if ring else -1)
            sim.set_lod_streams(streams)
            sim.set_field(0, field)
            sim.set_field(1, field * np.float32(0.03))
            sim.import_cells(cells)
            sim.PreLOD()
            sim.LODsolver(2)
            first = (sim.field(0), sim.field(1))
            sim.run_mechanics(4, 3)
            sim.sync()
            out.append((first, (sim.field(0), sim.field(1)), sim.export_cells()))
    for sub in range(2):
        assert bits_equal(out[0][0][sub], out[1][0][sub]), (N, sub)
        # after the cells move, several can share a voxel: float-atomic uptake sums (1e-5)
        np.testing.assert_allclose(out[0][1][sub], out[1][1][sub], rtol=1e-5, atol=0)
    assert np.array_equal(out[0][2].view(np.uint8), out[1][2].view(np.uint8))
