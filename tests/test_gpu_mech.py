"""Mechanics (FM_update) on the GPU against the oracle and the reference's own kernels.

Morton keys, the sort permutation and the reference-shaped s/e arrays are integer results and must
be bit-exact.  The force kernel reproduces the reference's candidate order and order-dependent
cutoff, so forces and positions match the oracle bit for bit (the oracle spells out the fused
multiply-adds nvcc forms); against the reference's own build they agree within 1e-5 relative.
"""
import numpy as np
import pytest

import oracle_lib as ol
import ref_lib
from cases import ball_cells
from gell_b200.cells import CELL_DTYPE, lattice_spheroid

pytestmark = pytest.mark.gpu

gb = pytest.importorskip("gell_b200")


def make_sim(N, length, cap=65536):
    return gb.Simulation(voxel_num=N, voxel_length=length, max_cell_num=cap)


def raw(c):
    return np.ascontiguousarray(c).view(np.uint8).reshape(len(c), CELL_DTYPE.itemsize)


@pytest.mark.parametrize("N,n,seed", [(32, 2000, 1), (32, 6000, 2), (50, 20000, 3)])
def test_fm_update_bit_exact_vs_oracle(N, n, seed):
    length = 10.0
    cells = ball_cells(N, length, n, seed)
    P = ol.params(N=N, len=length, cap=65536)
    with make_sim(N, length) as sim:
        sim.import_cells(cells)
        sim.FM_update()
        oc = cells.copy()
        okeys, operm, os_, oe = ol.fm_update(oc, P)
        np.testing.assert_array_equal(sim.dump_keys(), okeys)
        np.testing.assert_array_equal(sim.dump_perm(), operm)
        s, e = sim.dump_se()
        np.testing.assert_array_equal(s, os_)
        np.testing.assert_array_equal(e, oe)
        out = sim.export_cells()
        np.testing.assert_array_equal(raw(out), raw(oc))


def test_fm_update_many_steps_bit_exact():
    N, length = 32, 10.0
    cells = ball_cells(N, length, 4000, seed=5, radius_frac=0.25)
    P = ol.params(N=N, len=length, cap=65536)
    oc = cells.copy()
    with make_sim(N, length) as sim:
        sim.import_cells(cells)
        for step in range(25):
            sim.FM_update()
            ol.fm_update(oc, P)
        out = sim.export_cells()
        np.testing.assert_array_equal(raw(out), raw(oc))
        # the population is compressed enough that cells move and change bins
        assert not np.array_equal(out["pos"], cells["pos"])


def test_sentinel_orders_first_and_outside_cells_lose_sign():
    N, length = 32, 10.0
    cells = ball_cells(N, length, 500, seed=9, outside=8)
    with make_sim(N, length) as sim:
        sim.import_cells(cells)
        sim.FM_update()
        keys = sim.dump_keys()
        n_out = int((keys == -1).sum())
        # of the eight planted positions, (-3, .), (., -5, .) and the ones just inside the far
        # faces truncate into bins 0..N-1; only three are outside the grid
        assert n_out == 3
        assert np.all(keys[:n_out] == -1) and np.all(keys[n_out:] >= 0)
        assert np.all(np.diff(keys) >= 0)
        out = sim.export_cells()
        assert np.all(out["sign"][:n_out] == 0)


@pytest.mark.skipif(not ref_lib.available("t32"), reason="reference build oracle/_ref missing")
@pytest.mark.parametrize("seed", [1, 2])
def test_fm_update_vs_reference_kernels(seed):
    N, length = 32, 10.0
    cells = ball_cells(N, length, 5000, seed=seed)
    with ref_lib.RefSim("t32", 38.0, 1e5, 0.1) as ref, make_sim(N, length) as sim:
        ref.set_cells(cells)
        ref.fm_update()
        sim.import_cells(cells)
        sim.FM_update()
        np.testing.assert_array_equal(sim.dump_keys(), ref.keys())
        s, e = sim.dump_se()
        rs, re_ = ref.se()
        np.testing.assert_array_equal(s, rs)
        np.testing.assert_array_equal(e, re_)
        got, exp = sim.export_cells(), ref.cells()
        for f in ("sign", "mesh_idx", "phase", "r", "V", "Vf", "Vcs", "Vns", "cell_clock"):
            np.testing.assert_array_equal(got[f], exp[f], err_msg=f)
        same = np.mean(np.all(got["oldforce"].view(np.uint32) == exp["oldforce"].view(np.uint32), 1))
        print(f"forces bit-identical with the reference build: {same:.6f}")
        live = got["sign"] == 1
        fscale = np.abs(exp["oldforce"][live]).max()
        np.testing.assert_allclose(got["oldforce"][live], exp["oldforce"][live], rtol=1e-5, atol=1e-5 * fscale)
        np.testing.assert_allclose(got["pos"], exp["pos"], rtol=1e-5, atol=0)


@pytest.mark.skipif(not ref_lib.available("c2"), reason="reference build oracle/_ref missing")
def test_fm_full_size_keys_and_cell_list_vs_reference():
    """10^6 cells on the 400^3 grid: keys and s/e bit-exact against the reference's build."""
    N, length = 400, 10.0
    cells = lattice_spheroid(1_000_000, N * length / 2, 0, length, N)
    with ref_lib.RefSim("c2", 38.0, 1e5, 0.1) as ref, make_sim(N, length, cap=2_000_000) as sim:
        ref.set_cells(cells)
        ref.fm_update()
        sim.import_cells(cells)
        sim.FM_update()
        np.testing.assert_array_equal(sim.dump_keys(), ref.keys())
        s, e = sim.dump_se()
        rs, re_ = ref.se()
        np.testing.assert_array_equal(s, rs)
        np.testing.assert_array_equal(e, re_)
        got, exp = sim.export_cells(), ref.cells()
        np.testing.assert_array_equal(got["mesh_idx"], exp["mesh_idx"])
        np.testing.assert_allclose(got["pos"], exp["pos"], rtol=1e-5, atol=0)


def test_fm_full_size_sampled_vs_oracle():
    """10^6 cells, 400^3: sortedness and stability at full size, and the force of a sample of
    cells recomputed by the oracle from the sorted cells and the s/e arrays."""
    N, length = 400, 10.0
    cells = lattice_spheroid(1_000_000, N * length / 2, 0, length, N)
    P = ol.params(N=N, len=length, cap=2_000_000)
    with make_sim(N, length, cap=2_000_000) as sim:
        sim.import_cells(cells)
        sim.FM_update()
        keys, perm = sim.dump_keys(), sim.dump_perm()
        assert np.all(np.diff(keys) >= 0)
        same = keys[1:] == keys[:-1]
        assert np.all(perm[1:][same] > perm[:-1][same])  # stable
        assert np.array_equal(np.sort(perm), np.arange(len(perm)))
        s, e = sim.dump_se()
        out = sim.export_cells()
        sorted_in = cells[perm].copy()
        # keys and mesh_idx of the sorted input, as updateCellMeshIdx sets them
        ijk = (sorted_in["pos"] / np.float32(length)).astype(np.int32)
        sorted_in["mesh_idx"] = ijk[:, 0] + ijk[:, 1] * N + ijk[:, 2] * N * N
        rng = np.random.default_rng(0)
        for i in rng.choice(len(cells), 2000, replace=False):
            f = ol.force_one(sorted_in, int(i), P, s, e)
            assert np.array_equal(f.view(np.uint32), out["oldforce"][i].view(np.uint32)), i
