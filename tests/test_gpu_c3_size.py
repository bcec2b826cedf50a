"""Parity at the size of the birth/death workload: 600^3 voxels, millions of cells.

At this size the kernels take paths that smaller grids never reach:
* the radix sort of the Morton keys uses 8-bit digits (30 key bits at N = 600, so 4 passes of 8;
  N <= 400 gives 28 bits in 4 passes of 7);
* a line of the LOD sweeps is 19 groups of 32, so fewer line tiles fit per SM;
* birth and death scan and compact millions of flags over many blocks.

Checks: keys, s/e cell list and sorted cells against the reference's own build at 600^3
(include/FMkernel.cuh:22-53,181-202) and the permutation against the oracle's stable sort; both
substrates' fields after two substeps bit-exact against the oracle (include/LODkernel.cuh:24-136);
Philox birth and death compaction against the oracle (include/PDkernel.cuh:27-117)."""
import numpy as np
import pytest

import oracle_lib as ol
import ref_lib
from cases import one_per_voxel
from gell_b200.cells import CELL_DTYPE, lattice_spheroid, seed_ki67_states

pytestmark = pytest.mark.gpu

gb = pytest.importorskip("gell_b200")

N, LENGTH = 600, 10.0


def raw(c):
    return np.ascontiguousarray(c).view(np.uint8).reshape(len(c), CELL_DTYPE.itemsize)


def bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.skipif(not ref_lib.available("c3"), reason="reference build oracle/_ref missing")
def test_c3_keys_sort_and_cell_list_vs_reference():
    n = 2_500_000
    cells = lattice_spheroid(n, N * LENGTH / 2, 3, LENGTH, N)
    # a few cells outside the grid: key -1, ordered first
    cells["pos"][:5] = np.array([[-3, 10, 10], [6001, 10, 10], [10, -0.5, 10], [10, 10, 7000], [-20, -20, -20]],
                                np.float32)
    # and a few near the far corners, so the top digit of the 30-bit keys is not always zero
    cells["pos"][5:9] = np.array([[5995, 5995, 5995], [5, 5995, 5995], [5995, 5, 5995], [5995, 5995, 5]],
                                 np.float32)
    with ref_lib.RefSim("c3", 38.0, 1e5, 0.1) as ref, \
            gb.Simulation(voxel_num=N, voxel_length=LENGTH, max_cell_num=ref.cap) as sim:
        ref.set_cells(cells)
        ref.fm_update()
        sim.import_cells(cells)
        sim.FM_update()
        keys = sim.dump_keys()
        np.testing.assert_array_equal(keys, ref.keys())
        assert keys[0] == -1 and keys.max() >= (1 << 29)  # the top 8-bit digit is exercised
        s, e = sim.dump_se()
        rs, re_ = ref.se()
        np.testing.assert_array_equal(s, rs)
        np.testing.assert_array_equal(e, re_)
        got, exp = sim.export_cells(), ref.cells()
        for f in ("sign", "mesh_idx", "r", "V", "phase"):
            np.testing.assert_array_equal(got[f], exp[f], err_msg=f)
        np.testing.assert_allclose(got["pos"], exp["pos"], rtol=1e-5, atol=0)
        perm = sim.dump_perm()
    oc = cells.copy()
    okeys, operm, _, _ = ol.fm_update(oc, ol.params(N=N, len=LENGTH, cap=4_000_000))
    np.testing.assert_array_equal(perm, operm)
    np.testing.assert_array_equal(keys, okeys)


def test_c3_fields_two_substrates_two_substeps_vs_oracle():
    cells = one_per_voxel(N, LENGTH, seed=9, lo=200, hi=400)  # 8*10^6 cells, one per voxel
    rng = np.random.Generator(np.random.Philox(41))
    field = rng.uniform(10.0, 38.0, N ** 3).astype(np.float32)
    with gb.Simulation(voxel_num=N, voxel_length=LENGTH, max_cell_num=len(cells) + 1024) as sim:
        sim.add_substrate(gb.oxygen())
        sim.add_substrate(gb.drug())
        sim.set_field(0, field)
        sim.set_field(1, field / 38.0)
        sim.import_cells(cells)
        sim.PreLOD()
        sim.LODsolver(2)
        got = [sim.field(0), sim.field(1)]
    for sub, s in enumerate((gb.oxygen(), gb.drug())):
        rate = ol.prelod(cells, N, LENGTH, s.uptake)
        E, F = ol.mesh_init(N, LENGTH, s.diffusion, s.decay, 0.01)
        start = field if sub == 0 else field / 38.0
        exp = ol.lod_substeps(start, rate, E, F, N, 0.01, s.boundary, 2)
        assert bits_equal(got[sub], exp), f"substrate {sub}"


def test_c3_birth_and_death_philox_vs_oracle():
    n, cap = 1_500_000, 4_000_000
    cells = lattice_spheroid(n, N * LENGTH / 2, 7, LENGTH, N)
    seed_ki67_states(cells, 19)
    rng = np.random.Generator(np.random.Philox(43))
    field = rng.uniform(0.0, 14.0, N ** 3).astype(np.float32)  # proliferation and necrosis ramps
    with gb.Simulation(voxel_num=N, voxel_length=LENGTH, max_cell_num=cap,
                       rng_mode=gb.GELL_RNG_PHILOX, seed=4242) as sim:
        sim.add_substrate(gb.oxygen())
        sim.set_field(0, field)
        sim.import_cells(cells)
        nb = sim.CellBirth_kernel()
        born = sim.export_cells()
        nd = sim.CellDeath_kernel()
        survived = sim.export_cells()
    oc = np.concatenate([cells, gb.empty_cells(cap - n)])
    on = ol.birth_philox(oc, n, ol.params(N=N, len=LENGTH, cap=cap), field, 4242, 0)
    assert nb == on and nb > n + 1000, (nb, on)
    exp = oc[:on]
    for f in ("sign", "mesh_idx", "phase", "force", "oldforce"):
        np.testing.assert_array_equal(born[f], exp[f], err_msg=f)
    for f in ("V", "Vf", "Vcs", "Vns", "cell_clock"):
        np.testing.assert_array_equal(born[f].view(np.uint32), exp[f].view(np.uint32), err_msg=f)
    np.testing.assert_allclose(born["r"], exp["r"], rtol=1e-6)
    np.testing.assert_allclose(born["pos"], exp["pos"], rtol=1e-6, atol=1e-4)
    # death compacts what birth left, as the GPU holds it: bit-exact
    dc = born.copy()
    odn = ol.death(dc, len(dc))
    assert nd == odn and nd < nb, (nd, odn, nb)
    np.testing.assert_array_equal(raw(survived), raw(dc[:odn]))
