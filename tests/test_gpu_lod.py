"""LOD reaction-diffusion on the GPU against the oracle and the reference's own kernels.

The CUDA path is called through the C ABI (gell_b200.Simulation).  With one cell per voxel the
uptake map is order-independent, so the fields must match the oracle bit for bit; with several
cells per voxel both the reference and gell_b200 sum with float atomics, so fields agree within
1e-5 relative.
"""
import numpy as np
import pytest

import oracle_lib as ol
import ref_lib
from cases import ball_cells, one_per_voxel, random_field

pytestmark = pytest.mark.gpu

gb = pytest.importorskip("gell_b200")


def make_sim(N, length, cap=65536, subs=("o2",), **kw):
    sim = gb.Simulation(voxel_num=N, voxel_length=length, max_cell_num=cap, **kw)
    for s in subs:
        sim.add_substrate(gb.oxygen() if s == "o2" else gb.drug())
    return sim


def bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("N", [32, 37, 100])
def test_ef_prefactor_bit_exact(N):
    with make_sim(N, 10.0, subs=("o2", "drug")) as sim:
        for sub, s in enumerate((gb.oxygen(), gb.drug())):
            E, F = sim.dump_ef(sub)
            oE, oF = ol.mesh_init(N, 10.0, s.diffusion, s.decay, 0.01)
            assert bits_equal(E, oE) and bits_equal(F, oF)


@pytest.mark.parametrize("N,k", [(32, 1), (32, 10), (37, 3), (64, 2), (100, 3), (131, 2)])
def test_lod_bit_exact_one_cell_per_voxel(N, k):
    """N >= 100 reaches the groups whose Thomas factors have converged (uniform-group path)."""
    length = 10.0
    cells = one_per_voxel(N, length, seed=N, lo=N // 4, hi=N // 4 + N // 2)
    field = random_field(N, seed=7)
    with make_sim(N, length, cap=max(65536, len(cells)), subs=("o2", "drug")) as sim:
        sim.set_field(0, field)
        sim.set_field(1, field * 0.03)
        sim.import_cells(cells)
        sim.PreLOD()
        sim.LODsolver(k)
        for sub, s in enumerate((gb.oxygen(), gb.drug())):
            rate = ol.prelod(cells, N, length, s.uptake)
            assert bits_equal(sim.dump_rate(sub), rate)
            E, F = ol.mesh_init(N, length, s.diffusion, s.decay, 0.01)
            start = field if sub == 0 else field * 0.03
            exp = ol.lod_substeps(start, rate, E, F, N, 0.01, s.boundary, k)
            assert bits_equal(sim.field(sub), exp), f"substrate {sub}"


def test_lod_single_substrate_call_leaves_other_untouched():
    N, length = 32, 10.0
    field = random_field(N, seed=3)
    with make_sim(N, length, subs=("o2", "drug")) as sim:
        sim.set_field(0, field)
        sim.set_field(1, field)
        sim.LODsolver(2, sub=1)
        assert bits_equal(sim.field(0), field)
        E, F = ol.mesh_init(N, length, 5e4, 0.05, 0.01)
        exp = ol.lod_substeps(field, np.zeros(N ** 3, np.float32), E, F, N, 0.01, 1.0, 2)
        assert bits_equal(sim.field(1), exp)


def test_lod_many_cells_per_voxel_within_tolerance():
    N, length = 32, 10.0
    cells = ball_cells(N, length, 6000, seed=11, dead_frac=0.1)
    cells["phase"] = np.random.default_rng(1).choice([0, 1, 2, 3, 4, 5], len(cells))
    field = random_field(N, seed=5)
    with make_sim(N, length) as sim:
        sim.set_field(0, field)
        sim.import_cells(cells)
        sim.PreLOD()
        sim.LODsolver(10)
        rate = ol.prelod(cells, N, length, -10.0)
        np.testing.assert_allclose(sim.dump_rate(0), rate, rtol=1e-5, atol=1e-6)
        E, F = ol.mesh_init(N, length, 1e5, 0.1, 0.01)
        exp = ol.lod_substeps(field, rate, E, F, N, 0.01, 38.0, 10)
        np.testing.assert_allclose(sim.field(0), exp, rtol=1e-5, atol=0)


def test_lod_accuracy_vs_fp64():
    """FP32 LOD against the FP64 restatement of the same scheme (reported, loose bound)."""
    N, length = 32, 10.0
    cells = one_per_voxel(N, length, seed=2, lo=8, hi=24)
    field = random_field(N, seed=9)
    with make_sim(N, length) as sim:
        sim.set_field(0, field)
        sim.import_cells(cells)
        sim.PreLOD()
        sim.LODsolver(10)
        rate = ol.prelod(cells, N, length, -10.0)
        exp64 = ol.lod_substeps_f64(field, rate, N, length, 1e5, 0.1, 0.01, 38.0, 10)
        err = np.max(np.abs(sim.field(0) - exp64) / np.maximum(np.abs(exp64), 1e-3))
        print(f"max relative error vs FP64 after 10 substeps: {err:.3e}")
        assert err < 1e-4


@pytest.mark.skipif(not ref_lib.available("t32"), reason="reference build oracle/_ref missing")
def test_lod_vs_reference_kernels():
    """The reference's own Setboundary/meshupdate/LODkernel_x/y/z on the same input."""
    N, length = 32, 10.0
    cells = one_per_voxel(N, length, seed=4, lo=6, hi=26)
    field = random_field(N, seed=8)
    with ref_lib.RefSim("t32", 38.0, 1e5, 0.1) as ref, make_sim(N, length) as sim:
        E, F = ref.ef()
        gE, gF = sim.dump_ef(0)
        assert bits_equal(E, gE) and bits_equal(F, gF)
        ref.set_cells(cells)
        ref.set_field(field)
        ref.prelod()
        ref.lodsolver(10)
        sim.set_field(0, field)
        sim.import_cells(cells)
        sim.PreLOD()
        sim.LODsolver(10)
        assert bits_equal(sim.dump_rate(0), ref.rate())
        got, exp = sim.field(0), ref.field()
        same = np.mean(got.view(np.uint32) == exp.view(np.uint32))
        print(f"bit-identical voxels vs reference kernels: {same:.6f}")
        np.testing.assert_allclose(got, exp, rtol=1e-5, atol=0)


@pytest.mark.skipif(not ref_lib.available("t32d"), reason="reference build oracle/_ref missing")
def test_drug_vs_reference_kernels():
    N, length = 32, 10.0
    cells = ball_cells(N, length, 3000, seed=21)
    field = random_field(N, seed=12, lo=0.0, hi=1.0)
    with ref_lib.RefSim("t32d", 1.0, 5e4, 0.05) as ref, make_sim(N, length, subs=("drug",)) as sim:
        ref.set_cells(cells)
        ref.set_field(field)
        ref.prelod()
        ref.lodsolver(10)
        sim.set_field(0, field)
        sim.import_cells(cells)
        sim.PreLOD()
        sim.LODsolver(10)
        np.testing.assert_allclose(sim.field(0), ref.field(), rtol=1e-5, atol=0)


def test_lod_full_size_two_substrates_vs_oracle():
    """400^3, both substrates, two substeps: the size of the large workload, against the oracle."""
    N, length = 400, 10.0
    cells = one_per_voxel(N, length, seed=5, lo=150, hi=250)
    rng = np.random.Generator(np.random.Philox(31))
    field = rng.uniform(10.0, 38.0, N ** 3).astype(np.float32)
    with make_sim(N, length, cap=1_100_000, subs=("o2", "drug")) as sim:
        sim.set_field(0, field)
        sim.set_field(1, field / 38.0)
        sim.import_cells(cells)
        sim.PreLOD()
        sim.LODsolver(2)
        for sub, s in enumerate((gb.oxygen(), gb.drug())):
            rate = ol.prelod(cells, N, length, s.uptake)
            E, F = ol.mesh_init(N, length, s.diffusion, s.decay, 0.01)
            start = field if sub == 0 else field / 38.0
            exp = ol.lod_substeps(start, rate, E, F, N, 0.01, s.boundary, 2)
            assert bits_equal(sim.field(sub), exp), f"substrate {sub}"


def test_markstein_division_matches_ieee():
    """The back substitution divides with a precomputed reciprocal and two residual corrections;
    it must equal IEEE round-to-nearest division bit for bit."""
    with make_sim(16, 10.0, cap=16) as sim:
        assert sim.selftest_division(1 << 26, seed=11) == 0
        assert sim.selftest_division(1 << 26, seed=12) == 0


@pytest.mark.parametrize("N", [100, 160])
def test_exact_chain_option_gives_identical_fields(N):
    """The back substitution's speculative chain is verified against the exact one and redone
    where they differ; forcing the exact chain everywhere must give the same bits."""
    length = 10.0
    cells = one_per_voxel(N, length, seed=N + 1, lo=N // 4, hi=N // 4 + N // 2)
    field = random_field(N, seed=17)
    out = []
    for exact in (False, True):
        with make_sim(N, length, cap=max(65536, len(cells)), subs=("o2", "drug")) as sim:
            sim.set_exact_chain(exact)
            sim.set_field(0, field)
            sim.set_field(1, field * 0.03)
            sim.import_cells(cells)
            sim.PreLOD()
            sim.LODsolver(3)
            out.append((sim.field(0), sim.field(1)))
    for a, b in zip(out[0], out[1]):
        assert bits_equal(a, b)
    rate = ol.prelod(cells, N, length, -10.0)
    E, F = ol.mesh_init(N, length, 1e5, 0.1, 0.01)
    assert bits_equal(out[1][0], ol.lod_substeps(field, rate, E, F, N, 0.01, 38.0, 3))
