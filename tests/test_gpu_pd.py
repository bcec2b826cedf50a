"""Birth and death on the GPU against the oracle (Philox draws) and the reference (curand XORWOW).

Death is a stable compaction: bit-exact.  Birth with Philox draws: every mother and daughter field
matches the oracle bit for bit except positions and radii, which go through sinf/cosf/acosf and
pow (CUDA's versus the host's) and agree within 1e-6 relative.  Birth with the reference's own
XORWOW draws: mothers match the reference's kernel, daughters match as a set (the reference
appends them in atomic order).
"""
import numpy as np
import pytest

import oracle_lib as ol
import ref_lib
from cases import ball_cells, canonical
from gell_b200.cells import CELL_DTYPE

pytestmark = pytest.mark.gpu

gb = pytest.importorskip("gell_b200")

FLOATS = ("r", "V", "Vf", "Vcs", "Vns", "cell_clock")


def raw(c):
    return np.ascontiguousarray(c).view(np.uint8).reshape(len(c), CELL_DTYPE.itemsize)


def eventful_cells(N, length, n, seed):
    """Cells spread over phases and clocks so one biology step divides, kills and changes phase."""
    c = ball_cells(N, length, n, seed, outside=0)
    rng = np.random.Generator(np.random.Philox(seed + 100))
    c["phase"] = rng.choice([0, 0, 1, 1, 2, 3, 4, 5], n)
    c["cell_clock"] = rng.choice(np.array([0, 144, 774, 780, 800], np.float32), n)
    low = rng.random(n) < 0.2
    c["Vcs"][low] = np.float32(20.0)
    return c


def o2_field(N, seed):
    rng = np.random.Generator(np.random.Philox(seed))
    return rng.uniform(0.0, 12.0, N ** 3).astype(np.float32)


def test_death_bit_exact():
    N, length = 32, 10.0
    cells = ball_cells(N, length, 5000, seed=3, dead_frac=0.3)
    with gb.Simulation(voxel_num=N, voxel_length=length, max_cell_num=65536) as sim:
        sim.import_cells(cells)
        n = sim.CellDeath_kernel()
        oc = cells.copy()
        on = ol.death(oc, len(oc))
        assert n == on
        np.testing.assert_array_equal(raw(sim.export_cells()), raw(oc[:on]))


def test_death_empty_and_all_dead():
    N, length = 32, 10.0
    with gb.Simulation(voxel_num=N, voxel_length=length, max_cell_num=1024) as sim:
        sim.import_cells(gb.empty_cells(0))
        assert sim.CellDeath_kernel() == 0
        c = ball_cells(N, length, 300, seed=1, outside=0)
        c["sign"] = 0
        sim.import_cells(c)
        assert sim.CellDeath_kernel() == 0


@pytest.mark.parametrize("cap", [65536, 2700])
def test_birth_philox_vs_oracle(cap):
    N, length = 32, 10.0
    n = 2500
    cells = eventful_cells(N, length, n, seed=4)
    field = o2_field(N, 5)
    with gb.Simulation(voxel_num=N, voxel_length=length, max_cell_num=cap,
                       rng_mode=gb.GELL_RNG_PHILOX, seed=77) as sim:
        sim.add_substrate(gb.oxygen())
        sim.set_field(0, field)
        sim.import_cells(cells)
        nn = sim.CellBirth_kernel()
        got = sim.export_cells()
        oc = np.concatenate([cells, gb.empty_cells(cap)])[:max(cap, n)].copy()
        P = ol.params(N=N, len=length, cap=cap)
        on = ol.birth_philox(oc, n, P, field, 77, 0)
        assert nn == on and nn > n, (nn, on)
        exp = oc[:on]
        for f in ("sign", "mesh_idx", "phase", "force", "oldforce"):
            np.testing.assert_array_equal(got[f], exp[f], err_msg=f)
        for f in ("V", "Vf", "Vcs", "Vns", "cell_clock"):
            np.testing.assert_array_equal(got[f].view(np.uint32), exp[f].view(np.uint32), err_msg=f)
        np.testing.assert_allclose(got["r"], exp["r"], rtol=1e-6)
        np.testing.assert_allclose(got["pos"], exp["pos"], rtol=1e-6, atol=1e-4)
        if cap == 2700:
            assert nn == cap - 1  # capacity reached: the reference stops at Max_Cell_num - 1


@pytest.mark.skipif(not ref_lib.available("t32"), reason="reference build oracle/_ref missing")
def test_birth_xorwow_vs_reference_kernels():
    N, length = 32, 10.0
    n = 3000
    cells = eventful_cells(N, length, n, seed=6)
    field = o2_field(N, 8)
    with ref_lib.RefSim("t32", 38.0, 1e5, 0.1) as ref, \
            gb.Simulation(voxel_num=N, voxel_length=length, max_cell_num=ref.cap) as sim:
        ref.set_cells(cells)
        ref.set_field(field)
        rn = ref.birth()
        sim.add_substrate(gb.oxygen())
        sim.set_field(0, field)
        sim.import_cells(cells)
        nn = sim.CellBirth_kernel()
        assert nn == rn and nn > n
        got, exp = sim.export_cells(), ref.cells()
        m_same = np.mean(np.all(raw(got[:n]) == raw(exp[:n]), 1))
        print(f"mother records bit-identical with the reference kernel: {m_same:.6f}")
        for f in ("sign", "phase", "mesh_idx"):
            np.testing.assert_array_equal(got[f][:n], exp[f][:n], err_msg=f)
        for f in FLOATS:
            np.testing.assert_allclose(got[f][:n], exp[f][:n], rtol=1e-6, err_msg=f)
        np.testing.assert_allclose(got["pos"][:n], exp["pos"][:n], rtol=1e-6)
        gd, ed = canonical(got[n:]), canonical(exp[n:])
        d_same = np.mean(np.all(raw(gd) == raw(ed), 1))
        print(f"daughter records bit-identical as a set: {d_same:.6f}")
        np.testing.assert_allclose(gd["pos"], ed["pos"], rtol=1e-6)
        for f in FLOATS:
            np.testing.assert_allclose(gd[f], ed[f], rtol=1e-6, err_msg=f)


@pytest.mark.skipif(not ref_lib.available("t32"), reason="reference build oracle/_ref missing")
def test_death_vs_reference_kernel():
    N, length = 32, 10.0
    cells = ball_cells(N, length, 4000, seed=12, dead_frac=0.4)
    with ref_lib.RefSim("t32", 38.0, 1e5, 0.1) as ref, \
            gb.Simulation(voxel_num=N, voxel_length=length, max_cell_num=ref.cap) as sim:
        ref.set_cells(cells)
        rn = ref.death()
        sim.import_cells(cells)
        assert sim.CellDeath_kernel() == rn
        np.testing.assert_array_equal(raw(sim.export_cells()), raw(ref.cells()))


def test_birth_counts_chi_squared_over_seeds():
    """Birth/death event counts over 1000 independent Philox draws (successive biology steps of
    one context, so successive counters) against the binomial law of the Ki-67 probabilities at
    O2 = 38: proliferation 6/510 and apoptosis 6/10080 per biology step."""
    N, length = 32, 10.0
    n = 4000
    base = ball_cells(N, length, n, seed=1, outside=0, dead_frac=0.0)
    base["phase"] = 0
    base["cell_clock"] = 0.0
    p_pro = float(np.float32((1.0 / 8.5 / 60.0) * 6.0))
    p_apo = float(np.float32((1.0 / 7.0 / 24.0 / 60.0) * 6.0))
    pro, apo = [], []
    with gb.Simulation(voxel_num=N, voxel_length=length, max_cell_num=65536,
                       rng_mode=gb.GELL_RNG_PHILOX, seed=2024) as sim:
        sim.add_substrate(gb.oxygen())
        for _ in range(1000):
            sim.import_cells(base)
            sim.CellBirth_kernel()
            out = sim.export_cells()
            pro.append(int((out["phase"] == 1).sum()))
            apo.append(int((out["phase"] == 3).sum()))
    for obs, p in ((np.array(pro), p_pro), (np.array(apo), p_apo)):
        mean, var = n * p, n * p * (1 - p)
        chi2 = float(np.sum((obs - mean) ** 2 / var))
        # 1000 degrees of freedom: mean 1000, sd ~45; reject beyond ~5 sd
        assert 780 < chi2 < 1230, (chi2, obs.mean(), mean)
        assert abs(obs.mean() - mean) < 5 * np.sqrt(var / len(obs))


def ki67_probabilities(o2):
    """Per-biology-step probabilities of Cell::Phase_update_ki67adv (include/Cells.cuh:145-165) at
    oxygen level o2, computed as the reference does (float ramps times double rates, stored as
    float): proliferation, apoptosis, necrosis."""
    f = np.float32
    pro = float(f(f(f(1.0) * (f(o2) - f(5.0))) / (f(10.0) - f(5.0))) * (1.0 / 8.5 / 60.0) * 6.0)
    if o2 > 10.0:
        pro = float(f((1.0 / 8.5 / 60.0) * 6.0))
    elif o2 < 5.0:
        pro = 0.0
    apo = float(f((1.0 / 7.0 / 24.0 / 60.0) * 6.0))
    nec = float(f(f(f(1.0) * (f(5.0) - f(o2))) / (f(5.0) - f(2.5))) * (1.0 / 6.0 / 60.0) * 6.0)
    if o2 > 5.0:
        nec = 0.0
    elif o2 < 2.5:
        nec = float(f((1.0 / 6.0 / 60.0) * 6.0))
    return pro, apo, nec


@pytest.mark.parametrize("o2", [2.0, 4.0, 7.0, 12.0])
def test_phase_transitions_chi_squared_on_the_oxygen_ramps(o2):
    """Quiescent cells at a uniform oxygen level inside the proliferation ramp (7), above it (12),
    inside the necrosis ramp (4) and below it (2): counts of the three stochastic transitions over
    1000 Philox draws (successive biology steps) against their binomial laws.  A second population of
    dead cells, half of them shrinking below the removal threshold in this step, checks the removal
    count of CellDeath_kernel against the oracle on every draw."""
    N, length = 32, 10.0
    n = 4000
    base = ball_cells(N, length, n, seed=31, outside=0, dead_frac=0.0)
    base["phase"] = 0
    base["cell_clock"] = 0.0
    nd = 400
    dead = ball_cells(N, length, nd, seed=32, outside=0, dead_frac=0.0)
    dead["phase"] = 3
    dead["Vcs"] = np.where(np.arange(nd) % 2 == 0, np.float32(24.0), np.float32(400.0))
    cells = np.concatenate([base, dead])
    # oracle: which dead cells are removed (deterministic: Volume_update, then Vcs <= 24.4)
    oc = np.concatenate([cells, gb.empty_cells(2 * len(cells))])
    field = np.full(N ** 3, o2, np.float32)
    ol.birth_philox(oc, len(cells), ol.params(N=N, len=length, cap=len(oc)), field, 5, 0)
    removed_exp = int((oc["sign"][n:len(cells)] == 0).sum())
    assert 0 < removed_exp < nd
    p = ki67_probabilities(o2)
    counts = {1: [], 3: [], 4: []}
    with gb.Simulation(voxel_num=N, voxel_length=length, max_cell_num=65536,
                       rng_mode=gb.GELL_RNG_PHILOX, seed=9000 + int(o2 * 10)) as sim:
        sim.add_substrate(gb.oxygen())
        sim.set_field(0, field)
        for _ in range(1000):
            sim.import_cells(cells)
            nb = sim.CellBirth_kernel()
            out = sim.export_cells()
            for ph in counts:
                counts[ph].append(int((out["phase"][:n] == ph).sum()))
            assert nb == len(cells)  # quiescent cells do not divide within the step
            assert sim.CellDeath_kernel() == len(cells) - removed_exp
    for ph, prob in zip((1, 3, 4), p):
        obs = np.array(counts[ph])
        if prob == 0.0:
            assert obs.sum() == 0, ph
            continue
        mean, var = n * prob, n * prob * (1 - prob)
        chi2 = float(np.sum((obs - mean) ** 2 / var))
        # 1000 degrees of freedom: mean 1000, sd ~45-50; reject beyond ~5 sd
        assert 760 < chi2 < 1250, (ph, chi2, obs.mean(), mean)
        assert abs(obs.mean() - mean) < 5 * np.sqrt(var / len(obs)), (ph, obs.mean(), mean)


@pytest.mark.skipif(not ref_lib.available("t32"), reason="reference build oracle/_ref missing")
def test_volume_update_contraction_vs_reference_device():
    """Cell::Volume_update as the reference's device build computes it (include/Cells.cuh:91-143),
    on 2^20 random cells over all phases, against the oracle's restatements of the possible
    multiply-add fusions.  The one the kernels use (GO_VOL_DEVICE_REF) must match every bit."""
    n = 1 << 20
    rng = np.random.Generator(np.random.Philox(5))
    c = np.zeros(n, CELL_DTYPE)
    c["sign"] = 1
    c["phase"] = rng.integers(0, 6, n)
    c["V"] = rng.uniform(100, 6000, n).astype(np.float32)
    c["Vf"] = rng.uniform(0, 4000, n).astype(np.float32)
    c["Vns"] = rng.uniform(0, 600, n).astype(np.float32)
    c["Vcs"] = rng.uniform(0, 2000, n).astype(np.float32)
    dev = c.copy()
    assert ref_lib.lib("t32").gref_volume_update_device(dev.ctypes.data, n) == 0
    L = ol.lib()
    res = {}
    for name, mode in (("device", ol.GO_VOL_DEVICE), ("device_fused", ol.GO_VOL_DEVICE_FUSED),
                       ("swap", ol.GO_VOL_DEVICE_SWAP), ("swap_fused", ol.GO_VOL_DEVICE_SWAP_FUSED),
                       ("reference", ol.GO_VOL_DEVICE_REF)):
        o = c.copy()
        L.go_volume_update_modes(o.ctypes.data, n, mode)
        same = np.ones(n, bool)
        for f in ("Vf", "Vns", "Vcs", "V"):
            same &= o[f].view(np.uint32) == dev[f].view(np.uint32)
        res[name] = float(same.mean())
    print("Volume_update bit-match with the reference device build:", res)
    assert res["reference"] == 1.0
