"""Self-checks of the oracle on the CPU: published known answers, invariants of the algorithms,
and the FP32 scheme against its FP64 restatement."""
import numpy as np

import oracle_lib as ol
from cases import ball_cells, one_per_voxel, random_field
from gell_b200.cells import CELL_DTYPE


def test_philox_known_answers():
    # Known-answer vectors published with Random123 for philox4x32-10
    kat = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for ctr, key, out in kat:
        np.testing.assert_array_equal(ol.philox(ctr, key), np.array(out, np.uint32))


def test_u01_range():
    L = ol.lib()
    assert L.go_u01(0) == np.float32(2.0 ** -24)
    assert L.go_u01(0xFFFFFFFF) == 1.0


def test_stable_sort_orders_sentinel_first_and_keeps_ties():
    N, length = 32, 10.0
    cells = ball_cells(N, length, 3000, seed=2)
    P = ol.params(N=N, len=length, cap=65536)
    c = cells.copy()
    keys, perm, s, e = ol.fm_update(c, P)
    assert np.all(np.diff(keys) >= 0)
    assert keys[0] == -1
    tie = keys[1:] == keys[:-1]
    assert np.all(perm[1:][tie] > perm[:-1][tie])
    # s/e cover exactly the live cells inside the grid
    live = c["sign"] == 1
    cover = np.zeros(len(c), bool)
    for v in np.nonzero(e >= 0)[0]:
        cover[s[v]:e[v] + 1] = True
    assert np.all(cover[live])


def test_force_is_antisymmetric_for_an_isolated_pair():
    N, length = 16, 10.0
    P = ol.params(N=N, len=length, cap=16)
    c = np.zeros(2, CELL_DTYPE)
    c["sign"] = 1
    c["pos"] = [[80.0, 80.0, 80.0], [87.0, 81.0, 80.5]]
    c["r"] = 5.0
    c["V"] = 500.0
    c["phase"] = 0
    ol.fm_update(c, P)
    np.testing.assert_allclose(c["oldforce"][0], -c["oldforce"][1], rtol=1e-6)
    # overlapping cells (d < r1 + r2) repel
    d = c["pos"][0] - c["pos"][1]
    assert np.dot(c["oldforce"][0], d) > 0


def test_lod_fp32_close_to_fp64_and_boundary_held():
    N, length = 24, 10.0
    cells = one_per_voxel(N, length, seed=1, lo=6, hi=18)
    rate = ol.prelod(cells, N, length, -10.0)
    field = random_field(N, seed=3)
    E, F = ol.mesh_init(N, length, 1e5, 0.1, 0.01)
    p32 = ol.lod_substeps(field, rate, E, F, N, 0.01, 38.0, 10)
    p64 = ol.lod_substeps_f64(field, rate, N, length, 1e5, 0.1, 0.01, 38.0, 10)
    assert np.max(np.abs(p32 - p64) / np.abs(p64)) < 1e-5
    # the z sweep runs last, so its end faces hold the boundary value; the x and y faces are
    # reset by the next substep's Setboundary (include/LODkernel.cuh:288)
    g = p32.reshape(N, N, N)  # [z][y][x]
    for face in (g[0], g[-1]):
        assert np.all(face == np.float32(38.0))


def test_lod_line_equals_full_sweep_definition():
    """go_thomas_line is the per-line kernel the sweeps apply."""
    N = 40
    rng = np.random.default_rng(0)
    E, F = ol.mesh_init(N, 10.0, 1e5, 0.1, 0.01)
    line = rng.uniform(0, 40, N).astype(np.float32)
    a = line.copy()
    ol.lib().go_thomas_line(a.ctypes.data, 1, E.ctypes.data, F.ctypes.data, N, 38.0)
    Y = np.zeros(N, np.float32)
    Y[0] = 38.0
    for i in range(1, N - 1):
        Y[i] = np.float32(np.float64(line[i]) - np.float64(E[i]) * np.float64(Y[i - 1]))
    x = np.zeros(N, np.float32)
    x[N - 1] = 38.0
    s = np.float32(E[1] * F[0])
    for i in range(N - 2, 0, -1):
        x[i] = np.float32(np.float32(np.float64(Y[i]) - np.float64(s) * np.float64(x[i + 1])) / F[i])
    x[0] = 38.0
    # fused multiply-adds round once: equal to the exact double evaluation rounded to float
    np.testing.assert_array_equal(a, x)


def test_death_is_stable_compaction():
    N, length = 16, 10.0
    c = ball_cells(N, length, 1000, seed=4, dead_frac=0.3)
    keep = c[c["sign"] == 1].copy()
    n = ol.death(c, len(c))
    assert n == len(keep)
    np.testing.assert_array_equal(c[:n].view(np.uint8), keep.view(np.uint8))


def test_birth_philox_appends_in_mother_order():
    N, length = 24, 10.0
    n = 800
    c = ball_cells(N, length, n, seed=5, outside=0, dead_frac=0.0)
    c["phase"] = 1
    c["cell_clock"] = 780.0
    buf = np.concatenate([c, np.zeros(n + 8, CELL_DTYPE)])
    P = ol.params(N=N, len=length, cap=len(buf) + 10)
    field = np.full(N ** 3, 38.0, np.float32)
    nn = ol.birth_philox(buf, n, P, field, 1, 0)
    assert nn == 2 * n
    d = buf[n:nn]
    m = buf[:n]
    assert np.all(d["phase"] == 2) and np.all(m["phase"] == 2)
    # each daughter and its mother sit symmetric about the mother's old position
    centre = (d["pos"].astype(np.float64) + m["pos"]) / 2
    np.testing.assert_allclose(centre, c["pos"], atol=1e-3)


def test_fm_fp32_close_to_fp64():
    """The FP32 restatement of forcekernel + movementkernel against its FP64 restatement: forces
    within 1e-5 of the largest force, positions within 1e-4 um."""
    from cases import ball_cells
    cells = ball_cells(32, 10.0, 3000, seed=7)
    P = ol.params(N=32, len=10.0, cap=6000)
    srt, f64, p64 = ol.force_move_f64(cells, P)
    c32 = cells.copy()
    ol.fm_update(c32, P)
    alive = (srt["sign"] != 0) & (c32["sign"] != 0)
    assert alive.sum() > 2500
    fs = np.abs(f64[alive]).max()
    assert np.abs(c32["oldforce"][alive] - f64[alive]).max() < 1e-5 * fs
    assert np.abs(c32["pos"][alive] - p64[alive]).max() < 1e-4
