"""gell_sort_keys_noalloc, the Morton-key sort for callers that cannot allocate device memory.

Hosts that capture CUDA streams into graphs, that keep to a device-memory budget reserved up
front, or that only own their input and output buffers cannot let the library call cudaMalloc.
This entry point keeps its scratch in a fixed array inside the library instead.  Its result must
equal the sort that gell_fm_update performs and the oracle's stable sort (integer keys and
permutation: bit for bit), on two calls in a row, since the calls share that scratch.  This file
is collected last, so a run that stops at the first failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

import oracle_lib as ol
from cases import ball_cells

pytestmark = pytest.mark.gpu

gb = pytest.importorskip("gell_b200")
torch = pytest.importorskip("torch")

GELL_ERR_INVALID_ARG, GELL_ERR_CAPACITY = -1, -2


def lib():
    L = gb.load_library()
    L.gell_sort_keys_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_void_p]
    L.gell_sort_keys_noalloc.restype = ctypes.c_int
    return L


def key_bits(N):
    """Bit length of (largest Morton key on an N^3 grid + 1)."""
    m = sum(((((N - 1) >> b) & 1) * 7) << (3 * b) for b in range(10))
    return int(m + 1).bit_length()


def sort_noalloc(keys: np.ndarray, bits: int):
    dk = torch.from_numpy(np.ascontiguousarray(keys, np.int32)).cuda()
    ok = torch.full_like(dk, -7)
    op = torch.full_like(dk, -7)
    st = lib().gell_sort_keys_noalloc(dk.data_ptr(), ok.data_ptr(), op.data_ptr(), len(keys), bits, None)
    torch.cuda.synchronize()
    assert st == 0, gb.api.STATUS_NAMES.get(st, st)
    return ok.cpu().numpy(), op.cpu().numpy()


def oracle_sort(keys: np.ndarray):
    """The oracle's stable sort by signed key (the reference's thrust::sort_by_key order)."""
    k = np.ascontiguousarray(keys, np.int32).copy()
    cells = np.zeros(len(k), gb.CELL_DTYPE)
    perm = np.zeros(len(k), np.int32)
    ol.lib().go_stable_sort(cells.ctypes.data, k.ctypes.data, len(k), perm.ctypes.data)
    return k, perm


def fm_update_sort(cells, N, length, cap):
    """Sorted keys and permutation from the existing entry point (gell_fm_update), and the
    unsorted keys of the same cells (the reference's updateCellMeshIdx, via the oracle)."""
    with gb.Simulation(voxel_num=N, voxel_length=length, max_cell_num=cap) as sim:
        sim.import_cells(cells)
        sim.FM_update()
        keys_sorted, perm = sim.dump_keys(), sim.dump_perm()
    c = cells.copy()
    keys = np.zeros(len(c), np.int32)
    ol.lib().go_update_keys(c.ctypes.data, len(c), ctypes.byref(ol.params(N=N, len=length, cap=cap)),
                            keys.ctypes.data)
    return keys, keys_sorted, perm


def test_noalloc_sort_matches_fm_update_twice():
    torch.cuda.set_device(0)
    N, length = 64, 10.0
    for seed in (3, 4):  # two calls in a row share the scratch
        cells = ball_cells(N, length, 60000, seed=seed, radius_frac=0.45)
        keys, exp_keys, exp_perm = fm_update_sort(cells, N, length, 65536)
        got_keys, got_perm = sort_noalloc(keys, key_bits(N))
        np.testing.assert_array_equal(got_keys, exp_keys)
        np.testing.assert_array_equal(got_perm, exp_perm)
        o_keys, o_perm = oracle_sort(keys)
        np.testing.assert_array_equal(got_keys, o_keys)
        np.testing.assert_array_equal(got_perm, o_perm)
        assert got_keys[0] == -1  # the cells outside the grid order first


def test_noalloc_sort_at_the_size_limit():
    torch.cuda.set_device(0)
    N, length = 400, 10.0
    n = 1 << 20
    cells = gb.lattice_spheroid(n, N * length / 2, 0, length, N)
    keys, exp_keys, exp_perm = fm_update_sort(cells, N, length, 2_000_000)
    o_keys, o_perm = oracle_sort(keys)
    np.testing.assert_array_equal(exp_keys, o_keys)
    np.testing.assert_array_equal(exp_perm, o_perm)
    for _ in range(2):
        got_keys, got_perm = sort_noalloc(keys, key_bits(N))
        np.testing.assert_array_equal(got_keys, exp_keys)
        np.testing.assert_array_equal(got_perm, exp_perm)


@pytest.mark.parametrize("bits,n", [(8, 5000), (24, 300_000), (32, 70_000), (17, 1 << 20)])
def test_noalloc_sort_digit_widths_against_oracle(bits, n):
    """One pass (8 bits), 3 passes of 8-bit digits (24), 4 passes of 8 bits (32) and 3 passes of
    6 bits (17): random keys in [-1, 2^bits - 1) with many repeats, each sorted twice in a row."""
    torch.cuda.set_device(0)
    rng = np.random.default_rng(bits * 1000 + n)
    hi = (1 << bits) - 1  # key + 1 < 2^bits
    keys = rng.integers(-1, min(hi, 1 << 31) - 1, n, dtype=np.int64)
    keys[rng.random(n) < 0.3] = -1  # many cells outside the grid
    keys[: n // 10] = keys[n // 10: 2 * (n // 10)]  # repeated keys: stability matters
    keys = keys.astype(np.int32)
    o_keys, o_perm = oracle_sort(keys)
    np.testing.assert_array_equal(o_perm, np.argsort(keys, kind="stable"))
    for _ in range(2):
        got_keys, got_perm = sort_noalloc(keys, bits)
        np.testing.assert_array_equal(got_keys, o_keys)
        np.testing.assert_array_equal(got_perm, o_perm)


def test_noalloc_sort_rejects_aliased_buffers():
    torch.cuda.set_device(0)
    n = 4096
    a = torch.zeros(3 * n, dtype=torch.int32, device="cuda")
    k, s, p = a[:n], a[n:2 * n], a[2 * n:]
    L = lib()
    assert L.gell_sort_keys_noalloc(k.data_ptr(), s.data_ptr(), p.data_ptr(), n, 19, None) == 0
    half = a[n // 2: n // 2 + n]  # overlaps the second half of keys
    for keys, out, perm in ((k, k, p), (k, s, k), (k, s, s), (k, half, p)):
        st = L.gell_sort_keys_noalloc(keys.data_ptr(), out.data_ptr(), perm.data_ptr(), n, 19, None)
        assert st == GELL_ERR_INVALID_ARG
    torch.cuda.synchronize()


def test_noalloc_sort_rejects_too_many_keys():
    torch.cuda.set_device(0)
    n = (1 << 20) + 1
    dk = torch.zeros(n, dtype=torch.int32, device="cuda")
    do = torch.zeros(n, dtype=torch.int32, device="cuda")
    dp = torch.zeros(n, dtype=torch.int32, device="cuda")
    st = lib().gell_sort_keys_noalloc(dk.data_ptr(), do.data_ptr(), dp.data_ptr(), n, 28, None)
    assert st == GELL_ERR_CAPACITY
    assert lib().gell_sort_keys_noalloc(None, None, None, 5, 28, None) == GELL_ERR_INVALID_ARG
    assert lib().gell_sort_keys_noalloc(dk.data_ptr(), do.data_ptr(), dp.data_ptr(), 5, 0, None) == GELL_ERR_INVALID_ARG
