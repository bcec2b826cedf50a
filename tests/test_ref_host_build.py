"""The CPU baseline is the reference's own FM and LOD kernel bodies compiled for the host
(oracle/ref_host_harness.cpp, oracle/make_ref_host.py).  These CPU tests check that this build
computes what the reference computes, against the oracle, on a 32^3 grid:

* FM_update: the same sort (cell order), the same cells leaving the grid, forces and moved
  positions within FP32 rounding (g++ fuses multiply-adds differently from nvcc);
* PreLOD + LODsolver: the same field within 1e-5 relative.

It is only a baseline for timing, so nothing here is bit-exact by design."""
import os
import sys

import numpy as np
import pytest

import oracle_lib as ol
from cases import ball_cells, random_field

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import reference_build as rb  # noqa: E402

pytestmark = pytest.mark.skipif(not rb.host_available("t32"),
                                reason="host build of the reference not present (make -C oracle host)")

N, LENGTH = 32, 10.0


def test_host_build_fm_update_matches_oracle():
    cells = ball_cells(N, LENGTH, 4000, seed=21)
    with rb.HostRefSim("t32", 38.0, 1e5, 0.1) as h:
        assert h.N == N
        h.set_cells(cells)
        h.fm_update()
        got = h.cells()
    exp = cells.copy()
    ol.fm_update(exp, ol.params(N=N, len=LENGTH, cap=65536))
    np.testing.assert_array_equal(got["sign"], exp["sign"])
    np.testing.assert_array_equal(got["r"], exp["r"])  # same cells in the same (sorted) order
    live = exp["sign"] == 1
    np.testing.assert_array_equal(got["mesh_idx"][live], exp["mesh_idx"][live])
    np.testing.assert_allclose(got["pos"][live], exp["pos"][live], rtol=0, atol=1e-4)
    np.testing.assert_allclose(got["oldforce"][live], exp["oldforce"][live], rtol=1e-4, atol=1e-5)


def test_host_build_lod_matches_oracle():
    cells = ball_cells(N, LENGTH, 3000, seed=22)
    field = random_field(N, seed=23)
    with rb.HostRefSim("t32", 38.0, 1e5, 0.1) as h:
        h.set_cells(cells)
        h.fm_update()
        moved = h.cells()
        h.set_field(field)
        h.prelod()
        h.lodsolver(3)
        got = h.field()
    rate = ol.prelod(moved, N, LENGTH, -10.0)
    E, F = ol.mesh_init(N, LENGTH, 1e5, 0.1, 0.01)
    exp = ol.lod_substeps(field, rate, E, F, N, 0.01, 38.0, 3)
    np.testing.assert_allclose(got, exp, rtol=1e-5, atol=0)


def test_host_launch_rewrite_keeps_everything_but_the_launch_syntax():
    import make_ref_host as mk
    src = ("void f() {\n  k1 << <(n + 63) / 64, 64 >> > (a, b[i], g(c, d));\n"
           "  k2<<<grid, blk>>>(p);\n  int x = 1 << 3;\n}\n")
    out, n = mk.rewrite_launches(src)
    assert n == 2
    assert "gref_host_launch((n + 63) / 64, 64, [&] { k1(a, b[i], g(c, d)); });" in out
    assert "gref_host_launch(grid, blk, [&] { k2(p); });" in out
    assert "int x = 1 << 3;" in out
