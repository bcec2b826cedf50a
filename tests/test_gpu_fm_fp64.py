"""Mechanics on the GPU against the FP64 restatement of the force and movement kernels: the FP32
forces and moved positions of one FM_update (bit-identical with the reference's FP32 kernels, as
the parity tests show) are reported against double precision.  The candidate order and the
reference's stale cutoff are the same in both; the bounds are 1e-5 of the largest force and 1e-4 um
in position (the FP32 position grid at these coordinates is about 3e-5 um)."""
import numpy as np
import pytest

import oracle_lib as ol
from cases import ball_cells

pytestmark = pytest.mark.gpu

gb = pytest.importorskip("gell_b200")


@pytest.mark.parametrize("N,n", [(32, 3000), (64, 20000)])
def test_fm_update_vs_fp64_oracle(N, n):
    cells = ball_cells(N, 10.0, n, seed=7)
    P = ol.params(N=N, len=10.0, cap=2 * n)
    srt, f64, p64 = ol.force_move_f64(cells, P)
    with gb.Simulation(voxel_num=N, voxel_length=10.0, max_cell_num=2 * n) as sim:
        sim.import_cells(cells)
        sim.FM_update()
        out = sim.export_cells()
        sim.sync()
    assert len(out) == len(srt)
    alive = (srt["sign"] != 0) & (out["sign"] != 0)
    f32 = out["oldforce"][alive].astype(np.float64)  # the move keeps the force as oldforce
    p32 = out["pos"][alive].astype(np.float64)
    fs = np.abs(f64[alive]).max()
    ferr = np.abs(f32 - f64[alive]).max(1) / fs
    perr = np.abs(p32 - p64[alive]).max(1)
    print(f"N={N} n={n}: force error vs FP64 max {ferr.max():.2e} (99.9% {np.percentile(ferr, 99.9):.2e}) of "
          f"{fs:.3g}; position error max {perr.max():.2e} um")
    assert ferr.max() < 1e-5 and perr.max() < 1e-4
