"""Device time of whole mechanics steps of the reference's own CUDA build beside gell_b200's, on
the large workload (400^3 voxels of 10 um, oxygen + drug, 10^6 lattice-spheroid cells).

The reference façades (FM_update, PreLOD, LODsolver: include/FMkernel.cuh:181-202,
include/LODkernel.cuh:270-300) run through the harness built from the reference's unmodified
sources (oracle/ref_harness.cu); one step is FM_update + PreLOD of both substrates + 10 LODsolver
substeps of both, and whole steps are timed with CUDA events.  gell_b200 runs the same steps
through the C ABI.  The test prints both and asserts the target of this implementation: at least
3x the reference build's cell-updates/s.
"""
import json

import numpy as np
import pytest

import ref_lib
from gell_b200.cells import lattice_spheroid

pytestmark = pytest.mark.gpu

gb = pytest.importorskip("gell_b200")

N, LENGTH, NCELLS, SUBSTEPS = 400, 10.0, 1_000_000, 10


@pytest.mark.skipif(not (ref_lib.available("c2") and ref_lib.available("c2d")),
                    reason="reference build oracle/_ref missing")
def test_step_time_vs_reference_build():
    import torch

    cells = lattice_spheroid(NCELLS, N * LENGTH / 2, 0, LENGTH, N)
    ref = {}
    with ref_lib.RefSim("c2", 38.0, 1e5, 0.1) as o2, ref_lib.RefSim("c2d", 1.0, 5e4, 0.05) as drug:
        o2.set_cells(cells)

        def ref_step():
            o2.fm_update()
            o2.prelod()
            drug.prelod_on(o2)
            o2.lodsolver(SUBSTEPS)
            drug.lodsolver(SUBSTEPS)

        for _ in range(2):
            ref_step()
        a, b = ref_lib.RefEvent("c2"), ref_lib.RefEvent("c2")
        a.record()
        for _ in range(5):
            ref_step()
        b.record()
        ref["step"] = a.elapsed_ms(b) / 5
        a.close()
        b.close()
        ref["fm"] = o2.time_fm(2, 5)
        ref["lod_substep"] = o2.time_lod(2, 10) + drug.time_lod(2, 10)

    ours = {}
    with gb.Simulation(voxel_num=N, voxel_length=LENGTH, max_cell_num=2_000_000) as sim:
        sim.add_substrate(gb.oxygen())
        sim.add_substrate(gb.drug())
        sim.import_cells(cells)
        stream = torch.cuda.Stream()
        sim.set_stream(stream)

        def timed(fn, warm, iters):
            for _ in range(warm):
                fn()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record(stream)
            for _ in range(iters):
                fn()
            b.record(stream)
            torch.cuda.synchronize()
            return a.elapsed_time(b) / iters

        ours["fm"] = timed(sim.FM_update, 2, 5)
        ours["prelod"] = timed(sim.PreLOD, 2, 10)
        ours["lod_substep"] = timed(lambda: sim.LODsolver(1), 2, 10)
        ours["step"] = timed(lambda: (sim.FM_update(), sim.PreLOD(), sim.LODsolver(SUBSTEPS)), 2, 5)
        alive = int(sim.export_cells()["sign"].sum())

    rec = {"workload": "400^3, oxygen + drug, 10^6 cells, 1 step = FM_update + PreLOD + 10 substeps",
           "reference_ms": {k: round(v, 4) for k, v in ref.items()},
           "gell_b200_ms": {k: round(v, 4) for k, v in ours.items()},
           "speedup_step": round(ref["step"] / ours["step"], 3),
           "speedup_fm": round(ref["fm"] / ours["fm"], 3),
           "speedup_lod_substep": round(ref["lod_substep"] / ours["lod_substep"], 3),
           "cell_updates_per_s": {"reference": alive / (ref["step"] / 1e3), "gell_b200": alive / (ours["step"] / 1e3)}}
    print("REFERENCE_TIMING " + json.dumps(rec))
    assert all(np.isfinite(v) and v > 0 for v in list(ref.values()) + list(ours.values()))
    assert ref["step"] / ours["step"] >= 3.0, rec
