"""A host loop shaped like the reference's main() (Main.cu:108-128), written in C++ against
include/gell_compat.hpp (MechanicsMesh_struct::FM_update, Mesh_struct::PreLOD/LODsolver/
move_to_GPU/move_to_CPU, CellBirth_kernel, CellDeath_kernel, run_mechanics), runs on the GPU and
must leave exactly the cells and the oxygen and drug fields that the same calls through the Python
mirror of the C ABI (gell_b200.Simulation) leave, bit for bit."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from cases import ball_cells, random_field
from gell_b200.cells import CELL_DTYPE

pytestmark = pytest.mark.gpu

gb = pytest.importorskip("gell_b200")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

LOOP = r"""
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "gell_compat.hpp"

template <class T>
static std::vector<T> load(const char* path) {
    std::vector<T> v;
    FILE* f = std::fopen(path, "rb");
    if (!f) return v;
    std::fseek(f, 0, SEEK_END);
    long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    v.resize((size_t)n / sizeof(T));
    if (std::fread(v.data(), sizeof(T), v.size(), f) != v.size()) v.clear();
    std::fclose(f);
    return v;
}
template <class T>
static void save(const char* path, const std::vector<T>& v) {
    FILE* f = std::fopen(path, "wb");
    std::fwrite(v.data(), sizeof(T), v.size(), f);
    std::fclose(f);
}

// argv: N cells.bin o2.bin drug.bin out_cells.bin out_o2.bin out_drug.bin
int main(int argc, char** argv) {
    if (argc != 8) return 2;
    try {
        gell_params p = gell::reference_params();
        p.voxel_num = std::atoi(argv[1]);
        p.voxel_length = 10.f;
        p.max_cell_num = 65536;
        p.rng_mode = GELL_RNG_PHILOX;
        p.seed = 20261204;
        gell::Context ctx(p);
        gell::MechanicsMesh_struct MecMesh(ctx);
        gell::Mesh_struct O2Mesh(ctx, 38.f, 1e5f, 0.1f);
        gell::Mesh_struct DrugMesh(ctx, 1.f, 5e4f, 0.05f, 1.f, -1.f);
        O2Mesh.move_to_GPU(load<float>(argv[3]));
        DrugMesh.move_to_GPU(load<float>(argv[4]));
        ctx.cells_from_host(load<gell_cell>(argv[2]));
        // the reference's loop: biology step (birth), mechanics steps with their diffusion
        // substeps, death; integer counts
        for (int bio = 0; bio < 2; ++bio) {
            gell::CellBirth_kernel(ctx);
            for (int m = 0; m < 3; ++m) {
                MecMesh.FM_update();
                O2Mesh.PreLOD();
                DrugMesh.PreLOD();
                for (int s = 0; s < 10; ++s) {
                    O2Mesh.LODsolver();
                    DrugMesh.LODsolver();
                }
            }
            gell::CellDeath_kernel(ctx);
        }
        gell::run_mechanics(ctx, 3, 10);
        save(argv[5], ctx.cells_to_host());
        save(argv[6], O2Mesh.move_to_CPU());
        save(argv[7], DrugMesh.move_to_CPU());
        return 0;
    } catch (const gell::Error& e) {
        std::printf("status %d: %s\n", (int)e.status, e.what());
        return 3;
    }
}
"""


def python_loop(N, cells, o2, drug):
    with gb.Simulation(voxel_num=N, voxel_length=10.0, max_cell_num=65536, rng_mode=gb.GELL_RNG_PHILOX,
                       seed=20261204) as sim:
        sim.add_substrate(gb.oxygen())
        sim.add_substrate(gb.drug())
        sim.set_field(0, o2)
        sim.set_field(1, drug)
        sim.import_cells(cells)
        for _ in range(2):
            sim.CellBirth_kernel()
            for _ in range(3):
                sim.FM_update()
                sim.PreLOD(0)
                sim.PreLOD(1)
                for _ in range(10):
                    sim.LODsolver(1, 0)
                    sim.LODsolver(1, 1)
            sim.CellDeath_kernel()
        sim.run_mechanics(3, 10)
        return sim.export_cells(), sim.field(0), sim.field(1)


def test_reference_shaped_cpp_loop_matches_the_python_mirror(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ missing")
    N = 48
    cells = ball_cells(N, 10.0, 6000, seed=77, outside=0, phases=True)
    o2 = random_field(N, seed=78, lo=2.0, hi=38.0)
    drug = (random_field(N, seed=79, lo=0.1, hi=1.0)).astype(np.float32)
    files = {k: str(tmp_path / f"{k}.bin") for k in ("cells", "o2", "drug", "oc", "oo2", "odrug")}
    np.ascontiguousarray(cells).tofile(files["cells"])
    o2.tofile(files["o2"])
    drug.tofile(files["drug"])
    src = tmp_path / "loop.cpp"
    src.write_text(LOOP)
    exe = tmp_path / "loop"
    libpath = gb.load_library()._name
    cuda_lib = "/usr/local/cuda/lib64"
    r = subprocess.run([gxx, "-std=c++17", "-O1", f"-I{os.path.join(ROOT, 'include')}", str(src), libpath,
                        f"-L{cuda_lib}", "-lcudart", f"-Wl,-rpath,{os.path.dirname(libpath)}",
                        f"-Wl,-rpath,{cuda_lib}", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe), str(N), files["cells"], files["o2"], files["drug"], files["oc"], files["oo2"],
                        files["odrug"]], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    got_cells = np.fromfile(files["oc"], dtype=CELL_DTYPE)
    got_o2 = np.fromfile(files["oo2"], dtype=np.float32)
    got_drug = np.fromfile(files["odrug"], dtype=np.float32)
    exp_cells, exp_o2, exp_drug = python_loop(N, cells, o2, drug)
    assert len(got_cells) == len(exp_cells) and len(exp_cells) != len(cells)  # birth/death changed the count
    np.testing.assert_array_equal(got_cells.view(np.uint8), exp_cells.view(np.uint8))
    # float atomics order the uptake sums; with several cells per voxel the fields agree within
    # FP32 rounding of those sums (the tests' 1e-5 relative tolerance), usually bit for bit
    np.testing.assert_allclose(got_o2, exp_o2, rtol=1e-5, atol=0)
    np.testing.assert_allclose(got_drug, exp_drug, rtol=1e-5, atol=0)
