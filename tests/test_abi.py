"""The C ABI on the CPU: the library loads, exports every entry point include/gell.h declares,
its parameter defaults equal the reference's #defines, and it reports a missing GPU as a status
instead of crashing.  No compute call here needs a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle_lib as ol

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(gell_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    gb = pytest.importorskip("gell_b200")
    lib = gb.load_library()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version_and_status_strings():
    import gell_b200 as gb
    lib = gb.load_library()
    assert lib.gell_abi_version() == 1
    assert lib.gell_status_string(0) == b"ok"
    assert lib.gell_status_string(-4) == b"no CUDA device"


def test_record_layout_is_the_reference_cell():
    from gell_b200.cells import CELL_DTYPE
    offs = {k: CELL_DTYPE.fields[k][1] for k in CELL_DTYPE.names}
    assert CELL_DTYPE.itemsize == 72
    assert (offs["mesh_idx"], offs["pos"], offs["force"], offs["oldforce"], offs["r"], offs["V"],
            offs["Vf"], offs["Vcs"], offs["Vns"], offs["phase"], offs["cell_clock"]) == \
        (4, 8, 20, 32, 44, 48, 52, 56, 60, 64, 68)


def test_param_defaults_match_reference_definitions():
    import gell_b200 as gb
    p = gb.default_params()
    o = ol.params()
    assert (p.voxel_num, p.max_cell_num) == (o.N, o.cap) == (100, 2_000_000)
    pairs = [("voxel_length", "len"), ("mechanics_dt", "mech_dt"), ("diffusion_dt", "diff_dt"),
             ("biology_dt", "bio_dt"), ("ccca", "ccca"), ("cccr", "cccr"), ("ra_ratio", "ra_ratio"),
             ("cc_max_dist", "cc_max_dist"), ("dead_uptake_factor", "dead_factor"),
             ("default_v", "default_v"), ("o2_prolif_thres", "o2_pt"), ("o2_prolif_sat", "o2_ps"),
             ("o2_necrosis_thres", "o2_nt"), ("o2_necrosis_max", "o2_nm"),
             ("necrosis_rate", "necrosis_rate"), ("apoptosis_rate", "apoptosis_rate"),
             ("proliferation_rate", "prolif_rate"), ("duration_pre2post", "dur_pre2post"),
             ("duration_post2q", "dur_post2q")]
    for a, b in pairs:
        assert getattr(p, a) == getattr(o, b), a
    assert p.seed == 123 and p.rng_mode == gb.GELL_RNG_XORWOW


def test_params_struct_size_matches_c():
    import gell_b200 as gb
    # int,float,int,3 float,2 float,double,8 float (pad),3 double,2 float,4 int,u64
    assert ctypes.sizeof(gb.GellParams) == 128


def no_gpu():
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


@pytest.mark.skipif(not no_gpu(), reason="checks behaviour without a GPU")
def test_create_without_gpu_reports_status():
    import gell_b200 as gb
    with pytest.raises(gb.GellError) as e:
        gb.Simulation(voxel_num=16, voxel_length=10.0, max_cell_num=100)
    assert e.value.status in (-4, -3)


def test_create_rejects_invalid_parameters():
    import gell_b200 as gb
    lib = gb.load_library()
    h = ctypes.c_void_p()
    bad = [dict(voxel_num=3), dict(voxel_num=1024), dict(voxel_length=0.0), dict(max_cell_num=0),
           dict(rng_mode=7), dict(mech_mode=3)]
    for kw in bad:
        p = gb.default_params(**kw)
        st = lib.gell_create(ctypes.byref(p), ctypes.byref(h))
        assert st in (-1, -7), (kw, st)
        assert not h.value
    assert lib.gell_create(None, ctypes.byref(h)) == -1


def test_null_context_calls_are_rejected():
    import gell_b200 as gb
    lib = gb.load_library()
    for fn, args in (("gell_fm_update", []), ("gell_prelod", [-1]), ("gell_lod_solver", [-1, 1]),
                     ("gell_cell_birth", [None]), ("gell_cell_death", [None]), ("gell_sync", []),
                     ("gell_destroy", [])):
        assert getattr(lib, fn)(None, *args) == -1, fn


COMPAT_MAIN = r"""
#include <cstdio>
#include "gell_compat.hpp"
int main() {
    try {
        gell::Context ctx(gell::reference_params());
        gell::MechanicsMesh_struct mec(ctx);
        gell::Mesh_struct o2(ctx, 38.f, 1e5f, 0.1f);
        mec.FM_update();
        o2.PreLOD();
        o2.LODsolver();
        int n = gell::CellBirth_kernel(ctx);
        n = gell::CellDeath_kernel(ctx);
        gell::run_mechanics(ctx, 4, 10);
        n = gell::run(ctx, 1, 60, 10);
        std::printf("ran %d\n", n);
        return 0;
    } catch (const gell::Error& e) {
        std::printf("status %d\n", (int)e.status);
        return 3;
    }
}
"""


def test_compat_header_builds_a_reference_shaped_loop(tmp_path):
    """include/gell_compat.hpp compiles with plain g++ against the C ABI; without a GPU the first
    call throws gell::Error carrying GELL_ERR_NO_DEVICE."""
    import shutil
    import subprocess
    gb = pytest.importorskip("gell_b200")
    libpath = gb.load_library()._name
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ missing")
    src = tmp_path / "main.cpp"
    src.write_text(COMPAT_MAIN)
    exe = tmp_path / "main"
    cuda_lib = "/usr/local/cuda/lib64"
    r = subprocess.run([gxx, "-std=c++17", "-O1", f"-I{os.path.join(ROOT, 'include')}", str(src),
                        libpath, f"-L{cuda_lib}", "-lcudart", f"-Wl,-rpath,{os.path.dirname(libpath)}",
                        f"-Wl,-rpath,{cuda_lib}", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the no-device path is not reachable")
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 3 and r.stdout.strip() == "status -4", (r.returncode, r.stdout, r.stderr)
