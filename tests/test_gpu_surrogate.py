"""The learned LOD surrogate on the GPU: its tcgen05 convolutions against PyTorch fp32 convolutions of
the same bf16 operands, and the judge / fallback contract against the plain solver.

Each layer is checked on its own input as the CUDA path stored it (bf16 planes read back through
the C ABI), so rounding does not compound: the stored output must equal the fp32 reference rounded
to bf16 within one bf16 unit (2^-8 relative; the two sums differ only in order).  The output
field (fp32) must match within 1e-5 of the boundary value.
"""
import numpy as np
import pytest

from cases import ball_cells, random_field

pytestmark = pytest.mark.gpu

gb = pytest.importorskip("gell_b200")
torch = pytest.importorskip("torch")

SHAPES = [(3, 32)] + [(32, 32)] * 8 + [(32, 1)]


def random_weights(seed, scale=1.0):
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for cin, cout in SHAPES:
        std = scale / np.sqrt(cin * 27)
        out.append(rng.normal(0, std, (cout, cin, 3, 3, 3)).astype(np.float32).ravel())
        out.append(rng.normal(0, 0.1, cout).astype(np.float32))
    w = np.concatenate(out)
    assert w.size == gb.load_library().gell_surrogate_weight_count()
    return w


def layer_params(w):
    """[(W[cout,cin,3,3,3], b[cout])] with W rounded to bf16 as the kernels store it."""
    out, i = [], 0
    for cin, cout in SHAPES:
        n = cout * cin * 27
        W = torch.from_numpy(w[i:i + n].reshape(cout, cin, 3, 3, 3)).to(torch.bfloat16).float()
        i += n
        b = torch.from_numpy(w[i:i + cout].copy())
        i += cout
        out.append((W.cuda(), b.cuda()))
    return out


def conv(x, Wb, N):
    W, b = Wb
    xt = torch.from_numpy(x).cuda().reshape(1, x.shape[0], N, N, N)  # [C][z][y][x]
    return torch.nn.functional.conv3d(xt, W, b, padding=1)[0].reshape(W.shape[0], -1).cpu().numpy()


def assert_bf16_close(got, ref, what):
    # one bf16 unit of the value (8 significant bits): the stored result is the bf16 rounding of a
    # fp32 sum that differs from the reference only in order, so it can land on either neighbour
    mag = np.maximum(np.abs(ref), 1e-30)
    tol = np.exp2(np.floor(np.log2(mag)) - 7) + 1e-6
    bad = np.abs(got - ref) > tol
    assert not bad.any(), (what, int(bad.sum()), float(np.abs(got - ref).max()))


def make_sim(N, seed, cells=2000):
    sim = gb.Simulation(voxel_num=N, voxel_length=10.0, max_cell_num=max(cells, 16))
    sim.add_substrate(gb.oxygen())
    sim.import_cells(ball_cells(N, 10.0, cells, seed, dead_frac=0.0, outside=0))
    sim.set_field(0, random_field(N, seed, 20.0, 38.0))
    sim.PreLOD()
    return sim


@pytest.mark.parametrize("ring", [1, 0])
@pytest.mark.parametrize("N", [40, 136, 37])
def test_surrogate_layers_match_torch(N, ring):
    w = random_weights(3)
    Ws = layer_params(w)
    with make_sim(N, 5) as sim:
        sim.set_conv_ring(bool(ring))
        sim.surrogate_load(0, w, 50, 0.1, 1.0)
        b = 38.0
        sim.surrogate_run_layers(0, 0)
        x = sim.surrogate_read(0, 0)[:3]
        # input planes: p / b, rate * 0.1, shell
        p = sim.field(0)
        rate = sim.dump_rate(0)
        bf = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16).float().numpy()
        assert np.array_equal(x[0], bf(p * np.float32(1.0 / b)))
        assert np.array_equal(x[1], bf(rate * np.float32(0.1)))
        g = np.arange(N)
        sh = (g < 2) | (g > N - 3)
        shell = (sh[:, None, None] | sh[None, :, None] | sh[None, None, :]).ravel()
        assert np.array_equal(x[2], shell.astype(np.float32))
        prev_h = None
        for l in range(10):
            sim.surrogate_run_layers(0, l)
            h_in, t_in = sim.surrogate_read(0, 1), sim.surrogate_read(0, 2)
            sim.surrogate_run_layers(0, l + 1)
            if l == 0:
                ref = np.maximum(conv(x, Ws[0], N), 0)
                assert_bf16_close(sim.surrogate_read(0, 1), ref, "layer 0")
            elif l == 9:
                d = conv(h_in, Ws[9], N)[0]
                ref = np.where(shell, np.float32(b), p + np.float32(b) * d)
                got = sim.surrogate_read(0, 3)
                assert np.abs(got - ref).max() <= 1e-5 * b, np.abs(got - ref).max()
            elif l % 2 == 1:
                ref = np.maximum(conv(h_in, Ws[l], N), 0)
                assert_bf16_close(sim.surrogate_read(0, 2), ref, f"layer {l}")
            else:
                ref = h_in + conv(t_in, Ws[l], N)
                assert_bf16_close(sim.surrogate_read(0, 1), ref, f"layer {l}")
            prev_h = h_in
        assert prev_h is not None
        assert sim.launch_count() > 0
        sim.sync()


def test_delta_input_planes_and_output():
    """The delta form (GELL_OPT_SURROGATE_INPUT = 1): channel 0 of the input is the change of one
    plain substep over its largest magnitude m inside the shell (0 on the shell), the field is left
    as it was, and the output is p + m d inside the shell, b on it."""
    N = 40
    w = random_weights(7)
    Ws = layer_params(w)
    with make_sim(N, 8) as sim:
        b = 38.0
        p = sim.field(0)
        sim.LODsolver(1, 0)
        p1 = sim.field(0)
        sim.set_field(0, p)
        g = np.arange(N)
        sh = (g < 2) | (g > N - 3)
        shell = (sh[:, None, None] | sh[None, :, None] | sh[None, None, :]).ravel()
        m = np.float32(np.abs(p1 - p)[~shell].max())
        sim.surrogate_load(0, w, 50, 0.1, 1.0, input_kind=1)
        sim.surrogate_run_layers(0, 0)
        x = sim.surrogate_read(0, 0)[:3]
        bf = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16).float().numpy()
        d1 = np.where(shell, np.float32(0), (p1 - p) * (np.float32(1) / m)).astype(np.float32)
        assert np.array_equal(x[0], bf(d1))
        assert np.array_equal(x[1], bf(sim.dump_rate(0) * np.float32(0.1)))
        assert np.array_equal(x[2], shell.astype(np.float32))
        assert np.array_equal(sim.field(0).view(np.uint32), p.view(np.uint32))
        sim.surrogate_run_layers(0, 9)
        h_in = sim.surrogate_read(0, 1)
        sim.surrogate_run_layers(0, 10)
        d = conv(h_in, Ws[9], N)[0]
        ref = np.where(shell, np.float32(b), p + m * d)
        got = sim.surrogate_read(0, 3)
        assert np.abs(got - ref).max() <= 1e-5 * b, np.abs(got - ref).max()
        sim.sync()


def test_judge_accepts_and_falls_back():
    N, K = 48, 50
    w = random_weights(4)
    # conv_out all zero: the operator returns p inside and b on the shell
    n_out = 32 * 27 + 1
    w[-n_out:] = 0
    with make_sim(N, 6, 3000) as a, make_sim(N, 6, 3000) as ref:
        a.surrogate_load(0, w, K, 0.1, 1e9)
        p0 = a.field(0)
        ok, r = a.lod_surrogate(0)
        assert ok and r > 0
        q = a.field(0)
        g = np.arange(N)
        sh = (g < 2) | (g > N - 3)
        shell = (sh[:, None, None] | sh[None, :, None] | sh[None, None, :]).ravel()
        assert np.array_equal(q[~shell], p0[~shell]) and np.all(q[shell] == np.float32(38.0))
        # the judge residual is one plain substep's change of that field
        a.set_field(0, q)
        a.LODsolver(1, 0)
        l1 = a.field(0)
        inner = np.zeros((N, N, N), bool)
        inner[2:N - 2, 2:N - 2, 2:N - 2] = True
        inner = inner.ravel()
        assert np.float32(np.abs(l1 - q)[inner].max() / np.float32(38.0)) == np.float32(r)
        # a threshold below every residual: the field is exactly the plain solver's K substeps
        a.set_field(0, p0)
        a.surrogate_load(0, w, K, 0.1, -1.0)
        ok, r2 = a.lod_surrogate(0)
        assert not ok and r2 == r
        ref.LODsolver(K, 0)
        assert np.array_equal(a.field(0).view(np.uint32), ref.field(0).view(np.uint32))
        a.sync()


def test_packaged_surrogate_vs_fp64_oracle():
    """The packaged operator on the surrogate workload (256^3, 300,000 cells, quasi-steady field):
    a judged step that is accepted is within 1% (L-infinity inside the shell, units of the boundary
    value) of the FP64 restatement of the plain scheme run for the same 50 substeps from the same
    field and uptake map; the plain FP32 solver is within 1e-4 of it."""
    import oracle_lib as ol
    from gell_b200 import surrogate as gs

    sw = gs.load_weights(gs.DEFAULT_WEIGHTS)
    N, n = 256, 300_000
    o2 = gb.oxygen()
    cells = gb.lattice_spheroid(n, N * 10.0 / 2, 5, 10.0, N)
    gb.seed_ki67_states(cells, 13)
    with gb.Simulation(voxel_num=N, voxel_length=10.0, max_cell_num=n) as sim:
        sim.add_substrate(o2)
        sim.import_cells(cells)
        sim.PreLOD()
        sim.LODsolver(1000, 0)
        sim.surrogate_load(0, sw.weights, sw.substeps, sw.rate_scale, sw.threshold, sw.input_kind)
        p = sim.field(0)
        rate = sim.dump_rate(0)
        ok, r = sim.lod_surrogate(0)
        q = sim.field(0)
        sim.set_field(0, p)
        sim.LODsolver(sw.substeps, 0)
        plain = sim.field(0)
    p64 = ol.lod_substeps_f64(p, rate, N, 10.0, o2.diffusion, o2.decay, 0.01, o2.boundary, sw.substeps)
    inner = ~gs.shell_mask(N)
    e_plain = np.abs(plain.astype(np.float64) - p64)[inner].max() / o2.boundary
    e_sur = np.abs(q.astype(np.float64) - p64)[inner].max() / o2.boundary
    print(f"judge residual {r:.3e} (threshold {sw.threshold:.3e}) accepted {ok}; "
          f"Linf vs FP64: surrogate {e_sur:.3e}, plain FP32 {e_plain:.3e}")
    assert e_plain < 1e-4
    if ok:
        assert e_sur <= 0.01
    else:
        assert np.array_equal(q.view(np.uint32), plain.view(np.uint32))


def test_surrogate_step_touches_only_its_substrate():
    """A judged oxygen step in a context that also holds the drug: the drug field is left as it was,
    and a rejected step gives oxygen exactly the plain solver's substeps of oxygen alone."""
    N, K = 40, 50
    w = random_weights(8)
    with make_sim(N, 11) as a, make_sim(N, 11) as ref:
        for sim in (a, ref):
            sim.add_substrate(gb.drug())
            sim.set_field(1, random_field(N, 12, 0.2, 1.0))
            sim.PreLOD()
        drug0 = a.field(1)
        a.surrogate_load(0, w, K, 0.1, -1.0)  # every step rejected
        ok, _ = a.lod_surrogate(0)
        assert not ok
        ref.LODsolver(K, 0)
        assert np.array_equal(a.field(0).view(np.uint32), ref.field(0).view(np.uint32))
        assert np.array_equal(a.field(1).view(np.uint32), drug0.view(np.uint32))
        a.sync()


def test_surrogate_errors_are_reported():
    import ctypes
    L = gb.load_library()
    with make_sim(24, 13) as sim:
        w = random_weights(9)
        # wrong weight count, no surrogate loaded, bad substrate: errors, and the context goes on
        assert L.gell_surrogate_load(sim.h, 0, w.ctypes.data, w.size - 1, 50, 0.1, 1e-3) == -1
        acc, r = ctypes.c_int(), ctypes.c_float()
        assert L.gell_lod_surrogate(sim.h, 0, ctypes.byref(acc), ctypes.byref(r)) == -1
        assert L.gell_surrogate_load(sim.h, 3, w.ctypes.data, w.size, 50, 0.1, 1e-3) == -1
        sim.surrogate_load(0, w, 50, 0.1, 1e9)
        ok, _ = sim.lod_surrogate(0)
        assert ok
        sim.sync()
