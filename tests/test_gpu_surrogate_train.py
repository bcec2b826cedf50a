"""Training the learned LOD surrogate with the library's own kernels, against PyTorch autograd.

One training pair at learning rate 0 gives the gradient of the loss with respect to every weight
and bias.  PyTorch recomputes it in fp32 from the same bf16 weights and the same stored input, with
each stored activation rounded to bf16 as the CUDA path stores it (straight-through, so the
gradient passes unchanged).  The CUDA path also stores the gradient planes in bf16, so the two
agree to within a few parts in a thousand per layer; a wrong tap, transpose or mask would not.
"""
import numpy as np
import pytest

from cases import ball_cells, random_field

pytestmark = pytest.mark.gpu

gb = pytest.importorskip("gell_b200")
torch = pytest.importorskip("torch")

SHAPES = [(3, 32)] + [(32, 32)] * 8 + [(32, 1)]


def random_weights(seed):
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for cin, cout in SHAPES:
        out.append(rng.normal(0, 1.0 / np.sqrt(cin * 27), (cout, cin, 3, 3, 3)).astype(np.float32).ravel())
        out.append(rng.normal(0, 0.05, cout).astype(np.float32))
    w = np.concatenate(out)
    w[-(32 * 27 + 1):] *= 0.05  # a small last layer, as in a fit started near the identity map
    return w


def make_sim(N, seed, cells=2000):
    sim = gb.Simulation(voxel_num=N, voxel_length=10.0, max_cell_num=cells)
    sim.add_substrate(gb.oxygen())
    sim.import_cells(ball_cells(N, 10.0, cells, seed, dead_frac=0.0, outside=0))
    sim.set_field(0, random_field(N, seed, 20.0, 38.0))
    sim.PreLOD()
    return sim


def torch_grads(w, x, p, y, N, b=38.0, scale=None):
    """Loss and flat gradient of the operator in fp32, activations rounded to bf16 on the way.  The
    output is q = p + scale * d and the loss is in units of `scale` (default: b, the field form)."""
    scale = b if scale is None else scale
    dev = torch.device("cuda")

    def rnd(t):  # stored as bf16, gradient passed straight through
        return t + (t.to(torch.bfloat16).float() - t).detach()

    params, i = [], 0
    for cin, cout in SHAPES:
        n = cout * cin * 27
        W = torch.from_numpy(w[i:i + n].reshape(cout, cin, 3, 3, 3)).to(torch.bfloat16).float().to(dev)
        i += n
        bb = torch.from_numpy(w[i:i + cout].copy()).to(dev)
        i += cout
        W.requires_grad_(True)
        bb.requires_grad_(True)
        params += [W, bb]
    conv = torch.nn.functional.conv3d
    xt = torch.from_numpy(x).to(dev).reshape(1, 3, N, N, N)
    h = rnd(torch.relu(conv(xt, params[0], params[1], padding=1)))
    for k in range(4):
        t = rnd(torch.relu(conv(h, params[2 + 4 * k], params[3 + 4 * k], padding=1)))
        h = rnd(h + conv(t, params[4 + 4 * k], params[5 + 4 * k], padding=1))
    d = conv(h, params[18], params[19], padding=1)[0, 0].reshape(-1)
    g = np.arange(N)
    sh = (g < 2) | (g > N - 3)
    inner = torch.from_numpy(~(sh[:, None, None] | sh[None, :, None] | sh[None, None, :]).ravel()).to(dev)
    pt = torch.from_numpy(p).to(dev)
    yt = torch.from_numpy(y).to(dev)
    q = pt + scale * d
    e = ((q - yt) / scale)[inner]
    loss = (e * e).mean()
    loss.backward()
    flat = torch.cat([(prm.grad if prm.grad is not None else torch.zeros_like(prm)).reshape(-1) for prm in params])
    return float(loss.detach()), flat.cpu().numpy()


def layer_slices():
    out, i = [], 0
    for l, (cin, cout) in enumerate(SHAPES):
        n = cout * cin * 27
        out.append((f"W{l}", slice(i, i + n)))
        i += n
        out.append((f"b{l}", slice(i, i + cout)))
        i += cout
    return out


@pytest.mark.parametrize("N", [40, 136, 37])
def test_training_gradient_matches_autograd(N):
    w = random_weights(21)
    with make_sim(N, 9) as sim:
        sim.surrogate_train_init(0, w, 5, 0.1)
        p = sim.field(0)
        loss = sim.surrogate_train_pair(0, 0.0)
        grad = sim.surrogate_train_read(0, 1)
        y = sim.surrogate_train_read(0, 2)
        x = sim.surrogate_read(0, 0)[:3]
        # the field is left at the target, which is the plain solver's 5 substeps
        assert np.array_equal(sim.field(0).view(np.uint32), y.view(np.uint32))
        assert np.array_equal(sim.surrogate_train_read(0, 0), w)  # lr = 0: weights unchanged
        sim.sync()
    tloss, tgrad = torch_grads(w, x, p, y, N)
    assert abs(loss - tloss) <= 1e-3 * tloss, (loss, tloss)
    for name, sl in layer_slices():
        a, r = grad[sl].astype(np.float64), tgrad[sl].astype(np.float64)
        rel = np.linalg.norm(a - r) / max(np.linalg.norm(r), 1e-30)
        cos = float(a @ r / max(np.linalg.norm(a) * np.linalg.norm(r), 1e-30))
        print(f"{name}: |g| {np.linalg.norm(r):.3e} rel err {rel:.2e} cos {cos:.6f}")
        assert rel < 2e-2 and cos > 0.9995, (name, rel, cos)


def test_training_reduces_loss_on_a_pair():
    w = random_weights(22)
    with make_sim(48, 10) as sim:
        sim.surrogate_train_init(0, w, 5, 0.1)
        p = sim.field(0)
        losses = []
        for _ in range(30):
            sim.set_field(0, p)
            losses.append(sim.surrogate_train_pair(0, 2e-3))
        sim.sync()
    print("losses", losses[0], losses[-1])
    assert losses[-1] < 0.6 * losses[0]


@pytest.mark.parametrize("N", [40, 37])
def test_training_gradient_matches_autograd_delta_input(N):
    """The delta form (GELL_OPT_SURROGATE_INPUT = 1): the input is the change of one plain substep
    over its largest magnitude m, the output q = p + m d, the loss in units of m."""
    w = random_weights(23)
    with make_sim(N, 11) as sim:
        p = sim.field(0)
        sim.LODsolver(1, 0)
        p1 = sim.field(0)
        sim.set_field(0, p)
        g = np.arange(N)
        sh = (g < 2) | (g > N - 3)
        inner = ~(sh[:, None, None] | sh[None, :, None] | sh[None, None, :]).ravel()
        m = float(np.abs(p1 - p)[inner].max())
        assert m > 0
        sim.surrogate_train_init(0, w, 5, 0.1, input_kind=1)
        loss = sim.surrogate_train_pair(0, 0.0)
        grad = sim.surrogate_train_read(0, 1)
        y = sim.surrogate_train_read(0, 2)
        x = sim.surrogate_read(0, 0)[:3]
        assert np.array_equal(sim.field(0).view(np.uint32), y.view(np.uint32))
        sim.sync()
    tloss, tgrad = torch_grads(w, x, p, y, N, scale=np.float32(m))
    assert abs(loss - tloss) <= 1e-3 * tloss, (loss, tloss)
    for name, sl in layer_slices():
        a, r = grad[sl].astype(np.float64), tgrad[sl].astype(np.float64)
        rel = np.linalg.norm(a - r) / max(np.linalg.norm(r), 1e-30)
        cos = float(a @ r / max(np.linalg.norm(a) * np.linalg.norm(r), 1e-30))
        assert rel < 2e-2 and cos > 0.9995, (name, rel, cos)
