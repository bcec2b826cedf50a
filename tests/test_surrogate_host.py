"""Host side of the learned surrogate (no GPU): the weight file format, the layer table against the
library's own count, the boundary shell, and the initial weights."""
import numpy as np
import pytest

from gell_b200 import surrogate as gs


def test_weight_file_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    for kind in (0, 1):
        sw = gs.SurrogateWeights(rng.standard_normal(gs.weight_count()).astype(np.float32), 50, 0.1, 2.35e-3, kind)
        path = tmp_path / f"w{kind}.gsur"
        gs.save_weights(str(path), sw)
        back = gs.load_weights(str(path))
        assert (back.substeps, back.rate_scale, back.threshold, back.input_kind) == (50, np.float32(0.1),
                                                                                     np.float32(2.35e-3), kind)
        assert np.array_equal(back.weights, sw.weights)
        raw = path.read_bytes()
        assert raw[:8] == b"GSUR0002" and len(raw) == 8 + 24 + 4 * gs.weight_count()


def test_version_one_weight_files_load_as_the_field_form(tmp_path):
    import struct
    w = np.arange(gs.weight_count(), dtype=np.float32)
    path = tmp_path / "v1.gsur"
    path.write_bytes(b"GSUR0001" + struct.pack("<iffq", 50, 0.1, 5e-3, w.size) + w.astype("<f4").tobytes())
    back = gs.load_weights(str(path))
    assert back.input_kind == 0 and back.substeps == 50 and np.array_equal(back.weights, w)


def test_weight_file_rejects_bad_input(tmp_path):
    bad = tmp_path / "bad.gsur"
    bad.write_bytes(b"NOTAFILE" + bytes(20))
    with pytest.raises(ValueError):
        gs.load_weights(str(bad))
    sw = gs.SurrogateWeights(np.zeros(gs.weight_count(), np.float32))
    good = tmp_path / "good.gsur"
    gs.save_weights(str(good), sw)
    good.write_bytes(good.read_bytes()[:-4])  # one weight short
    with pytest.raises(ValueError):
        gs.load_weights(str(good))


def test_layer_table_matches_the_library():
    import gell_b200 as gb
    assert gs.weight_count() == gb.load_library().gell_surrogate_weight_count() == 224929


def test_packaged_weights_load():
    sw = gs.load_weights(gs.DEFAULT_WEIGHTS)
    assert sw.weights.size == gs.weight_count() and np.isfinite(sw.weights).all()
    assert sw.substeps == 50 and 0 < sw.threshold < 0.01


@pytest.mark.parametrize("N", [8, 13, 40])
def test_shell_is_the_four_boundary_layers(N):
    m = gs.shell_mask(N).reshape(N, N, N)  # [z][y][x]
    g = np.arange(N)
    layer = (g < 2) | (g >= N - 2)
    for z in range(N):
        for y in range(N):
            expect = layer | layer[y] | layer[z]
            assert np.array_equal(m[z, y], expect)


def test_initial_weights_start_from_the_identity_map():
    w = gs.init_weights(3)
    assert w.size == gs.weight_count()
    last = 32 * 27 + 1
    assert not w[-last:].any() and w[:-last].any()
    # each earlier layer within 1/sqrt(fan_in)
    i = 0
    for ci, co in gs.SHAPES[:-1]:
        n = co * ci * 27 + co
        assert np.abs(w[i:i + n]).max() <= 1.0 / np.sqrt(ci * 27)
        i += n
