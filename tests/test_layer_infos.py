"""The layer-info JSON front end and image files (LayerInfos.md;
unblending/src/unblending_io.cpp:12-170, unblending/io/image_qt.cpp:6-82):
parsing rules, the precision the library derives, the writer's format,
round trips and error behaviour, and the image naming and 8-bit rules. Host
code only."""
import json
import os

import numpy as np
import pytest

from unblending_b200 import io as uio
from unblending_b200 import synthetic as syn


def layer(mode, mu, var, op="source-over"):
    return {"color_model": {"color_variance": var, "primary_color": mu}, "comp_op": op, "mode": mode}


def test_modes_comp_ops_and_scalar_variance():
    text = json.dumps([layer(name, [0.1 * k, 0.2, 0.3], 0.01 * (k + 1), "source-over" if k % 2 else "plus")
                       for k, name in enumerate(uio.MODE_NAMES)])
    layers = uio.parse_layer_infos(text)
    assert [l.mode for l in layers] == list(range(13))
    for k, l in enumerate(layers):
        assert l.comp == ((1, 1, 1) if k % 2 else (2, 1, 1))
        np.testing.assert_array_equal(l.mean, [0.1 * k, 0.2, 0.3])
        v = 0.01 * (k + 1)
        np.testing.assert_allclose(l.precision, np.eye(3) / v, rtol=1e-15, atol=0)
        assert l.precision[0, 1] == 0.0 and l.precision[2, 1] == 0.0


def test_full_covariance_reads_column_by_column():
    items = [0.05, 0.01, 0.002, 0.013, 0.04, 0.003, 0.004, 0.005, 0.06]   # not symmetric on purpose
    (l,) = uio.parse_layer_infos(json.dumps([layer("Screen", [0.5, 0.4, 0.3], items)]))
    cov = np.array(items).reshape(3, 3).T          # element (row, col) at index col * 3 + row
    np.testing.assert_allclose(l.precision, np.linalg.inv(cov), rtol=1e-12)
    np.testing.assert_allclose(l.precision @ cov, np.eye(3), atol=1e-12)


def test_comp_op_other_than_source_over_reads_as_plus():
    text = json.dumps([{"color_model": {"color_variance": 0.1, "primary_color": [0, 0, 0]}, "mode": "Normal"},
                       layer("Normal", [0, 0, 0], 0.1, "darken")])
    assert [l.comp for l in uio.parse_layer_infos(text)] == [(2, 1, 1), (2, 1, 1)]


@pytest.mark.parametrize("text", [
    "",
    "[",
    '{"mode": "Normal"}',
    json.dumps([layer("Normal", [0, 0, 0], 0.1)]) + " x",
    json.dumps([layer("Vivid", [0, 0, 0], 0.1)]),
    json.dumps([{"color_model": {"color_variance": 0.1, "primary_color": [0, 0, 0]}}]),
    json.dumps([layer("Normal", [0, 0], 0.1)]),
    json.dumps([layer("Normal", [0, 0, 0], [0.1] * 8)]),
    json.dumps([layer("Normal", [0, 0, 0], "0.1")]),
    json.dumps([layer("Normal", [0, 0, 0], 0.0)]),
    json.dumps([layer("Normal", [0, 0, 0], [1, 2, 3, 2, 4, 6, 1, 1, 1])]),   # singular
    '[{"color_model": {"color_variance": 0.1, "primary_color": [0, 0, 01]}, "mode": "Normal"}]',
])
def test_malformed_input_is_rejected(text):
    with pytest.raises(ValueError):
        uio.parse_layer_infos(text)


def test_json_syntax_details():
    text = ('\n [ { "mode" : "Nor\\u006dal", "comp_op":"source-over",\t"color_model":{"primary_color":'
            '[1e-1, 2.5E-1, -0.0], "color_variance": 1.25e-2, "extra": [true, false, null, {"k": "\\"\\\\\\/"}]}} ] ')
    (l,) = uio.parse_layer_infos(text)
    assert l.mode == 0 and l.comp == (1, 1, 1)
    np.testing.assert_array_equal(l.mean, [0.1, 0.25, -0.0])
    np.testing.assert_allclose(l.precision, np.eye(3) / 0.0125, rtol=1e-15)
    assert uio.parse_layer_infos("[]") == []


def test_format_matches_the_written_format():
    layers = uio.parse_layer_infos(json.dumps([layer("Normal", [0.131, 0.131, 0.212], 0.1),
                                               layer("HardLight", [1.0, 0.566, 1.0], 0.015, "plus")]))
    text = uio.format_layer_infos(layers)
    doc = json.loads(text)
    assert text.startswith('[{"color_model": {"color_variance": ')
    assert list(doc[0].keys()) == ["color_model", "comp_op", "mode"]
    assert list(doc[0]["color_model"].keys()) == ["color_variance", "primary_color"]
    assert doc[0]["mode"] == "Normal" and doc[1]["mode"] == "HardLight"
    assert doc[0]["comp_op"] == "source-over" and doc[1]["comp_op"] == "plus"
    # A multiple of the identity is written as one number (the inverse of the
    # inverse carries a few ulps).
    assert isinstance(doc[0]["color_model"]["color_variance"], float)
    assert doc[0]["color_model"]["color_variance"] == pytest.approx(0.1, rel=1e-14)
    assert doc[0]["color_model"]["primary_color"] == [0.131, 0.131, 0.212]


def test_round_trip_of_generated_layers(tmp_path):
    rng = np.random.default_rng(5)
    specs = syn.make_layers(rng, [0, 1, 2, 3, 6, 9])
    path = uio.export_layer_infos(specs, str(tmp_path))
    assert os.path.basename(path) == "layer_infos.json"
    back = uio.import_layer_infos(path)
    doc = json.load(open(path))
    assert all(isinstance(d["color_model"]["color_variance"], list) for d in doc)   # full covariances
    for a, b in zip(specs, back):
        assert a.mode == b.mode and tuple(a.comp) == tuple(b.comp)
        np.testing.assert_array_equal(a.mean, b.mean)
        np.testing.assert_allclose(b.precision, a.precision, rtol=1e-12, atol=1e-9)
    # Each trip inverts twice; the covariance drifts by ulps, not more.
    again = uio.parse_layer_infos(uio.format_layer_infos(back))
    for a, b in zip(back, again):
        np.testing.assert_allclose(b.precision, a.precision, rtol=1e-12, atol=1e-9)


def test_image_files_naming_and_8bit_rules(tmp_path):
    pytest.importorskip("PIL")
    L, h, w = 3, 5, 7
    rng = np.random.default_rng(2)
    packed = rng.uniform(-0.2, 1.2, size=(L, h, w, 4))
    infos = syn.make_layers(rng, [0, 6, 12])
    paths = uio.export_layers(packed, str(tmp_path), "layer", with_alpha_channel=True, with_blend_mode_suffix=True,
                              layer_infos=infos)
    names = sorted(os.path.basename(p) for p in paths)
    assert names == sorted(["layer_0_Normal.png", "layer-alpha_0.png", "layer_1_ColorDodge.png", "layer-alpha_1.png",
                            "layer_2_LinearDodge.png", "layer-alpha_2.png"])
    from PIL import Image
    img = np.asarray(Image.open(tmp_path / "layer_1_ColorDodge.png"))
    assert img.shape == (h, w, 4) and img.dtype == np.uint8
    np.testing.assert_array_equal(img, (np.clip(packed[1], 0, 1) * 255).astype(np.uint8))
    alpha = np.asarray(Image.open(tmp_path / "layer-alpha_2.png"))
    np.testing.assert_array_equal(alpha, (np.clip(packed[2, ..., 3], 0, 1) * 255).astype(np.uint8))
    # Reading: 8-bit channels / 255.
    rgb = uio.read_image(str(tmp_path / "layer_0_Normal.png"))
    assert rgb.shape == (h, w, 3) and rgb.dtype == np.float64
    np.testing.assert_array_equal(rgb * 255.0, (np.clip(packed[0, ..., :3], 0, 1) * 255).astype(np.uint8))
    with pytest.raises(ValueError):
        uio.export_layers(packed, str(tmp_path), "x", with_blend_mode_suffix=True, layer_infos=infos[:2])


def test_cpp_host_of_the_cpp_api(tmp_path):
    """A C++ program using the C++ API reads and writes the layer-info file
    and meets the buffer API's argument rules (no device work)."""
    import subprocess
    from tests.cpp_client import build
    exe = build(tmp_path)
    rng = np.random.default_rng(9)
    src = tmp_path / "in"
    src.mkdir()
    uio.export_layer_infos(syn.make_layers(rng, [0, 1, 2, 9]), str(src))
    out = tmp_path / "out"
    out.mkdir()
    r = subprocess.run([exe, "host", str(src / "layer_infos.json"), str(out)], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "ok 4"
    assert uio.import_layer_infos(str(out / "layer_infos.json"))[3].mode == 9
