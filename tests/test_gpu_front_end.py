"""The front end on either side of the path, on the GPU: an image file and a
layer-info file in, both passes through the C++ API from a C++ program and
through the Python mirror, layer images out.

Checks: the C++ host and the C ABI give bit-identical results from the same
files; the layers read from the file reach the solver unchanged (the FP64
solve of the file's image matches the oracle run on the same layers); the
written layer images follow the 8-bit rules.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle
from tests.parity import PIXEL_FRACTION, report
from unblending_b200 import io as uio
from unblending_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def test_files_in_layers_out(cuda, tmp_path):
    pytest.importorskip("PIL")
    from tests.cpp_client import build
    wl = syn.generate(40, 32, [0, 1, 2, 6], (4.0, 12.0), seed=31)
    uio.save_image(str(tmp_path / "input.png"), wl.image)
    uio.export_layer_infos(wl.layers, str(tmp_path))
    image = uio.read_image(str(tmp_path / "input.png"))          # 8-bit quantized target
    layers = uio.import_layer_infos(str(tmp_path / "layer_infos.json"))
    h, w, _ = image.shape
    L = len(layers)

    # C++ host through the C++ API.
    exe = build(tmp_path)
    image.tofile(tmp_path / "image.f64")
    r = subprocess.run([exe, "solve", str(tmp_path / "layer_infos.json"), str(tmp_path / "image.f64"), str(w), str(h),
                        str(tmp_path / "first.f64"), str(tmp_path / "final.f64")], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    first_cpp = np.fromfile(tmp_path / "first.f64").reshape(L, h, w, 4)
    final_cpp = np.fromfile(tmp_path / "final.f64").reshape(L, h, w, 4)

    # Python mirror of the same calls.
    first = cuda.compute_color_unmixing(image, layers, True)
    final = cuda.perform_matte_refinement(image, first, layers, True, True)
    assert np.array_equal(first, first_cpp) and np.array_equal(final, final_cpp)

    # The file's layers reach the solver unchanged: FP64 solve vs the oracle
    # on the same layers and image.
    out64, _, _, _ = cuda.unmix_ex(image, layers, solver=cuda.solver_options(precision=1))
    x, _ = oracle.unmix(image, layers)
    r64 = report(out64, oracle.pack(x, L, w, h), layers, False)
    assert r64["frac_rgba_1e-3"] >= PIXEL_FRACTION, r64

    paths = uio.export_layers(final, str(tmp_path), "layer", with_alpha_channel=True, with_blend_mode_suffix=True,
                              layer_infos=layers)
    assert len(paths) == 2 * L and all(os.path.exists(p) for p in paths)
    back = uio.read_image(paths[0])
    np.testing.assert_array_equal(np.round(back * 255), (np.clip(final[0, ..., :3], 0, 1) * 255).astype(np.uint8))
