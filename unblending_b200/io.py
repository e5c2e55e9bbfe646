"""Input and output formats on either side of the path: the layer-info JSON
file and image files.

Layer infos (LayerInfos.md; unblending/src/unblending_io.cpp:125-170 of the
reference): parsing and formatting run in the library's C++ reader
(`unblending_parse_layer_infos` / `unblending_format_layer_infos`), so the
precision matrices equal those the C++ API computes.

Images (unblending/io/image_qt.cpp:6-34,65-82): an input image reads as
8-bit channels / 255; a layer is written as 8-bit RGBA with each channel
clipped to [0, 1] and truncated after scaling by 255, to
`<prefix>_<index>[_<Mode>].png`, its alpha (with_alpha_channel) to
`<prefix>-alpha_<index>.png`. The reference draws that alpha map through a
colour map; it is written here as 8-bit grey. Image files need Pillow.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import OK, BUFFER_TOO_SMALL, _check, _layers, lib
from .synthetic import LayerSpec, UnblendingLayer

MODE_NAMES = ["Normal", "Multiply", "Screen", "Overlay", "Darken", "Lighten", "ColorDodge", "ColorBurn",
              "HardLight", "SoftLight", "Difference", "Exclusion", "LinearDodge"]


# ------------------------------------------------------------ layer infos --
def parse_layer_infos(text: str) -> list[LayerSpec]:
    """Layer specs of a layer-info JSON text, bottom layer first. Raises
    ValueError for malformed text, an unknown mode name or a singular
    covariance."""
    data = text.encode("utf-8")
    count = ctypes.c_size_t(0)
    rc = lib.unblending_parse_layer_infos(data, None, 0, ctypes.byref(count))
    if rc not in (OK, BUFFER_TOO_SMALL):
        _check(rc)
    arr = (UnblendingLayer * max(1, count.value))()
    _check(lib.unblending_parse_layer_infos(data, arr, count.value, ctypes.byref(count)))
    out = []
    for k in range(count.value):
        l = arr[k]
        prec = np.array(l.precision[:], dtype=np.float64).reshape(3, 3)
        out.append(LayerSpec(mode=int(l.blend_mode), mean=np.array(l.mean[:], dtype=np.float64),
                             covariance=np.linalg.inv(prec), comp=(l.comp_x, l.comp_y, l.comp_z),
                             precision_matrix=prec))
    return out


def import_layer_infos(path: str) -> list[LayerSpec]:
    """Layer specs of a layer-info JSON file (import_layer_infos)."""
    with open(path, "r", encoding="utf-8") as f:
        return parse_layer_infos(f.read())


def format_layer_infos(layers) -> str:
    """Layer-info JSON text of layer specs (the precision is inverted back
    to the covariance)."""
    arr, n = _layers(layers)
    length = ctypes.c_size_t(0)
    rc = lib.unblending_format_layer_infos(arr, n, None, 0, ctypes.byref(length))
    if rc not in (OK, BUFFER_TOO_SMALL):
        _check(rc)
    buf = ctypes.create_string_buffer(length.value + 1)
    _check(lib.unblending_format_layer_infos(arr, n, buf, len(buf), ctypes.byref(length)))
    return buf.value.decode("utf-8")


def export_layer_infos(layers, directory: str) -> str:
    """Writes <directory>/layer_infos.json (export_layer_infos); returns the path."""
    path = os.path.join(directory, "layer_infos.json")
    with open(path, "w", encoding="utf-8") as f:
        f.write(format_layer_infos(layers))
    return path


# ----------------------------------------------------------------- images --
def _pil():
    try:
        from PIL import Image
    except ImportError as e:   # image files only; the solver does not need it
        raise ImportError("image files need Pillow (PIL)") from e
    return Image


def to_8bit(values: np.ndarray) -> np.ndarray:
    """Channels in [0, 1] to 8 bits the reference's way: clip, scale by 255,
    truncate (image_processing.cpp:57-62)."""
    return (np.clip(np.asarray(values, dtype=np.float64), 0.0, 1.0) * 255.0).astype(np.uint8)


def read_image(path: str) -> np.ndarray:
    """(height, width, 3) float64 RGB in [0, 1] of an image file: each 8-bit
    channel / 255 (image_qt.cpp:17-34)."""
    Image = _pil()
    with Image.open(path) as im:
        rgb = np.asarray(im.convert("RGBA"), dtype=np.float64)[..., :3]
    return np.ascontiguousarray(rgb / 255.0)


def save_image(path: str, values: np.ndarray) -> None:
    """Writes (h, w, 3|4) values in [0, 1] (or (h, w) grey) as an 8-bit PNG."""
    Image = _pil()
    v = to_8bit(values)
    mode = {2: "L"}.get(v.ndim) or {3: "RGB", 4: "RGBA"}[v.shape[2]]
    Image.fromarray(v, mode=mode).save(path)


def export_layers(layers: np.ndarray, directory: str, prefix: str, with_alpha_channel: bool = False,
                  with_blend_mode_suffix: bool = False, layer_infos=None) -> list[str]:
    """Writes each layer of a packed (L, h, w, 4) result as
    <directory>/<prefix>_<index>[_<Mode>].png and, with_alpha_channel, its
    alpha as <prefix>-alpha_<index>.png; returns the paths written."""
    layers = np.asarray(layers, dtype=np.float64)
    if layers.ndim != 4 or layers.shape[3] != 4:
        raise ValueError("layers must be packed (L, height, width, 4)")
    if with_blend_mode_suffix and (layer_infos is None or len(layer_infos) != layers.shape[0]):
        raise ValueError("the blend-mode suffix needs one layer info per layer")
    paths = []
    for index in range(layers.shape[0]):
        suffix = "_" + MODE_NAMES[layer_infos[index].mode] if with_blend_mode_suffix else ""
        path = os.path.join(directory, f"{prefix}_{index}{suffix}.png")
        save_image(path, layers[index])
        paths.append(path)
        if with_alpha_channel:
            path = os.path.join(directory, f"{prefix}-alpha_{index}.png")
            save_image(path, layers[index, ..., 3])
            paths.append(path)
    return paths
