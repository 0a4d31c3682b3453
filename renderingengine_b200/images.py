"""Image outputs of a film: the reference harness's capture formats.

`film_rgb` reads a film plane as a (height, width, 3) linear-RGB image (top
row first, the order RayGen numbers pixels), `hash_linear_rgb` is the
reference's identity hash of such an image (HashLinearRgbPixels,
src/rt/cpu/ImageOutput.cpp:343-380), `write_exr` its 32-bit float OpenEXR
output (WriteLinearRgbExr, ImageOutput.cpp:156-216), and `write_report` the
JSON report of a render (WriteReport, src/rt/cpu/ReferenceMain.cpp:214-259)
with the same keys and formatting.  Hash and EXR run in the C library
(re_image_hash_linear_rgb, re_image_write_exr).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _native as N

ABI_V0_VERSION = 1  # contracts/AbiVersion.hpp:9, the report's contract_numeric


def _rgb(image: np.ndarray) -> np.ndarray:
    img = np.ascontiguousarray(image, np.float32)
    if img.ndim != 3 or img.shape[2] != 3:
        raise ValueError("expected a (height, width, 3) linear-RGB image")
    return img


def film_rgb(renderer, plane: int, width: int, height: int, offset: int = 0) -> np.ndarray:
    """A film plane of a view as a (height, width, 3) float32 image."""
    px = renderer.read_view(plane, offset, width * height) if offset else renderer.read(plane, width * height)
    return np.ascontiguousarray(px[:, :3].reshape(height, width, 3))


def hash_linear_rgb(image: np.ndarray) -> int:
    """64-bit FNV-1a identity hash of a linear-RGB image (re_image_hash_linear_rgb)."""
    img = _rgb(image)
    h, w = img.shape[:2]
    out = C.c_uint64(0)
    N.check(N.load().re_image_hash_linear_rgb(w, h, N.ptr(img), img.size, C.byref(out)))
    return int(out.value)


def write_exr(path, image: np.ndarray) -> None:
    """Writes a 32-bit float RGB OpenEXR file (ZIP compression)."""
    img = _rgb(image)
    h, w = img.shape[:2]
    N.check(N.load().re_image_write_exr(str(path).encode(), w, h, N.ptr(img), img.size))


def write_report(path, *, width: int, height: int, spp: int, max_bounces: int, seed: int, threads: int,
                 scene_hash: int, image_hash: int, ray_count: int, shadow_ray_count: int, non_finite_count: int,
                 elapsed_ms: float, exr: str = "", preview_bmp: str = "",
                 scope: str = "cuda-wavefront-film-v0") -> str:
    """The JSON report of a render in WriteReport's key order and number
    formats (hashes as 0x%016x, elapsed with three decimals); returns it."""
    def esc(s: str) -> str:
        out = []
        for ch in s:
            out.append({'"': '\\"', "\\": "\\\\", "\b": "\\b", "\f": "\\f", "\n": "\\n", "\r": "\\r",
                        "\t": "\\t"}.get(ch, ch))
        return "".join(out)

    text = ("{\n"
            f'  "scope": "{esc(scope)}",\n'
            '  "contract": "abi-v0",\n'
            f'  "contract_numeric": {ABI_V0_VERSION},\n'
            f'  "width": {width},\n'
            f'  "height": {height},\n'
            f'  "spp": {spp},\n'
            f'  "max_bounces": {max_bounces},\n'
            f'  "seed": {seed},\n'
            f'  "threads_requested": {threads},\n'
            f'  "scene_hash_fnv1a64": "0x{scene_hash:016x}",\n'
            f'  "linear_rgb_hash_fnv1a64": "0x{image_hash:016x}",\n'
            f'  "ray_count": {ray_count},\n'
            f'  "shadow_ray_count": {shadow_ray_count},\n'
            f'  "non_finite_count": {non_finite_count},\n'
            f'  "elapsed_ms": {elapsed_ms:.3f},\n'
            f'  "exr": "{esc(exr)}",\n'
            f'  "preview_bmp": "{esc(preview_bmp)}"\n'
            "}\n")
    Path(path).write_text(text)
    return text
