"""Capture formats of a film (re_image_hash_linear_rgb, re_image_write_exr,
images.write_report) on the CPU: the identity hash against the reference's
golden Cornell report and the oracle restatement, the EXR through an
independent decoder, the JSON report's keys and formats."""
import importlib.util
import json
from pathlib import Path

import numpy as np
import pytest

from renderingengine_b200 import _native as N
from renderingengine_b200 import images

GOLDEN = Path(__file__).parent / "golden"


def _decoder():
    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.decode_exr


def _golden():
    rgb = np.load(GOLDEN / "cornell_256x256_64spp_seed1.npz")["rgb"]
    meta = json.loads((GOLDEN / "cornell_256x256_64spp_seed1.json").read_text())
    return rgb, meta


def test_hash_matches_the_reference_golden_report(native, oracle):
    """The golden EXR's pixels hash to the golden report's
    linear_rgb_hash_fnv1a64 (rt/cpu/references/wave1/cornell-256x256-64spp-seed1.json),
    through the C library and through the oracle restatement."""
    rgb, meta = _golden()
    want = int(meta["linear_rgb_hash"], 16)
    assert images.hash_linear_rgb(rgb) == want
    assert oracle.linear_rgb_hash(rgb) == want


def test_hash_edge_cases(native, oracle):
    rng = np.random.default_rng(4)
    for h, w in [(1, 1), (3, 7), (17, 5)]:
        img = rng.standard_normal((h, w, 3)).astype(np.float32)
        img.reshape(-1)[::5] = 0.0
        assert images.hash_linear_rgb(img) == oracle.linear_rgb_hash(img)
        neg = img.copy()
        neg[neg == 0.0] = -0.0
        assert images.hash_linear_rgb(neg) == images.hash_linear_rgb(img)  # -0 folds to +0
    img = rng.random((4, 4, 3)).astype(np.float32)
    assert images.hash_linear_rgb(img) != images.hash_linear_rgb(img.reshape(2, 8, 3))  # dimensions are hashed
    for bad in (np.zeros((0, 4, 3), np.float32), np.full((2, 2, 3), np.nan, np.float32),
                np.full((2, 2, 3), np.inf, np.float32)):
        with pytest.raises(N.NativeError) as e:
            images.hash_linear_rgb(bad)
        assert e.value.code == N.INVALID_ARGUMENT
    lib = N.load()
    import ctypes as C
    out = C.c_uint64(7)
    ok = np.zeros(12, np.float32)
    assert lib.re_image_hash_linear_rgb(2, 2, N.ptr(ok), 11, C.byref(out)) == N.INVALID_ARGUMENT  # count
    assert out.value == 0


@pytest.mark.parametrize("shape", [(256, 256), (21, 37), (1, 1), (33, 16)])
def test_exr_round_trip(native, tmp_path, shape):
    """Written with re_image_write_exr, read back with the fixture decoder:
    every component bit for bit, for compressible (golden, flat) and
    incompressible (noise, stored raw) blocks and a ragged last block."""
    decode = _decoder()
    h, w = shape
    if shape == (256, 256):
        img, _ = _golden()
    else:
        rng = np.random.default_rng(h * 100 + w)
        img = rng.standard_normal((h, w, 3)).astype(np.float32) * np.float32(1e3)
        img[: h // 2] = 0.25  # a flat half compresses, the noise half does not
    path = tmp_path / "film.exr"
    images.write_exr(path, img)
    back = decode(path)
    assert back.shape == img.shape
    np.testing.assert_array_equal(back.view(np.uint32), np.ascontiguousarray(img).view(np.uint32))
    with pytest.raises(N.NativeError):
        images.write_exr(tmp_path / "bad.exr", np.full((2, 2, 3), np.nan, np.float32))
    with pytest.raises(N.NativeError):
        images.write_exr(tmp_path / "no" / "such" / "dir.exr", img)


def test_report_keys_and_formats(tmp_path):
    text = images.write_report(tmp_path / "r.json", width=256, height=256, spp=64, max_bounces=8, seed=1, threads=0,
                               scene_hash=0x80597851AE8052C2, image_hash=0x6B666A36F93DF86D, ray_count=14714873,
                               shadow_ray_count=8572432, non_finite_count=0, elapsed_ms=2289.3291,
                               exr="out/cornell \"a\".exr")
    d = json.loads(text)
    assert list(d) == ["scope", "contract", "contract_numeric", "width", "height", "spp", "max_bounces", "seed",
                       "threads_requested", "scene_hash_fnv1a64", "linear_rgb_hash_fnv1a64", "ray_count",
                       "shadow_ray_count", "non_finite_count", "elapsed_ms", "exr", "preview_bmp"]
    assert d["scene_hash_fnv1a64"] == "0x80597851ae8052c2" and d["linear_rgb_hash_fnv1a64"] == "0x6b666a36f93df86d"
    assert '"elapsed_ms": 2289.329,' in text and d["exr"] == 'out/cornell "a".exr'
    assert (tmp_path / "r.json").read_text() == text
