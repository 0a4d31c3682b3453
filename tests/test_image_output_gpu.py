"""Capture formats of a GPU-rendered film: the film read as linear RGB, its
identity hash (C library = oracle restatement; the same for the same render
on another renderer), its EXR (read back bit for bit) and the JSON report
with the frame telemetry."""
import importlib.util
import json
from pathlib import Path

import numpy as np
import pytest

from renderingengine_b200 import images, scenes
from renderingengine_b200.traversal import Scene
from renderingengine_b200.wavefront import FILM_MEAN, Renderer, frame_constants

pytestmark = pytest.mark.gpu


def _render(sd, scene, w, h, frames, depth):
    r = Renderer(w, h, depth)
    r.set_scene(scene, sd)
    rays = shadows = 0
    for f in range(frames):
        r.render(frame_constants(sd.camera, w, h, f, depth, seed=1), accumulate=f > 0)
        t = r.collect()
        rays, shadows, nonfinite = t.total_path_rays, t.total_shadow_rays, t.non_finite
    return r, rays, shadows, nonfinite


def test_film_capture_formats(native, oracle, tmp_path):
    sd = scenes.cornell_reference()
    w, h, frames, depth = 96, 64, 8, 8
    scene = Scene(sd.triangles, sd.fingerprint)
    r, rays, shadows, nonfinite = _render(sd, scene, w, h, frames, depth)
    rgb = images.film_rgb(r, FILM_MEAN, w, h)
    assert rgb.shape == (h, w, 3) and np.isfinite(rgb).all() and rgb.max() > 0
    digest = images.hash_linear_rgb(rgb)
    assert digest == oracle.linear_rgb_hash(rgb)
    again, *_ = _render(sd, scene, w, h, frames, depth)
    assert images.hash_linear_rgb(images.film_rgb(again, FILM_MEAN, w, h)) == digest
    spec = importlib.util.spec_from_file_location("make_golden", Path(__file__).parent / "golden" / "make_golden.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    path = tmp_path / "cornell.exr"
    images.write_exr(path, rgb)
    np.testing.assert_array_equal(mod.decode_exr(path).view(np.uint32), rgb.view(np.uint32))
    text = images.write_report(tmp_path / "cornell.json", width=w, height=h, spp=frames, max_bounces=depth, seed=1,
                               threads=0, scene_hash=sd.fingerprint, image_hash=digest, ray_count=rays,
                               shadow_ray_count=shadows, non_finite_count=nonfinite, elapsed_ms=0.0,
                               exr=str(path))
    rep = json.loads(text)
    assert rep["linear_rgb_hash_fnv1a64"] == f"0x{digest:016x}" and rep["ray_count"] == rays > 0
