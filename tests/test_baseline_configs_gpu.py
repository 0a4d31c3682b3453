"""The benchmark configurations at their stated sizes, against the oracle.

- Cornell workload (640x360, 1 spp per frame for 3 frames, max bounce 4,
  NEE+MIS, binned SAH with 32 bins and leaves <= 4): the progressive film of
  the three frames against the oracle's mean of the same three samples; the
  32-bin hierarchy's closest hits equal the 16-bin one's (the reference
  builds 16 bins, rt/cpu/Bvh.hpp:68).
- Traversal-bound scene (2,424,832 triangles, 1920x1080, max bounce 8, GPU
  LBVH): the full frame's film against the oracle on 65,536 seeded pixels.
- Many-light ReSTIR DI (the same scene + 10,000 emissive triangles,
  1280x720, 32 RIS candidates, M-cap 20, 5 neighbours in a 30-px disk):
  two consecutive frames' reservoirs and direct term against the oracle's
  ReSTIR on the whole frame (its spatial pass needs every pixel)."""
import numpy as np
import pytest

from renderingengine_b200 import _native as N
from renderingengine_b200 import scenes
from renderingengine_b200 import workloads as W
from renderingengine_b200.traversal import Scene
from renderingengine_b200.wavefront import FILM_MEAN, FILM_SAMPLE, Renderer, frame_constants

pytestmark = pytest.mark.gpu
RTOL, ATOL = 1e-4, 1e-6


def _close_rows(a, b):
    return np.all(np.abs(a - b) <= ATOL + RTOL * np.abs(b), axis=-1)


def test_cornell_workload_three_frames_32_bins(native, oracle):
    sd = scenes.cornell_box()
    w, h, depth = 640, 360, 4
    scene = Scene(sd.triangles, sd.fingerprint, 1, N.BUILD_FLATTENED_SAH, sah_bins=32)
    scene16 = Scene(sd.triangles, sd.fingerprint, 1, N.BUILD_FLATTENED_SAH, sah_bins=16)
    rays = scenes.to_ray_records(scenes.pinhole_rays(sd.camera, w, h, seed=9))
    a, b = scene.trace(rays), scene16.trace(rays)
    # Same closest hits, up to near-ties (equal distances within 1e-6 t).
    diff = np.flatnonzero(np.any(a["ids"] != b["ids"], axis=1))
    assert len(diff) <= len(rays) // 10000, len(diff)
    ta, tb = a["position_t"][diff, 3].astype(np.float64), b["position_t"][diff, 3].astype(np.float64)
    assert np.all(np.abs(ta - tb) <= 1e-6 * np.abs(tb))
    r = Renderer(w, h, depth)
    r.set_scene(scene, sd)
    nodes, order = scene.export_flat()
    inp = oracle.OracleRenderInputs(sd, nodes, order)
    acc = np.zeros((w * h, 3))
    for k in range(3):
        fc = frame_constants(sd.camera, w, h, k, depth, seed=47)
        r.render(fc, accumulate=k > 0)
        r.collect()
        planes, _, _ = oracle.render(inp, fc)
        acc += planes["sample"][:, :3]
    film = r.read(FILM_MEAN, w * h)[:, :3]
    ok = _close_rows(film, (acc / 3).astype(np.float32))
    assert ok.mean() >= 0.999, ok.mean()
    r.close()
    scene.close()
    scene16.close()


def test_traversal_bound_full_frame_on_seeded_pixels(native, oracle):
    sd = scenes.heightfield_scene()
    w, h, depth = 1920, 1080, 8
    scene = Scene(sd.triangles, sd.fingerprint, 1, N.BUILD_LBVH)
    r = Renderer(w, h, depth)
    r.set_scene(scene, sd)
    fc = frame_constants(sd.camera, w, h, 3, depth)
    r.render(fc, accumulate=False)
    tel = r.collect()
    assert tel.fatal_mask == 0 and tel.non_finite == 0
    film = r.read(FILM_SAMPLE, w * h)[:, :3]
    nodes, order = scene.export_flat()
    inp = oracle.OracleRenderInputs(sd, nodes, order)
    px = np.sort(np.random.default_rng(65536).choice(w * h, 65536, replace=False)).astype(np.uint32)
    ref, _, _ = oracle.render(inp, fc, pixels=px, threads=16)
    ok = _close_rows(film[px], ref["sample"][:, :3])
    assert ok.mean() >= 0.999, ok.mean()
    assert (ref["libm_calls"][~ok] > 0).all()  # mismatches only on paths that evaluated libm transcendentals
    r.close()
    scene.close()


def test_many_light_restir_720p(native, oracle):
    sd = scenes.add_emissive_triangles(scenes.heightfield_scene(), count=10000)
    w, h, depth = 1280, 720, 4
    scene = Scene(sd.triangles, sd.fingerprint)
    r = Renderer(w, h, depth)
    r.set_scene(scene, sd, light_selection=1)
    r.set_restir(**W.RESTIR_MANY_LIGHTS)
    nodes, order = scene.export_flat()
    inp = oracle.OracleRenderInputs(sd, nodes, order)
    ors = oracle.OracleRestir(inp, light_selection=1, **W.RESTIR_MANY_LIGHTS)
    n = w * h
    prev_surf = prev_pub = None
    path = W.camera_path(sd.camera, 2, seed=0xC2)
    int_words = np.r_[16:32, 40:64]
    for k, cam in enumerate(path):
        fc = frame_constants(cam, w, h, k, depth, estimator=N.ESTIMATOR_RESTIR_PRIMARY, light_selection=1)
        r.render(fc, accumulate=False)
        assert r.collect().fatal_mask == 0
        surf = r.restir_read(N.RESTIR_SURFACES, n)
        published = r.restir_read(N.RESTIR_PUBLISHED, n)
        direct = r.restir_read(N.RESTIR_DIRECT, n)
        out = ors.frame(fc, surf.view(np.float32), prev_surf, prev_pub, threads=16)
        same_int = np.all(published[:, int_words] == out["published"][:, int_words], axis=1)
        assert same_int.mean() >= 0.995, f"frame {k}: {same_int.mean():.4f}"
        ok = _close_rows(direct, out["direct"]).all(axis=0)
        assert ok.mean() >= 0.995, f"frame {k}: direct {ok.mean():.4f}"
        prev_surf, prev_pub = surf.view(np.float32), published
    r.close()
    scene.close()
