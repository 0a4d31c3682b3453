"""Alpha-masked geometry on the device (re_scene_set_alpha_masks): the
checkerboard closed form through closest- and any-hit batches on both
hierarchies, invalid mappings reported as invalid hits, and wavefront films
of a scene with 6,000 masked leaf triangles equal to the oracle's pixel for
pixel under every traversal loop, from host and from device records."""
import numpy as np
import pytest

import alpha_scenes as S
from helpers import OracleScene
from renderingengine_b200 import _native as N
from renderingengine_b200 import scenes
from renderingengine_b200.traversal import Scene
from renderingengine_b200.wavefront import FILM_SAMPLE, Renderer, frame_constants

pytestmark = pytest.mark.gpu
RTOL, ATOL, MIN_FRACTION = 1e-4, 1e-6, 0.999


def _ray_records(x, y):
    r = np.zeros((len(x), 8), np.float32)
    r[:, 0], r[:, 1], r[:, 2], r[:, 3] = x, y, 1.0, 1e-4
    r[:, 6], r[:, 7] = -1.0, 1e30
    return scenes.to_ray_records(r)


@pytest.mark.parametrize("build", [N.BUILD_FLATTENED_SAH, N.BUILD_LBVH], ids=["sah", "lbvh"])
def test_checkerboard_closed_form_on_device(native, build):
    sd = S.checker_quads()
    scene = Scene(sd.triangles, sd.fingerprint, 1, build)
    scene.set_alpha_masks(sd.extra["alpha"])
    c = (np.arange(S.CHECKER * 4) + 0.5) / (S.CHECKER * 4)
    x, y = (a.ravel() for a in np.meshgrid(c, c))
    keep = S.checker_expected(x, y)
    for any_hit in (False, True):
        hits = scene.trace(_ray_records(x, y), any_hit=any_hit)
        assert (hits["metadata"][:, 1] == N.HIT_KIND_TRIANGLE).all()
        t = hits["position_t"][:, 3]
        np.testing.assert_array_equal(t == np.float32(1.0), keep)
        np.testing.assert_array_equal(t == np.float32(2.0), ~keep)
    # An invalid mapping (a sampler id the scene does not hold) ends traversal as invalid.
    bad = dict(sd.extra["alpha"], materials=np.concatenate([S.v0_material(1.0, 0.5, 0, S.SAMPLER + 1),
                                                            S.v0_material()]))
    scene.set_alpha_masks(bad)
    hits = scene.trace(_ray_records(x, y))
    assert (hits["metadata"][:, 1] == N.HIT_KIND_INVALID).all()
    scene.close()


@pytest.mark.parametrize("traversal", [0, 1, 2, 4, 5, 6])
@pytest.mark.parametrize("build", [N.BUILD_FLATTENED_SAH, N.BUILD_LBVH], ids=["sah", "lbvh"])
def test_foliage_film_matches_oracle(native, oracle, build, traversal):
    sd = S.foliage()
    w, h, depth = 160, 96, 6
    scene = Scene(sd.triangles, sd.fingerprint, 1, build)
    scene.set_alpha_masks(sd.extra["alpha"])
    r = Renderer(w, h, depth)
    r.set_scene(scene, sd)
    r.set_tuning(traversal=traversal)
    fc = frame_constants(sd.camera, w, h, 2, depth, seed=0xA1FA5)
    r.render(fc, accumulate=False)
    tel = r.collect()
    nodes, order = scene.export_flat()
    inp = oracle.OracleRenderInputs(sd, nodes, order)
    ref, rays, shadows = oracle.render(inp, fc)
    got = r.read(FILM_SAMPLE, w * h)[:, :3]
    ok = (np.abs(got - ref["sample"][:, :3]) <= ATOL + RTOL * np.abs(ref["sample"][:, :3])).all(axis=1)
    assert ok.mean() >= MIN_FRACTION, ok.mean()
    # Every pixel outside the tolerance evaluated a libm transcendental on its path.
    assert (ref["libm_calls"][~ok] > 0).all()
    assert abs(tel.path_rays - rays) <= max(2, rays // 2000)
    assert abs(tel.shadow_rays - shadows) <= max(2, shadows // 2000)
    assert tel.fatal_mask == 0 and tel.non_finite == 0
    r.close()
    scene.close()


def test_foliage_from_device_records_equals_host_records(native):
    import torch

    sd = S.foliage(seed=5, leaves=1500)
    host = Scene(sd.triangles, sd.fingerprint, 1, N.BUILD_LBVH)
    host.set_alpha_masks(sd.extra["alpha"])
    d = torch.from_numpy(np.ascontiguousarray(sd.triangles).view(np.uint8).copy()).cuda()
    dev = Scene.from_device(d.data_ptr(), len(sd.triangles), sd.fingerprint)
    dev.set_alpha_masks(sd.extra["alpha"])
    rays = scenes.to_ray_records(scenes.pinhole_rays(sd.camera, 256, 160, seed=4))
    a, b = host.trace(rays), dev.trace(rays)
    np.testing.assert_array_equal(a.view(np.uint8), b.view(np.uint8))
    assert (a["metadata"][:, 1] != N.HIT_KIND_INVALID).all()
    host.close()
    dev.close()
