"""Batched views (re_renderer_render_views): many cameras over several
resident scenes in one persistent launch give, view for view, bit-identical
films to the same views rendered alone (per-path random streams are keyed
by the pixel within the view and the sample)."""
import numpy as np
import pytest

from renderingengine_b200 import _native as N
from renderingengine_b200 import scenes
from renderingengine_b200.scenes import Camera
from renderingengine_b200.traversal import Scene
from renderingengine_b200.wavefront import FILM_MEAN, FILM_SAMPLE, Renderer, frame_constants

pytestmark = pytest.mark.gpu


def _shift(cam: Camera, k: float) -> Camera:
    pos = (np.asarray(cam.position, np.float64) + np.asarray(cam.right, np.float64) * k).astype(np.float32)
    return Camera(pos, cam.forward, cam.right, cam.up, cam.tan_half_fov)


@pytest.fixture(scope="module")
def world():
    datas = [scenes.cornell_box(),
             scenes.add_emissive_triangles(scenes.heightfield_scene(grid=48, spheres=48, seed=2), count=200, seed=5),
             scenes.triangle_soup(30000, seed=4)]
    built = [Scene(sd.triangles, 100 + i) for i, sd in enumerate(datas)]
    return datas, built


def _views(datas):
    """(slot, width, height, depth, estimator, light selection, camera shift)."""
    return [(0, 64, 48, 4, 2, 0, 0.0), (1, 96, 64, 6, 2, 1, 0.0), (2, 40, 40, 3, 1, 0, 0.0),
            (1, 80, 48, 4, N.ESTIMATOR_RESTIR_PRIMARY, 1, 0.002), (0, 32, 32, 8, 0, 0, 0.01),
            (1, 48, 48, 5, 2, 1, 0.004)]


def test_batched_views_equal_views_alone(native, world):
    datas, built = world
    specs = _views(datas)
    batch = Renderer(256, 256, 8)
    for slot in range(3):
        sel = 1 if slot == 1 else 0
        batch.bind_scene(slot, built[slot], datas[slot], light_selection=sel)
    batch.set_restir(candidates=8, spatial_neighbors=3)
    # Path ranges with gaps between the views.
    offsets, cur = [], 0
    for (_, w, h, *_rest) in specs:
        cur += 37
        offsets.append(cur)
        cur += w * h
    samples = 3
    got = {}
    for smp in range(samples):
        views = []
        for k, (slot, w, h, depth, est, sel, sh) in enumerate(specs):
            cam = _shift(datas[slot].camera, sh * smp)
            views.append(dict(frame=frame_constants(cam, w, h, 7 + smp, depth, estimator=est, light_selection=sel,
                                                    seed=0xABC + k),
                              slot=slot, offset=offsets[k], accumulate=smp > 0, key=1000 + k))
        batch.render_views(views)
        tel = batch.collect()
        assert tel.fatal_mask == 0
        for k, (slot, w, h, *_r) in enumerate(specs):
            got[(k, smp)] = batch.read_view(FILM_SAMPLE, offsets[k], w * h)
    means = {k: batch.read_view(FILM_MEAN, offsets[k], s[1] * s[2]) for k, s in enumerate(specs)}
    for k, (slot, w, h, depth, est, sel, sh) in enumerate(specs):
        alone = Renderer(w, h, 8)
        alone.set_scene(built[slot], datas[slot], light_selection=sel)
        alone.set_restir(candidates=8, spatial_neighbors=3)
        for smp in range(samples):
            cam = _shift(datas[slot].camera, sh * smp)
            alone.render(frame_constants(cam, w, h, 7 + smp, depth, estimator=est, light_selection=sel,
                                         seed=0xABC + k), accumulate=smp > 0)
            alone.collect()
            ref = alone.read(FILM_SAMPLE, w * h)
            np.testing.assert_array_equal(got[(k, smp)].view(np.uint32), ref.view(np.uint32),
                                          err_msg=f"view {k} sample {smp}")
        np.testing.assert_array_equal(means[k].view(np.uint32), alone.read(FILM_MEAN, w * h).view(np.uint32))


def test_batch_contract(native, world):
    datas, built = world
    r = Renderer(128, 128, 4)
    r.bind_scene(2, built[0], datas[0])
    fc = frame_constants(datas[0].camera, 64, 64, 0, 4)
    with pytest.raises(N.NativeError) as e:
        r.render_views([dict(frame=fc, slot=2, offset=0), dict(frame=fc, slot=2, offset=4000)])
    assert e.value.code == N.INVALID_ARGUMENT  # overlapping path ranges
    with pytest.raises(N.NativeError) as e:
        r.render_views([dict(frame=fc, slot=5, offset=0)])
    assert e.value.code == N.MISSING_SCENE
    with pytest.raises(N.NativeError) as e:
        r.render_views([dict(frame=fc, slot=2, offset=128 * 128 - 100)])
    assert e.value.code == N.INVALID_ARGUMENT  # beyond the path capacity
    r.render_views([dict(frame=fc, slot=2, offset=0), dict(frame=fc, slot=2, offset=8192)])
    assert r.collect().fatal_mask == 0
    r.unbind_scene(2)
    with pytest.raises(N.NativeError):
        r.render_views([dict(frame=fc, slot=2, offset=0)])
    assert r.capacity == 128 * 128
