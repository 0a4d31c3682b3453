"""Seeded workload generators (renderingengine_b200/workloads.py): the
64-view batch mix, the Poisson request stream over the 16-scene pool, the
camera path, and the first-in-first-out latency model of serial plain
launches."""
import numpy as np

from renderingengine_b200 import scenes
from renderingengine_b200 import workloads as W


def test_batch_views_follow_the_mix():
    sl = [(scenes.cornell_box(), 0, False, 0.05)] * 3 + [(scenes.cornell_box(), 1, True, 0.02)]
    views = W.batch_views(sl)
    key = lambda vs: [(v.scene, v.width, v.height, v.spp, v.seed, tuple(v.camera.position)) for v in vs]
    assert len(views) == 64 and key(views) == key(W.batch_views(sl))  # seeded
    assert {(v.width, v.height) for v in views} <= set(W.BATCH_RESOLUTIONS)
    assert {v.spp for v in views} == set(W.BATCH_SPP)
    assert [v.scene for v in views] == [k % 4 for k in range(64)]
    assert all(v.restir == (v.scene == 3) for v in views)
    assert len({v.seed for v in views}) == 64


def test_request_stream_is_a_seeded_prefix():
    a, b = W.request_stream(50), W.request_stream(200)
    assert a == b[:50]
    t = np.array([q.arrival for q in b])
    assert np.all(np.diff(t) > 0)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert 0.5 / W.SERVE_RATE < gaps.mean() < 2.0 / W.SERVE_RATE
    assert {q.spp for q in b} == set(W.SERVE_SPP) and {(q.width, q.height) for q in b} == set(W.SERVE_RESOLUTIONS)
    assert 0.3 < np.mean([q.restir for q in b]) < 0.7


def test_serving_pool_sizes_are_log_spaced():
    pool = W.serving_pool()
    n = np.array([r.triangles for r in pool])
    assert len(pool) == 16 and n[0] == 10_000 and n[-1] == 5_000_000
    ratios = n[1:] / n[:-1]
    assert np.allclose(ratios, ratios[0], rtol=1e-3)
    assert [r.kind for r in pool[:2]] == ["heightfield", "soup"]


def test_camera_path_is_smooth_and_seeded():
    cam = scenes.Camera.look_at((0.5, 0.55, -0.35), (0.5, 0.05, 0.55), 45.0)
    p1 = W.camera_path(cam, 60)
    p2 = W.camera_path(cam, 60)
    eyes = np.array([c.position for c in p1])
    assert np.array_equal(eyes, np.array([c.position for c in p2]))
    step = np.linalg.norm(np.diff(eyes, axis=0), axis=1)
    assert step.max() < 0.05 and step.mean() > 1e-4
    assert np.abs(eyes - cam.position).max() < 0.3


def test_fifo_latencies():
    lat, span = W.fifo_latencies([0.0, 0.1, 0.15, 1.0], [0.2, 0.2, 0.05, 0.1])
    # starts 0, 0.2, 0.4, 1.0 -> done 0.2, 0.4, 0.45, 1.1
    np.testing.assert_allclose(lat, [0.2, 0.3, 0.3, 0.1])
    assert abs(span - 1.1) < 1e-12
