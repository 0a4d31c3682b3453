"""Render server (re_server_*): requests of different scenes, extents,
sample counts and estimators arrive over time, are admitted as path ranges
and budget free up, and share launches; each request's film equals the same
request rendered alone, also when the HBM budget forces scenes out and back
in (least recently used first)."""
import numpy as np
import pytest

from renderingengine_b200 import _native as N
from renderingengine_b200 import scenes
from renderingengine_b200.serving import RenderServer
from renderingengine_b200.traversal import Scene
from renderingengine_b200.wavefront import FILM_MEAN, Renderer, frame_constants

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pool():
    return {
        10: (scenes.cornell_box(), 0),
        11: (scenes.add_emissive_triangles(scenes.heightfield_scene(grid=48, spheres=48, seed=2), count=200, seed=5), 1),
        12: (scenes.triangle_soup(40000, seed=4), 0),
        13: (scenes.heightfield_scene(grid=64, spheres=32, seed=9), 0),
    }


def _requests(rng, keys, count):
    out = []
    for i in range(count):
        key = int(rng.choice(keys))
        w, h = [(64, 48), (96, 64), (48, 48), (128, 72)][int(rng.integers(0, 4))]
        spp = int(rng.choice([1, 2, 4]))
        est = int(rng.choice([2, 2, 1, N.ESTIMATOR_RESTIR_PRIMARY]))
        depth = int(rng.integers(2, 7))
        out.append(dict(key=key, w=w, h=h, spp=spp, est=est, depth=depth, sample=int(rng.integers(0, 50)),
                        seed=0x1000 + i, arrival=0.002 * i))
    return out


def _alone(pool, q):
    sd, sel = pool[q["key"]]
    r = Renderer(q["w"], q["h"], 8)
    r.set_scene(Scene(sd.triangles, 77, 1, N.BUILD_LBVH), sd, light_selection=sel)
    r.set_restir()
    for k in range(q["spp"]):
        r.render(frame_constants(sd.camera, q["w"], q["h"], q["sample"] + k, q["depth"], estimator=q["est"],
                                 light_selection=sel, seed=q["seed"]), accumulate=k > 0)
    r.collect()
    return r.read(FILM_MEAN, q["w"] * q["h"])


def _serve(pool, reqs, budget, capacity=40000):
    srv = RenderServer(budget, capacity, max_depth=8, max_batch_views=16)
    for key, (sd, sel) in pool.items():
        srv.register_scene(key, sd, light_selection=sel)
    t0 = srv.clock()
    ids = []
    for q in reqs:
        sd, sel = pool[q["key"]]
        fc = frame_constants(sd.camera, q["w"], q["h"], q["sample"], q["depth"], estimator=q["est"],
                             light_selection=sel, seed=q["seed"])
        ids.append(srv.submit(q["key"], fc, q["spp"], arrival_time=t0 + q["arrival"]))
    srv.drain()
    return srv, ids


def test_served_requests_equal_requests_alone(native, pool):
    rng = np.random.default_rng(3)
    reqs = _requests(rng, list(pool), 24)
    srv, ids = _serve(pool, reqs, budget=40 << 30)
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["launches"] < sum(q["spp"] for q in reqs)  # requests shared launches
    assert 0.0 <= st["latency_p50"] <= st["latency_p99"]
    for q, rid in zip(reqs, ids):
        s = srv.poll(rid)
        assert s.state == N.REQUEST_DONE and s.samples_done == q["spp"]
        assert s.admit_time >= s.arrival_time - 1e-6 and s.completion_time >= s.admit_time
        np.testing.assert_array_equal(srv.result(rid).view(np.uint32), _alone(pool, q).view(np.uint32),
                                      err_msg=str(q))
        srv.release(rid)


def test_budget_evicts_least_recently_used_scenes(native, pool):
    """A budget that holds the path pool and one scene at a time: scenes are
    built, evicted and rebuilt as requests alternate, results unchanged."""
    probe = RenderServer(40 << 30, 40000, max_depth=8)
    fixed = probe.stats()["resident_bytes"]
    probe.close()
    # Charge of a scene before its build, as the server states it.
    charge = {k: len(sd.triangles) * 260 + sd.materials.nbytes + len(sd.lights) * (sd.lights.itemsize + 24)
              + sd.fixture_triangles.nbytes + (1 << 20) for k, (sd, _) in pool.items()}
    rng = np.random.default_rng(5)
    reqs = _requests(rng, [11, 12, 13], 9)
    for i, q in enumerate(reqs):
        q["key"] = [11, 12, 13][i % 3]
        q["arrival"] = 0.02 * i
    srv, ids = _serve(pool, reqs, budget=fixed + max(charge[k] for k in (11, 12, 13)))
    st = srv.stats()
    assert st["completed"] == len(reqs)
    assert st["evictions"] >= 6 and st["scene_builds"] >= 7
    assert st["resident_bytes"] <= st["budget_bytes"]
    for q, rid in zip(reqs, ids):
        np.testing.assert_array_equal(srv.result(rid).view(np.uint32), _alone(pool, q).view(np.uint32))


def test_request_that_cannot_fit_fails(native, pool):
    probe = RenderServer(40 << 30, 40000, max_depth=8)
    fixed = probe.stats()["resident_bytes"]
    probe.close()
    srv = RenderServer(fixed + (1 << 20), 40000, max_depth=8)
    sd, _ = pool[12]
    srv.register_scene(12, sd)
    rid = srv.submit(12, frame_constants(sd.camera, 32, 32, 0, 3), 1)
    srv.drain()
    s = srv.poll(rid)
    assert s.state == N.REQUEST_FAILED and s.error == N.BUDGET_EXCEEDED
    with pytest.raises(N.NativeError):
        srv.submit(12, frame_constants(sd.camera, 512, 512, 0, 3), 1)  # larger than the path pool
    with pytest.raises(N.NativeError):
        srv.submit(99, frame_constants(sd.camera, 32, 32, 0, 3), 1)  # unknown scene


@pytest.mark.parametrize("window", [N.BACKFILL_DEFAULT, 0])
def test_backfilling_admits_small_requests_past_a_waiting_one(native, pool, window):
    """Two requests that need most of the path pool each and a small one
    behind them: with backfilling the small one starts while the second
    large one waits for the first to finish; with a window of 0 admission
    keeps arrival order.  Films equal the requests rendered alone."""
    sd, sel = pool[13]
    srv = RenderServer(40 << 30, 40000, max_depth=8, max_batch_views=16, backfill_window=window)
    srv.register_scene(13, sd, light_selection=sel)
    reqs = [dict(key=13, w=192, h=192, spp=6, est=2, depth=4, sample=0, seed=0x31, arrival=0.0),
            dict(key=13, w=192, h=192, spp=2, est=2, depth=4, sample=3, seed=0x32, arrival=0.0),
            dict(key=13, w=32, h=32, spp=1, est=2, depth=4, sample=5, seed=0x33, arrival=0.0)]
    t0 = srv.clock()
    ids = [srv.submit(q["key"], frame_constants(sd.camera, q["w"], q["h"], q["sample"], q["depth"], estimator=q["est"],
                                                light_selection=sel, seed=q["seed"]), q["spp"], arrival_time=t0)
           for q in reqs]
    srv.drain()
    st = [srv.poll(i) for i in ids]
    assert all(s.state == N.REQUEST_DONE for s in st)
    if window == 0:
        assert srv.stats()["backfilled"] == 0
        assert st[2].admit_time >= st[1].admit_time
    else:
        assert srv.stats()["backfilled"] >= 1
        assert st[2].admit_time < st[1].admit_time
        assert st[2].completion_time < st[1].completion_time
    for q, rid in zip(reqs, ids):
        np.testing.assert_array_equal(srv.result(rid).view(np.uint32), _alone(pool, q).view(np.uint32))
