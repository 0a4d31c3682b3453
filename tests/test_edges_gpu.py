"""Edge cases of the GPU path through the C ABI: empty trace batches, the
smallest hierarchies (one, two, three and five triangles; a root that is a
leaf), one-pixel and ragged frames at the maximum path depth, a view that
ends exactly at the path capacity, and a launch of the maximum view count."""
import numpy as np
import pytest

from helpers import OracleScene, nodes_as_words
from renderingengine_b200 import _native as N
from renderingengine_b200 import scenes
from renderingengine_b200.traversal import CudaTraversalBackend, GpuSceneBuildRequest, GpuTraceBatch, Scene
from renderingengine_b200.wavefront import FILM_MEAN, FILM_SAMPLE, Renderer, frame_constants

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-4, 1e-6


def _one_triangle():
    """A single Lambert triangle under a sphere light: the hierarchy is one
    leaf, which the device layouts hang under a synthetic root."""
    pos = np.array([[[-1, 0, -1], [1, 0, -1], [0, 0, 1]]], np.float32)
    tri = scenes.canonical_triangles(pos, None, np.zeros(1, np.uint32), np.arange(1, dtype=np.uint32),
                                     np.zeros(1, np.uint32))
    mats = scenes.material(scenes.LAMBERT, base=(0.6, 0.7, 0.8))
    lights = scenes.sphere_light((0.0, 1.2, 0.0), 0.25, (8.0, 8.0, 8.0))
    cam = scenes.Camera.look_at((0.0, 1.5, -2.0), (0.0, 0.0, 0.0), 55.0)
    return scenes.SceneData("one-triangle", tri, mats, lights, np.zeros(0, scenes.FIXTURE_TRIANGLE_DTYPE), cam,
                            fingerprint=0x0101)


def _oracle_frame(oracle, sd, fc):
    os_ = OracleScene(sd)
    return oracle.render(oracle.OracleRenderInputs(sd, os_.nodes, os_.order), fc)


def _within(got, ref):
    return np.abs(got - ref) <= ATOL + RTOL * np.abs(ref)


def test_empty_trace_batches_succeed_and_write_nothing(native):
    sd = scenes.cornell_box()
    scene = Scene(sd.triangles, 21)
    empty = np.zeros(0, N.RAY_DTYPE)
    assert len(scene.trace(empty)) == 0
    assert len(scene.trace(empty, any_hit=True)) == 0
    hits, counters = scene.trace(empty, counters=True)
    assert len(hits) == 0 and counters["node_tests"] == 0 and counters["triangle_tests"] == 0
    # A zero-count batch inside non-empty buffers leaves the hit records as they were.
    be = CudaTraversalBackend()
    assert be.BuildOrUpdateScene(GpuSceneBuildRequest(sd.triangles, 21, 1))
    rays = scenes.to_ray_records(scenes.pinhole_rays(sd.camera, 8, 8))
    hits = np.zeros(len(rays), N.HIT_DTYPE)
    hits.view(np.uint8)[:] = 0xAB
    before = hits.copy()
    for fn in (be.RecordTraceClosestBatch, be.RecordTraceAnyBatch):
        st = fn(GpuTraceBatch(rays, hits, 21, 10, 20, 0, 1))
        assert st, st.message
    assert hits.tobytes() == before.tobytes()
    # The scene check still applies to an empty batch.
    assert be.RecordTraceClosestBatch(GpuTraceBatch(rays, hits, 22, 0, 0, 0, 1)).code == N.MISSING_SCENE


@pytest.mark.parametrize("count", [1, 2, 3, 5])
def test_smallest_lbvh_equals_reference_karras_build(native, oracle, count):
    """Hierarchies of one to five triangles, node for node against
    SoftwareGpu::BuildKarrasLbvh (src/rt/software_gpu/SoftwareGpu.cpp:1265-1345),
    and their hits against the flattened SAH."""
    import ctypes as C
    sd = scenes.triangle_soup(count, seed=3, max_edge=0.3)
    scene = Scene(sd.triangles, 31, 1, N.BUILD_LBVH)
    nodes, order = scene.export_flat()
    assert len(nodes) == 2 * count - 1
    if oracle.ref_available():
        tri = sd.triangles
        v = np.ascontiguousarray(tri["positions"][:, :, :3].reshape(-1, 9), np.float32)
        ids = np.ascontiguousarray(tri["metadata"][:, 2], np.uint32)
        rnodes = np.zeros((2 * count, 12), np.float32)
        prim = np.zeros(count, np.uint32)
        morton = np.zeros((count, 2), np.uint32)
        depth, status = C.c_uint32(0), C.c_int(0)
        cnt = oracle.ref_lib().ref_lbvh_build(v.ctypes.data, ids.ctypes.data, count, rnodes.ctypes.data,
                                              2 * count, prim.ctypes.data, morton.ctypes.data, C.byref(depth),
                                              C.byref(status))
        assert cnt == 2 * count - 1, status.value
        np.testing.assert_array_equal(nodes_as_words(nodes).view(np.uint32), rnodes[:cnt].view(np.uint32))
        np.testing.assert_array_equal(order, morton[:, 1])
        assert scene.info().max_depth == depth.value
    rays = scenes.to_ray_records(scenes.random_rays((0, 0, 0), (1, 1, 1), 20000, 6))
    sah = Scene(sd.triangles, 31, 1, N.BUILD_FLATTENED_SAH)
    a, b = sah.trace(rays), scene.trace(rays)
    np.testing.assert_array_equal(a["metadata"], b["metadata"])
    np.testing.assert_array_equal(a["position_t"].view(np.uint32), b["position_t"].view(np.uint32))
    np.testing.assert_array_equal(sah.trace(rays, any_hit=True)["metadata"][:, 1],
                                  scene.trace(rays, any_hit=True)["metadata"][:, 1])


@pytest.mark.parametrize("build", [N.BUILD_FLATTENED_SAH, N.BUILD_LBVH], ids=["sah", "lbvh"])
def test_one_triangle_scene_frame(native, oracle, build):
    """Every traversal loop over a hierarchy whose root is a leaf: the same
    film bit for bit, equal to the oracle."""
    sd = _one_triangle()
    w, h, depth = 48, 32, 6
    r = Renderer(w, h, depth)
    r.set_scene(Scene(sd.triangles, sd.fingerprint, 1, build), sd)
    fc = frame_constants(sd.camera, w, h, 1, depth, seed=0x77)
    outs = []
    for mode in (0, 1, 2, 3, 4):
        r.set_tuning(traversal=mode)
        r.render(fc, accumulate=False)
        tel = r.collect()
        assert tel.fatal_mask == 0 and tel.non_finite == 0
        outs.append(r.read(FILM_SAMPLE, w * h))
    for o in outs[1:]:
        np.testing.assert_array_equal(o.view(np.uint32), outs[0].view(np.uint32))
    ref, rays, shadows = _oracle_frame(oracle, sd, fc)
    assert _within(outs[0][:, :3], ref["sample"][:, :3]).all(axis=-1).mean() >= 0.999
    assert np.count_nonzero(outs[0][:, :3].sum(axis=1)) > w * h // 8  # the triangle is lit and in view


@pytest.mark.parametrize("w,h", [(1, 1), (7, 3), (1, 97), (129, 1)])
def test_one_pixel_and_ragged_frames_at_maximum_depth(native, oracle, w, h):
    """Frames of one pixel, one row or one column and sizes that fill no
    block, at the maximum path depth (16 bounces): every pixel equals the
    oracle; the per-bounce profile has 16 entries."""
    sd = scenes.cornell_box()
    depth = 16
    r = Renderer(w, h, depth)
    r.set_scene(Scene(sd.triangles, sd.fingerprint), sd)
    fc = frame_constants(sd.camera, w, h, 5, depth, seed=0xD00D, rr=[16.0, 0.05, 0.95, 1e-4])
    r.render(fc, accumulate=False)
    tel = r.collect()
    assert tel.fatal_mask == 0 and tel.non_finite == 0
    ref, rays, shadows = _oracle_frame(oracle, sd, fc)
    got = r.read(FILM_SAMPLE, w * h)
    assert _within(got[:, :3], ref["sample"][:, :3]).all(), (got[:, :3], ref["sample"][:, :3])
    assert tel.path_rays == rays and tel.shadow_rays == shadows
    prof = r.profile(fc)
    assert len(prof["rays"]) == depth and prof["rays"][0] == w * h
    with pytest.raises(N.NativeError):
        Renderer(w, h, depth + 1)


def test_view_at_capacity_end_and_maximum_view_count(native):
    """256 views of 2x2 pixels fill a 32x32 path capacity exactly, the last
    one ending at the capacity; each equals its view rendered alone.  An
    empty view list and 257 views are rejected."""
    sd = scenes.cornell_box()
    built = Scene(sd.triangles, sd.fingerprint)
    r = Renderer(32, 32, 4)
    r.bind_scene(0, built, sd)
    cap = r.capacity
    assert cap == 1024
    fcs = [frame_constants(sd.camera, 2, 2, 3, 4, seed=0x400 + k) for k in range(256)]
    views = [dict(frame=fcs[k], slot=0, offset=4 * k, key=k) for k in range(256)]
    assert views[-1]["offset"] + 4 == cap
    r.render_views(views)
    assert r.collect().fatal_mask == 0
    for k in (0, 1, 77, 254, 255):
        alone = Renderer(2, 2, 4)
        alone.set_scene(built, sd)
        alone.render(fcs[k], accumulate=False)
        alone.collect()
        np.testing.assert_array_equal(r.read_view(FILM_SAMPLE, 4 * k, 4).view(np.uint32),
                                      alone.read(FILM_SAMPLE, 4).view(np.uint32), err_msg=f"view {k}")
        np.testing.assert_array_equal(r.read_view(FILM_MEAN, 4 * k, 4).view(np.uint32),
                                      alone.read(FILM_MEAN, 4).view(np.uint32))
    with pytest.raises(N.NativeError) as e:
        r.render_views(views + [dict(frame=fcs[0], slot=0, offset=0, key=999)])
    assert e.value.code == N.INVALID_ARGUMENT
    with pytest.raises(N.NativeError) as e:
        r.render_views([])
    assert e.value.code == N.INVALID_ARGUMENT
    # One larger view placed flush against the end of the capacity.
    big = frame_constants(sd.camera, 16, 8, 2, 4, seed=0x99)
    r.render_views([dict(frame=big, slot=0, offset=cap - 128, key=5000)])
    assert r.collect().fatal_mask == 0
    alone = Renderer(16, 8, 4)
    alone.set_scene(built, sd)
    alone.render(big, accumulate=False)
    alone.collect()
    np.testing.assert_array_equal(r.read_view(FILM_SAMPLE, cap - 128, 128).view(np.uint32),
                                  alone.read(FILM_SAMPLE, 128).view(np.uint32))
