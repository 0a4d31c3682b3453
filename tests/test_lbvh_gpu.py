"""GPU LBVH build (Morton codes, radix sort, Karras hierarchy, refit) against
the reference's own SoftwareGpu::BuildKarrasLbvh, and hit parity with the
flattened SAH."""
import numpy as np
import pytest

from helpers import OracleScene, nodes_as_words
from renderingengine_b200 import _native as N
from renderingengine_b200 import scenes
from renderingengine_b200.traversal import Scene
from renderingengine_b200.wavefront import FILM_SAMPLE, Renderer, frame_constants

pytestmark = pytest.mark.gpu


def _ref_lbvh(oracle, tri):
    v = np.ascontiguousarray(tri["positions"][:, :, :3].reshape(-1, 9), np.float32)
    ids = np.ascontiguousarray(tri["metadata"][:, 2], np.uint32)
    n = len(tri)
    cap = 2 * n
    nodes = np.zeros((cap, 12), np.float32)
    prim_ids = np.zeros(n, np.uint32)
    morton = np.zeros((n, 2), np.uint32)
    import ctypes as C
    depth = C.c_uint32(0)
    status = C.c_int(0)
    cnt = oracle.ref_lib().ref_lbvh_build(v.ctypes.data, ids.ctypes.data, n, nodes.ctypes.data, cap,
                                          prim_ids.ctypes.data, morton.ctypes.data, C.byref(depth),
                                          C.byref(status))
    assert cnt > 0, status.value
    return nodes[:cnt], prim_ids, morton, depth.value


@pytest.mark.parametrize("make", [scenes.cornell_reference, lambda: scenes.triangle_soup(20000, seed=5),
                                  lambda: scenes.heightfield_scene(grid=64, spheres=64, seed=2)])
def test_gpu_lbvh_equals_reference_karras_build(native, oracle, make):
    """Node for node: same topology (pre-order numbering), bounds, parents,
    leaf order and depth as SoftwareGpu::BuildKarrasLbvh
    (src/rt/software_gpu/SoftwareGpu.cpp:1265-1345)."""
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    sd = make()
    scene = Scene(sd.triangles, sd.fingerprint, 1, N.BUILD_LBVH)
    nodes, order = scene.export_flat()
    rnodes, rprim_ids, rmorton, rdepth = _ref_lbvh(oracle, sd.triangles)
    assert len(nodes) == len(rnodes) == 2 * len(sd.triangles) - 1
    np.testing.assert_array_equal(nodes_as_words(nodes).view(np.uint32), rnodes.view(np.uint32))
    np.testing.assert_array_equal(order, rmorton[:, 1])
    np.testing.assert_array_equal(sd.triangles["metadata"][order, 2], rprim_ids)
    assert scene.info().max_depth == rdepth
    assert scene.info().gpu_build_ms > 0


@pytest.mark.parametrize("make,ray_maker", [
    (scenes.cornell_reference, lambda sd: scenes.pinhole_rays(sd.camera, 128, 96, seed=1)),
    (lambda: scenes.triangle_soup(50000, seed=9), lambda sd: scenes.random_rays((0, 0, 0), (1, 1, 1), 100000, 4)),
    (lambda: scenes.heightfield_scene(grid=128, spheres=256, seed=3),
     lambda sd: scenes.pinhole_rays(sd.camera, 320, 200, seed=2)),
])
def test_lbvh_hits_equal_sah_hits(native, make, ray_maker):
    sd = make()
    rays = scenes.to_ray_records(ray_maker(sd))
    a = Scene(sd.triangles, 5, 1, N.BUILD_FLATTENED_SAH).trace(rays)
    b = Scene(sd.triangles, 5, 1, N.BUILD_LBVH).trace(rays)
    np.testing.assert_array_equal(a["metadata"], b["metadata"])
    np.testing.assert_array_equal(a["ids"], b["ids"])
    np.testing.assert_array_equal(a["position_t"].view(np.uint32), b["position_t"].view(np.uint32))
    ao = Scene(sd.triangles, 5, 1, N.BUILD_FLATTENED_SAH).trace(rays, any_hit=True)
    bo = Scene(sd.triangles, 5, 1, N.BUILD_LBVH).trace(rays, any_hit=True)
    np.testing.assert_array_equal(ao["metadata"][:, 1], bo["metadata"][:, 1])


def test_lbvh_frame_equals_sah_frame(native):
    """The whole wavefront frame over the LBVH is bit-identical to the SAH
    frame (closest hits are identical, everything downstream is per path)."""
    sd = scenes.heightfield_scene(grid=64, spheres=128, seed=6)
    w, h, depth = 160, 120, 8
    films = []
    for kind in (N.BUILD_FLATTENED_SAH, N.BUILD_LBVH):
        scene = Scene(sd.triangles, 9, 1, kind)
        r = Renderer(w, h, depth)
        r.set_scene(scene, sd)
        r.render(frame_constants(sd.camera, w, h, 0, depth), accumulate=False)
        r.collect()
        films.append(r.read(FILM_SAMPLE, w * h))
    np.testing.assert_array_equal(films[0].view(np.uint32), films[1].view(np.uint32))


def test_full_size_lbvh_build(native, oracle):
    """2,424,832 triangles: the GPU LBVH builds, and a 200k-ray subset of the
    1080p camera rays hits exactly what the SAH hits."""
    sd = scenes.heightfield_scene()
    scene = Scene(sd.triangles, 17, 1, N.BUILD_LBVH)
    info = scene.info()
    assert info.node_count == 2 * len(sd.triangles) - 1
    rays = scenes.pinhole_rays(sd.camera, 1920, 1080, seed=11)
    sel = np.random.default_rng(0).choice(len(rays), 200_000, replace=False)
    rec = scenes.to_ray_records(rays[sel])
    a = scene.trace(rec)
    b = Scene(sd.triangles, 17, 1, N.BUILD_FLATTENED_SAH).trace(rec)
    np.testing.assert_array_equal(a["ids"], b["ids"])
    np.testing.assert_array_equal(a["position_t"][:, 3], b["position_t"][:, 3])
    print(f"LBVH GPU build {info.gpu_build_ms:.2f} ms (device), {info.build_ms:.1f} ms total")
