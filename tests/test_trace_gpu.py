"""GPU parity of the trace-batch kernels (RecordTraceClosestBatch /
RecordTraceAnyBatch) against the CPU oracle and the reference's own
SoftwareGpu::Trace, through the C ABI."""
import numpy as np
import pytest

from helpers import OracleScene, nodes_as_words, software_rays, tri_vertices
from renderingengine_b200 import _native as N
from renderingengine_b200 import scenes
from renderingengine_b200.traversal import (CudaTraversalBackend, GpuSceneBuildRequest, GpuTraceBatch, Scene)

pytestmark = pytest.mark.gpu

INVALID = 0xFFFFFFFF


def _gpu_and_oracle(oracle, sd, rays8, any_hit=False, build_kind=N.BUILD_FLATTENED_SAH):
    os_ = OracleScene(sd)
    scene = Scene(sd.triangles, sd.fingerprint, 1, build_kind)
    hits, counters = scene.trace(scenes.to_ray_records(rays8), any_hit=any_hit, counters=True)
    ref = oracle.trace(os_.nodes, os_.tri_v, os_.tri_key, rays8, any_hit=any_hit)
    scene.close()
    return os_, hits, counters, ref


def _oracle_ids(os_, ref):
    tri = ref["tri"]
    ok = tri != INVALID
    inst = np.full(len(tri), INVALID, np.uint32)
    prim = np.full(len(tri), INVALID, np.uint32)
    inst[ok] = os_.leaf_triangles["identity"][tri[ok], 0]
    prim[ok] = os_.leaf_triangles["identity"][tri[ok], 1]
    return ok, inst, prim


CASES = [
    ("cornell", scenes.cornell_reference, lambda sd: scenes.pinhole_rays(sd.camera, 128, 96, seed=1)),
    ("soup", lambda: scenes.triangle_soup(50000, seed=9),
     lambda sd: scenes.random_rays((0, 0, 0), (1, 1, 1), 100000, 4)),
    ("heightfield", lambda: scenes.heightfield_scene(grid=96, spheres=128, seed=3),
     lambda sd: scenes.pinhole_rays(sd.camera, 320, 200, seed=2)),
]


@pytest.mark.parametrize("name,make,ray_maker", CASES)
def test_closest_hit_bit_exact_against_oracle(native, oracle, name, make, ray_maker):
    sd = make()
    rays = ray_maker(sd)
    os_, hits, counters, ref = _gpu_and_oracle(oracle, sd, rays)
    ok, inst, prim = _oracle_ids(os_, ref)
    kind = hits["metadata"][:, 1]
    assert np.all(kind != N.HIT_KIND_INVALID)
    np.testing.assert_array_equal(kind == N.HIT_KIND_TRIANGLE, ok)
    np.testing.assert_array_equal(hits["ids"][:, 0], inst)
    np.testing.assert_array_equal(hits["ids"][:, 1], prim)
    # t, u, v are bit-identical (same operation sequence, no FMA contraction).
    np.testing.assert_array_equal(hits["position_t"][ok, 3], ref["t"][ok])
    np.testing.assert_array_equal(hits["geometric_normal_bary_u"][ok, 3], ref["u"][ok])
    np.testing.assert_array_equal(hits["shading_normal_bary_v"][ok, 3], ref["v"][ok])
    # Same visiting order, so the traversal counters agree exactly.
    assert counters["node_tests"] == ref["node_tests"]
    assert counters["triangle_tests"] == ref["tri_tests"]
    # Ray identity propagates; misses carry tMax.
    np.testing.assert_array_equal(hits["metadata"][:, 0], np.arange(len(rays), dtype=np.uint32))
    assert np.all(hits["position_t"][~ok, 3] == rays[~ok, 7])
    # Hit positions lie on the ray.
    p = rays[ok, :3] + rays[ok, 4:7] * ref["t"][ok, None]
    np.testing.assert_allclose(hits["position_t"][ok, :3], p, rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("name,make,ray_maker", CASES)
def test_any_hit_visibility_against_oracle(native, oracle, name, make, ray_maker):
    sd = make()
    rays = ray_maker(sd)
    rays[:, 7] = np.where(np.arange(len(rays)) % 2 == 0, 1e30, 0.5)  # finite and infinite shadow rays
    os_, hits, _, ref = _gpu_and_oracle(oracle, sd, rays, any_hit=True)
    np.testing.assert_array_equal(hits["metadata"][:, 1] == N.HIT_KIND_TRIANGLE, ref["tri"] != INVALID)


def test_against_reference_softwaregpu_trace(native, oracle):
    """Closest-hit primitive IDs equal the reference's SoftwareGpu::Trace."""
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    sd = scenes.heightfield_scene(grid=64, spheres=64, seed=5)
    rays = scenes.pinhole_rays(sd.camera, 200, 150, seed=3)
    os_ = OracleScene(sd)
    ref_hits, _ = oracle.ref_trace(nodes_as_words(os_.nodes), os_.tri_v, os_.traversal_id, software_rays(rays),
                                   stack_capacity=128, threads=8)
    scene = Scene(sd.triangles, sd.fingerprint)
    hits = scene.trace(scenes.to_ray_records(rays))
    ok = hits["metadata"][:, 1] == N.HIT_KIND_TRIANGLE
    traversal = np.full(len(rays), INVALID, np.uint32)
    lookup = dict(zip(map(tuple, sd.triangles["identity"][:, :2].tolist()), sd.triangles["metadata"][:, 2]))
    traversal[ok] = [lookup[(int(a), int(b))] for a, b in hits["ids"][ok, :2]]
    np.testing.assert_array_equal(traversal, ref_hits[:, 4])
    np.testing.assert_array_equal(hits["position_t"][ok, 3], ref_hits[ok, 0].view(np.float32))


def test_l3_statistical_parity_corpus(native, oracle):
    """1,000,000 seeded rays of TraversalParityTests.cpp:62-134 on the GPU: no
    hit/miss or ID mismatch against the FP64 brute force, relative t <= 1e-5."""
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    tris, ids, rays, bid, bt = oracle.ref_l3_parity_corpus(1_000_000)
    tri = scenes.canonical_triangles(tris.reshape(-1, 3, 3), None, np.zeros(18, np.uint32), ids,
                                     np.zeros(18, np.uint32))
    scene = Scene(tri, 0x4C33)
    hits = scene.trace(scenes.to_ray_records(rays))
    hit = hits["metadata"][:, 1] == N.HIT_KIND_TRIANGLE
    assert np.sum(hit != (bid != INVALID)) == 0
    assert np.sum(hits["ids"][hit, 1] != bid[hit]) == 0
    t = hits["position_t"][hit, 3].astype(np.float64)
    assert (np.abs(t - bt[hit]) / np.maximum(1.0, np.abs(bt[hit]))).max() <= 1e-5


def test_caller_flattened_nodes_give_same_hits(native, oracle):
    """A caller that already ran FlattenCanonicalL3BinnedSah can hand its 48 B
    nodes and leaf-ordered triangles over; hits equal the internal build."""
    sd = scenes.cornell_box()
    os_ = OracleScene(sd)
    rays = scenes.to_ray_records(scenes.pinhole_rays(sd.camera, 64, 64, seed=4))
    a = Scene(sd.triangles, 7).trace(rays)
    b = Scene(os_.leaf_triangles, 7, nodes=os_.nodes).trace(rays)
    np.testing.assert_array_equal(a["ids"], b["ids"])
    np.testing.assert_array_equal(a["position_t"], b["position_t"])


def test_backend_status_contract(native):
    """IGpuTraversalBackend semantics: MissingScene without a scene or on a
    fingerprint/generation mismatch, InvalidArgument on bad input, invalid rays
    become HitKindInvalid."""
    be = CudaTraversalBackend()
    sd = scenes.cornell_box()
    rays = scenes.to_ray_records(scenes.pinhole_rays(sd.camera, 16, 16))
    hits = np.zeros(len(rays), N.HIT_DTYPE)
    st = be.RecordTraceClosestBatch(GpuTraceBatch(rays, hits, 11, 0, 0, len(rays), 1))
    assert not st and st.code == N.MISSING_SCENE
    assert not be.BuildOrUpdateScene(GpuSceneBuildRequest(sd.triangles, 0, 1))
    assert be.BuildOrUpdateScene(GpuSceneBuildRequest(sd.triangles, 11, 1))
    st = be.RecordTraceClosestBatch(GpuTraceBatch(rays, hits, 11, 0, 0, len(rays), 2))
    assert st.code == N.MISSING_SCENE
    bad = rays.copy()
    bad["direction_tmax"][5, :3] = [0.0, 0.0, 2.0]   # not unit length
    bad["origin_tmin"][6, 0] = np.nan
    bad["origin_tmin"][7, 3] = 5.0                   # tMin >= tMax
    bad["direction_tmax"][7, 3] = 1.0
    st = be.RecordTraceClosestBatch(GpuTraceBatch(bad, hits, 11, 0, 0, len(rays), 1))
    assert st, st.message
    assert list(hits["metadata"][5:8, 1]) == [N.HIT_KIND_INVALID] * 3
    # Offsets are record indices.
    hits2 = np.zeros(len(rays) + 5, N.HIT_DTYPE)
    assert be.RecordTraceAnyBatch(GpuTraceBatch(rays, hits2, 11, 10, 5, 20, 1))
    assert np.all(hits2["metadata"][5:25, 0] == np.arange(10, 30))
    broken = sd.triangles.copy()
    broken["positions"][0, 0, 0] = np.inf
    st = be.BuildOrUpdateScene(GpuSceneBuildRequest(broken, 12, 1))
    assert st.code == N.INVALID_ARGUMENT


def test_device_memory_batch(native, oracle):
    """Device-resident ray/hit buffers (torch allocations) on a stream."""
    import torch
    sd = scenes.heightfield_scene(grid=32, spheres=16, seed=1)
    rays = scenes.to_ray_records(scenes.pinhole_rays(sd.camera, 64, 48, seed=7))
    scene = Scene(sd.triangles, 99)
    host = scene.trace(rays)
    d_rays = torch.from_numpy(rays.view(np.uint8).copy()).cuda()
    d_hits = torch.zeros(len(rays) * N.HIT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        scene.trace_device(d_rays.data_ptr(), d_hits.data_ptr(), len(rays), stream=stream.cuda_stream)
    stream.synchronize()
    dev = d_hits.cpu().numpy().view(N.HIT_DTYPE)
    np.testing.assert_array_equal(dev.view(np.uint32), host.view(np.uint32))


def test_chunked_host_batches_equal_one_launch(native):
    """A host-memory batch of more than one chunk (pipelined uploads,
    traversals and downloads, ragged last chunk, at record offsets, pinned
    and pageable) equals the same rays traced from device memory in one
    launch, closest and any hit."""
    import torch
    sd = scenes.heightfield_scene(grid=48, spheres=64, seed=2)
    rays = scenes.to_ray_records(scenes.random_rays((0, 0, 0), (1, 0.3, 1), 700_001, 13))
    scene = Scene(sd.triangles, 98)
    d_rays = torch.from_numpy(rays.view(np.uint8).copy()).cuda()
    for any_hit in (False, True):
        d_hits = torch.zeros(len(rays) * N.HIT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
        scene.trace_device(d_rays.data_ptr(), d_hits.data_ptr(), len(rays), any_hit=any_hit)
        torch.cuda.synchronize()
        want = d_hits.cpu().numpy().view(N.HIT_DTYPE)
        np.testing.assert_array_equal(scene.trace(rays, any_hit=any_hit).view(np.uint32), want.view(np.uint32))
        pinned_rays = torch.from_numpy(rays.view(np.uint8).copy()).pin_memory().numpy().view(N.RAY_DTYPE)
        hits = torch.zeros((len(rays) + 3) * N.HIT_DTYPE.itemsize, dtype=torch.uint8).pin_memory().numpy()
        hits = hits.view(N.HIT_DTYPE)
        be = CudaTraversalBackend()
        assert be.BuildOrUpdateScene(GpuSceneBuildRequest(sd.triangles, 98, 1))
        fn = be.RecordTraceAnyBatch if any_hit else be.RecordTraceClosestBatch
        st = fn(GpuTraceBatch(pinned_rays, hits, 98, 1, 3, len(rays) - 1, 1))
        assert st, st.message
        np.testing.assert_array_equal(hits[3:3 + len(rays) - 1].view(np.uint32), want[1:].view(np.uint32))


def test_full_size_heightfield_subset(native, oracle):
    """The 2,424,832-triangle heightfield + icosphere scene: a 200k-ray seeded
    subset of the 1080p camera rays matches the oracle bit-exactly."""
    sd = scenes.heightfield_scene()
    assert len(sd.triangles) == 2_424_832
    rays = scenes.pinhole_rays(sd.camera, 1920, 1080, seed=11)
    sel = np.random.default_rng(0).choice(len(rays), 200_000, replace=False)
    os_, hits, _, ref = _gpu_and_oracle(oracle, sd, rays[sel])
    ok, inst, prim = _oracle_ids(os_, ref)
    np.testing.assert_array_equal(hits["ids"][:, 0], inst)
    np.testing.assert_array_equal(hits["ids"][:, 1], prim)
    np.testing.assert_array_equal(hits["position_t"][ok, 3], ref["t"][ok])
