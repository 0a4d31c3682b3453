"""CPU tests: the product host SAH builder and the traversal oracle, pinned
against the reference's own CPU code (oracle/_ref) and its golden corpora.
No GPU needed."""
import json

import numpy as np
import pytest

from helpers import OracleScene, header_symbols, host_sah, nodes_as_words, software_rays, tri_vertices
from renderingengine_b200 import _native as N
from renderingengine_b200 import scenes


def test_library_exports_every_declared_symbol(native):
    declared = header_symbols()
    assert len(declared) >= 10
    for name in declared:
        assert hasattr(native, name), f"{name} declared in include/re_b200.h but not exported"
    assert set(declared) == set(N.declared_symbols()), "ctypes binding and header disagree"
    assert native.re_execution_architecture_token() == b"cuda-wavefront"
    assert native.re_abi_version() == (1 << 16)


def test_capability_rule(native):
    import ctypes as C
    why = C.c_char_p()
    assert native.re_capability_is_built(0, 1, 2, C.byref(why)) == 1
    assert native.re_capability_is_built(0, 4, 3, C.byref(why)) == 1
    assert native.re_capability_is_built(1, 1, 2, C.byref(why)) == 0 and b"PBR" in why.value
    assert native.re_capability_is_built(0, 2, 2, C.byref(why)) == 0


def _ref_sah(oracle, tri):
    ids = tri["metadata"][:, 2].copy()
    return oracle.ref_sah_build(tri_vertices(tri), ids)


@pytest.mark.parametrize("make", [scenes.cornell_reference, scenes.cornell_box,
                                  lambda: scenes.triangle_soup(20000, seed=5),
                                  lambda: scenes.heightfield_scene(grid=48, spheres=40, seed=2)])
def test_host_sah_matches_reference_build(native, oracle, make):
    """The product binned-SAH build equals Bvh<float>(BinnedSah) +
    FlattenCanonicalL3BinnedSah node for node (bounds, links, parents) and in
    leaf order and depth."""
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    sd = make()
    nodes, order, depth = host_sah(sd.triangles)
    rnodes, rorder, rdepth = _ref_sah(oracle, sd.triangles)
    assert len(nodes) == len(rnodes)
    np.testing.assert_array_equal(nodes_as_words(nodes).view(np.uint32)[:, [0, 1, 2, 4, 5, 6, 8, 9, 10, 11]],
                                  rnodes.view(np.uint32)[:, [0, 1, 2, 4, 5, 6, 8, 9, 10, 11]])
    np.testing.assert_array_equal(order, rorder)
    assert depth == rdepth


def test_host_sah_rejects_bad_input(native):
    sd = scenes.cornell_box()
    tri = sd.triangles.copy()
    tri["positions"][3, 1, 0] = np.nan
    with pytest.raises(N.NativeError) as e:
        host_sah(tri)
    assert e.value.code == N.INVALID_ARGUMENT and "non-finite" in str(e.value)
    with pytest.raises(N.NativeError):
        host_sah(sd.triangles, bins=1)


def _compare_oracle_with_reference(oracle, sd, rays, any_hit=False):
    os_ = OracleScene(sd)
    mine = oracle.trace(os_.nodes, os_.tri_v, os_.tri_key, rays, any_hit=any_hit)
    ref_hits, ref_cnt = oracle.ref_trace(nodes_as_words(os_.nodes), os_.tri_v, os_.traversal_id,
                                         software_rays(rays, 1 if any_hit else 0), any_hit=any_hit,
                                         stack_capacity=128)
    ref_prim = ref_hits[:, 4]
    mine_prim = np.where(mine["tri"] == 0xFFFFFFFF, 0xFFFFFFFF,
                         os_.traversal_id[np.minimum(mine["tri"], len(os_.traversal_id) - 1)])
    return os_, mine, ref_hits, ref_prim, mine_prim, ref_cnt


@pytest.mark.parametrize("make,ray_maker", [
    (scenes.cornell_reference, lambda sd: scenes.pinhole_rays(sd.camera, 96, 96, seed=1)),
    (lambda: scenes.triangle_soup(30000, seed=9), lambda sd: scenes.random_rays((0, 0, 0), (1, 1, 1), 40000, 4)),
    (lambda: scenes.heightfield_scene(grid=64, spheres=64, seed=3),
     lambda sd: scenes.pinhole_rays(sd.camera, 160, 120, seed=2)),
])
def test_oracle_trace_equals_softwaregpu_trace(native, oracle, make, ray_maker):
    """Closest hit of the traversal restatement equals SoftwareGpu::Trace
    (same primitive, bit-identical t/u/v: the triangle test is identical and
    the tie rule agrees because traversal IDs follow (instance, primitive))."""
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    sd = make()
    rays = ray_maker(sd)
    os_, mine, ref_hits, ref_prim, mine_prim, ref_cnt = _compare_oracle_with_reference(oracle, sd, rays)
    assert np.all(mine["status"] == 0)
    np.testing.assert_array_equal(mine_prim, ref_prim)
    hit = ref_prim != 0xFFFFFFFF
    assert hit.sum() > len(rays) * 0.05
    tbary = ref_hits[:, :3].view(np.float32)
    np.testing.assert_array_equal(mine["t"][hit], tbary[hit, 0])
    np.testing.assert_array_equal(mine["u"][hit], tbary[hit, 1])
    np.testing.assert_array_equal(mine["v"][hit], tbary[hit, 2])
    # Any-hit visibility agrees as a boolean.
    _, mine_a, ref_a, ref_prim_a, _, _ = _compare_oracle_with_reference(oracle, sd, rays, any_hit=True)
    np.testing.assert_array_equal(mine_a["tri"] != 0xFFFFFFFF, ref_prim_a != 0xFFFFFFFF)


def test_oracle_l3_parity_corpus(native, oracle):
    """The reference's statistical parity corpus (1,000,000 PCG rays over the
    18-triangle scene, TraversalParityTests.cpp:62-134): zero hit/miss and ID
    mismatches against the FP64 brute force, relative t error <= 1e-5."""
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    tris, ids, rays, bid, bt = oracle.ref_l3_parity_corpus(1_000_000)
    pos = tris.reshape(-1, 3, 3)
    tri = scenes.canonical_triangles(pos, None, np.zeros(18, np.uint32), ids, np.zeros(18, np.uint32))
    tri["metadata"][:, 2] = ids
    sd = scenes.SceneData("l3", tri, scenes.material(0), np.zeros(0, N.LIGHT_DTYPE),
                          np.zeros(0, scenes.FIXTURE_TRIANGLE_DTYPE), scenes.cornell_box().camera)
    os_ = OracleScene(sd)
    r = oracle.trace(os_.nodes, os_.tri_v, os_.tri_key, rays)
    prim = np.where(r["tri"] == 0xFFFFFFFF, 0xFFFFFFFF, os_.traversal_id[np.minimum(r["tri"], 17)])
    assert np.sum((prim == 0xFFFFFFFF) != (bid == 0xFFFFFFFF)) == 0
    hit = bid != 0xFFFFFFFF
    assert np.sum(prim[hit] != bid[hit]) == 0
    rel = np.abs(r["t"][hit].astype(np.float64) - bt[hit]) / np.maximum(1.0, np.abs(bt[hit]))
    assert rel.max() <= 1e-5


@pytest.mark.slow
def test_reference_cornell_reproduces_golden_fixture(oracle):
    """oracle/_ref's RenderCornellReference reproduces the golden JSON
    (rt/cpu/references/wave1/cornell-256x256-64spp-seed1.json): scene hash,
    ray and shadow-ray counts exactly."""
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    golden = json.loads((__import__("pathlib").Path(__file__).parent / "golden" /
                         "cornell_256x256_64spp_seed1.json").read_text())
    px, st = oracle.ref_cornell(256, 256, 64, 8, 1, 0)
    assert st["scene_hash"] == int(golden["scene_hash"], 16)
    assert st["rays"] == golden["ray_count"]
    assert st["shadow_rays"] == golden["shadow_ray_count"]
    assert st["non_finite"] == golden["non_finite_count"]
    assert np.isfinite(px).all()
