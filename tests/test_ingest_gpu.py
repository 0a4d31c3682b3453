"""Scene ingestion on the GPU (re_scene_expand_canonical) against the
reference's own BuildCanonicalTraversalScene (oracle/_ref): every record of
the expansion bit for bit -- world positions, renormalised normals,
texcoords, identity and metadata -- into host and into device memory, on a
small scene with an invisible instance, a mirrored instance and a
zero-length normal, and at the benchmark scene's full size (2,424,832
triangles); device-side errors carry the reference's messages."""
import numpy as np
import pytest
import torch

from renderingengine_b200 import _native as N
from renderingengine_b200 import ingest
from test_ingest import ref_expand, small_scene

pytestmark = pytest.mark.gpu


def _edge_scene():
    v, ix, g, inst, m = small_scene()
    inst = inst.copy()
    v = v.copy()
    inst["metadata"][2, 3] = 0                      # invisible
    inst["object_to_world"][3, 0] *= -1.0          # mirrored (negative determinant)
    inst["world_to_object"][3, :, 0] *= -1.0
    v["normal"][5] = 0.0                            # zero-length normal -> zero after the transform
    return v, ix, g, inst, m


@pytest.mark.parametrize("make", [small_scene, _edge_scene], ids=["small", "edges"])
def test_expansion_equals_reference(native, oracle, make):
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    scene = make()
    want, err = ref_expand(oracle, scene)
    assert err == ""
    got = ingest.expand_canonical(*scene)
    assert len(got) == len(want)
    np.testing.assert_array_equal(got.view(np.uint8), want.view(np.uint8))
    dev = torch.zeros(len(want) * N.TRIANGLE_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    n = ingest.expand_canonical(*scene, out_ptr=dev.data_ptr(), out_capacity=len(want))
    torch.cuda.synchronize()
    assert n == len(want)
    np.testing.assert_array_equal(dev.cpu().numpy(), want.view(np.uint8).reshape(-1))


def test_device_errors_match_the_reference(native, oracle):
    v, ix, g, inst, m = small_scene()
    bad_vertex = g.copy()
    bad_vertex["index_range"][1, 2] = len(v)  # vertex offset past the array
    bad_nan = inst.copy()
    bad_nan["object_to_world"][4, 0, 0] = np.nan
    for scene, message in [((v, ix, bad_vertex, inst, m), "Canonical traversal triangle references an invalid vertex."),
                           ((v, ix, g, bad_nan, m), "Canonical traversal transform produced non-finite geometry.")]:
        with pytest.raises(N.NativeError) as e:
            ingest.expand_canonical(*scene)
        assert e.value.code == N.INVALID_ARGUMENT and message in str(e.value)
        if oracle.ref_available():
            assert ref_expand(oracle, scene)[1] == message


def _split(scene):
    """The full scene as two scenes the reference can expand: the heightfield
    instance alone, and the sphere instances over the sphere mesh alone
    (BuildCanonicalTraversalScene reserves index count / 3 x instance count
    records up front, too many for the combined scene)."""
    v, ix, g, inst, m = scene
    nh = int(g["index_range"][0, 1])
    a = (v, ix[:nh], g[:1], inst[:1], m)
    gb = g[1:].copy()
    gb["index_range"][:, 0] -= nh
    ib = inst[1:].copy()
    ib["metadata"][:, 0] -= 1
    b = (v, ix[nh:], gb, ib, m)
    return a, b


def test_full_size_expansion_equals_reference(native, oracle):
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    scene = ingest.instanced_heightfield()
    got = ingest.expand_canonical(*scene)
    assert len(got) == 2_424_832
    a, b = _split(scene)
    want_a, err_a = ref_expand(oracle, a)
    want_b, err_b = ref_expand(oracle, b)
    assert err_a == "" and err_b == ""
    want_b["metadata"][:, 2] += len(want_a)  # traversal IDs continue after the heightfield
    want = np.concatenate([want_a, want_b])
    np.testing.assert_array_equal(got.view(np.uint8), want.view(np.uint8))


def test_scene_from_device_records_equals_scene_from_host(native):
    """Expansion into HBM, then the scene built from the device records: the
    same hierarchy (node for node) and the same hits as the scene built from
    a host copy of the same records; device-side primitive checks reject a
    degenerate triangle and duplicate traversal IDs."""
    from renderingengine_b200 import scenes
    from renderingengine_b200.traversal import Scene
    scene = ingest.instanced_heightfield(grid=64, spheres=256, seed=5)
    host = ingest.expand_canonical(*scene)
    n = len(host)
    dev = torch.zeros(n * N.TRIANGLE_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    assert ingest.expand_canonical(*scene, out_ptr=dev.data_ptr(), out_capacity=n) == n
    torch.cuda.synchronize()
    a = Scene(host, 91, 1, N.BUILD_LBVH)
    b = Scene.from_device(dev.data_ptr(), n, 91)
    na, oa = a.export_flat()
    nb, ob = b.export_flat()
    np.testing.assert_array_equal(na.view(np.uint8), nb.view(np.uint8))
    np.testing.assert_array_equal(oa, ob)
    rays = scenes.to_ray_records(scenes.random_rays((0, 0, 0), (1, 0.3, 1), 50000, 7))
    ha, hb = a.trace(rays), b.trace(rays)
    np.testing.assert_array_equal(ha.view(np.uint8), hb.view(np.uint8))
    np.testing.assert_array_equal(a.trace(rays, any_hit=True)["metadata"], b.trace(rays, any_hit=True)["metadata"])
    bad = host.copy()
    bad["positions"][3, 2] = bad["positions"][3, 0]  # degenerate
    dbad = torch.from_numpy(bad.view(np.uint8).copy()).cuda()
    with pytest.raises(N.NativeError, match="degenerate"):
        Scene.from_device(dbad.data_ptr(), n, 92)
    dup = host.copy()
    dup["metadata"][7, 2] = dup["metadata"][8, 2]
    ddup = torch.from_numpy(dup.view(np.uint8).copy()).cuda()
    with pytest.raises(N.NativeError, match="unique"):
        Scene.from_device(ddup.data_ptr(), n, 93)
