"""Scene ingestion (re_scene_expand_canonical) on the CPU: the reference's
own BuildCanonicalTraversalScene (oracle/_ref) on an instanced scene, and
the entry point's host-side validation, which rejects a scene with the
reference's messages before any device work."""
import ctypes as C

import numpy as np
import pytest

from renderingengine_b200 import _native as N
from renderingengine_b200 import ingest


def ref_expand(oracle, scene):
    v, ix, g, inst, m = [np.ascontiguousarray(a) for a in scene]
    cap = ingest.expansion_count(g, inst) + 16
    out = np.zeros(cap, N.TRIANGLE_DTYPE)
    err = C.create_string_buffer(256)
    n = oracle.ref_lib().ref_canonical_expand(v.ctypes.data, len(v), ix.ctypes.data, len(ix), g.ctypes.data, len(g),
                                              inst.ctypes.data, len(inst), m.ctypes.data, len(m), out.ctypes.data,
                                              cap, err, 256)
    return (out[:n], "") if n >= 0 else (None, err.value.decode())


def small_scene():
    return ingest.instanced_heightfield(grid=8, spheres=12, subdivisions=1, seed=3, per_instance=2)


def test_reference_expansion_of_an_instanced_scene(native, oracle):
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    scene = small_scene()
    tris, err = ref_expand(oracle, scene)
    assert err == ""
    assert len(tris) == 8 * 8 * 2 + 12 * 80
    assert np.array_equal(tris["metadata"][:, 2], np.arange(len(tris)))  # traversal IDs in output order
    assert np.all(tris["positions"][:, :, 3] == 1.0) and np.all(tris["normals"][:, :, 3] == 0.0)


def _expect_error(scene, message, oracle=None):
    with pytest.raises(N.NativeError) as e:
        ingest.expand_canonical(*scene)
    assert e.value.code == N.INVALID_ARGUMENT and message in str(e.value)
    if oracle is not None and oracle.ref_available():
        _, ref_err = ref_expand(oracle, scene)
        assert ref_err == message


def test_host_validation_matches_the_reference(native, oracle):
    v, ix, g, inst, m = small_scene()
    hidden = inst.copy()
    hidden["metadata"][:, 3] = 0
    _expect_error((v, ix, g, hidden, m), "Canonical traversal expansion produced no visible triangles.", oracle)
    bad_range = inst.copy()
    bad_range["metadata"][3, 1] = 5
    _expect_error((v, ix, g, bad_range, m), "Canonical instance geometry range is invalid during traversal expansion.",
                  oracle)
    bad_mat = g.copy()
    bad_mat["identity"][1, 2] = 9
    _expect_error((v, ix, bad_mat, inst, m), "Canonical traversal geometry references an invalid material.", oracle)
    bad_idx = g.copy()
    bad_idx["index_range"][1, 1] += 6
    _expect_error((v, ix, bad_idx, inst, m), "Canonical traversal triangle index range is invalid.", oracle)
    _expect_error((v[:0], ix, g, inst, m), "requires a validated, identified scene view", None)
