"""re_lbvh_build_static, the allocation-free GPU LBVH build, against the
allocating build of re_scene_create(RE_BUILD_LBVH) + re_scene_export_flat:
same leaf order and, after renumbering the Karras nodes in pre-order, the
same flattened records word for word, on two calls in a row.  This file is
collected last so the static scratch is exercised after every other test
has used the device."""
import ctypes as C

import numpy as np
import pytest

from helpers import nodes_as_words
from renderingengine_b200 import _native as N
from renderingengine_b200 import scenes
from renderingengine_b200.traversal import Scene


def test_rejects_counts_beyond_the_static_capacity(native):
    """Checked before anything touches the device (runs without a GPU)."""
    lib = N.load()
    buf = np.zeros(64, np.float32)
    too_many = N.LBVH_STATIC_MAX_TRIANGLES + 1
    rc = lib.re_lbvh_build_static(buf.ctypes.data, buf.ctypes.data, too_many, buf.ctypes.data, buf.ctypes.data, None)
    assert rc == N.INVALID_ARGUMENT
    assert b"static scratch capacity" in lib.re_last_error()
    assert lib.re_lbvh_build_static(buf.ctypes.data, buf.ctypes.data, 0, buf.ctypes.data, buf.ctypes.data,
                                    None) == N.INVALID_ARGUMENT


def _preorder(nodes: np.ndarray, order: np.ndarray, positions: np.ndarray) -> np.ndarray:
    """Karras nodes -> the reference's pre-order flat records (the numbering
    re_scene_export_flat emits)."""
    n = len(order)
    out = np.zeros(2 * n - 1, N.NODE_DTYPE)
    leaf_pos = positions[order]  # (n, 3, 3) in sorted order
    count = 0
    stack = [(0 if n > 1 else N.LBVH_CHILD_LEAF, 0xFFFFFFFF, True)]
    while stack:
        code, parent, is_left = stack.pop()
        idx = count
        count += 1
        if parent != 0xFFFFFFFF:
            out["links"][parent, 0 if is_left else 2] = idx
        if code & N.LBVH_CHILD_LEAF:
            k = code & ~N.LBVH_CHILD_LEAF
            out["bounds_min"][idx, :3] = leaf_pos[k].min(axis=0)
            out["bounds_max"][idx, :3] = leaf_pos[k].max(axis=0)
            out["links"][idx] = (k, 1, 0xFFFFFFFF, parent)
        else:
            out["bounds_min"][idx, :3] = nodes["bounds_min"][code]
            out["bounds_max"][idx, :3] = nodes["bounds_max"][code]
            out["links"][idx] = (0xFFFFFFFF, 0, 0xFFFFFFFF, parent)
            stack.append((int(nodes["right"][code]), idx, False))
            stack.append((int(nodes["left"][code]), idx, True))
    assert count == 2 * n - 1
    return out


def _static_build(tri: np.ndarray):
    import torch

    lib = N.load()
    n = len(tri)
    pos = torch.from_numpy(np.ascontiguousarray(tri["positions"][:, :, :4], np.float32)).cuda()
    ids = torch.from_numpy(np.ascontiguousarray(tri["metadata"][:, 2], np.uint32).view(np.int32)).cuda()
    order = torch.zeros(n, dtype=torch.int32, device="cuda")
    nodes = torch.zeros((max(n - 1, 1), 8), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    N.check(lib.re_lbvh_build_static(pos.data_ptr(), ids.data_ptr(), n, order.data_ptr(), nodes.data_ptr(), None))
    torch.cuda.synchronize()
    o = order.cpu().numpy().view(np.uint32).copy()
    nd = nodes.cpu().numpy().copy().view(N.LBVH_NODE_DTYPE).reshape(-1)[: n - 1]
    return o, nd


CASES = [
    ("cornell", scenes.cornell_reference),
    ("soup-20k", lambda: scenes.triangle_soup(20000, seed=5)),
    ("heightfield", lambda: scenes.heightfield_scene(grid=64, spheres=64, seed=2)),
    ("soup-max", lambda: scenes.triangle_soup(N.LBVH_STATIC_MAX_TRIANGLES, seed=8)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,make", CASES)
def test_static_build_equals_allocating_build_twice(native, name, make):
    sd = make()
    tri = sd.triangles
    want_nodes, want_order = Scene(tri, sd.fingerprint, 1, N.BUILD_LBVH).export_flat()
    positions = np.ascontiguousarray(tri["positions"][:, :, :3], np.float32)
    for call in range(2):
        order, nodes = _static_build(tri)
        np.testing.assert_array_equal(order, want_order, err_msg=f"{name} call {call}: leaf order")
        flat = _preorder(nodes, order, positions)
        np.testing.assert_array_equal(nodes_as_words(flat).view(np.uint32), nodes_as_words(want_nodes).view(np.uint32),
                                      err_msg=f"{name} call {call}: flattened records")


@pytest.mark.gpu
def test_steady_state_call_allocates_nothing(native):
    """After the first call (which loads the module and resolves the scratch
    address), further calls leave the device's free memory unchanged."""
    import torch

    lib = N.load()
    sd = scenes.triangle_soup(30000, seed=2)
    tri = sd.triangles
    n = len(tri)
    pos = torch.from_numpy(np.ascontiguousarray(tri["positions"][:, :, :4], np.float32)).cuda()
    ids = torch.from_numpy(np.ascontiguousarray(tri["metadata"][:, 2], np.uint32).view(np.int32)).cuda()
    order = torch.zeros(n, dtype=torch.int32, device="cuda")
    nodes = torch.zeros((n - 1, 8), dtype=torch.float32, device="cuda")
    N.check(lib.re_lbvh_build_static(pos.data_ptr(), ids.data_ptr(), n, order.data_ptr(), nodes.data_ptr(), None))
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        N.check(lib.re_lbvh_build_static(pos.data_ptr(), ids.data_ptr(), n, order.data_ptr(), nodes.data_ptr(),
                                         None))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
