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


@pytest.mark.gpu
def test_single_triangle_writes_only_the_order(native):
    """count == 1 launches no hierarchy kernel: order_out == [0] and a NULL
    nodes_out is accepted."""
    import torch

    lib = N.load()
    tri = scenes.triangle_soup(1, seed=4).triangles
    pos = torch.from_numpy(np.ascontiguousarray(tri["positions"][:, :, :4], np.float32)).cuda()
    ids = torch.tensor([7], dtype=torch.int32, device="cuda")
    order = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    for _ in range(2):
        N.check(lib.re_lbvh_build_static(pos.data_ptr(), ids.data_ptr(), 1, order.data_ptr(), None, None))
        torch.cuda.synchronize()
        assert order.cpu().tolist() == [0]


@pytest.mark.gpu
def test_build_on_a_caller_stream(native):
    """Launched on a non-default stream: the result is complete once that
    stream has synchronised, and equals the build on the default stream."""
    import torch

    lib = N.load()
    sd = scenes.triangle_soup(12000, seed=11)
    tri = sd.triangles
    want_order, want_nodes = _static_build(tri)
    n = len(tri)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        pos = torch.from_numpy(np.ascontiguousarray(tri["positions"][:, :, :4], np.float32)).cuda()
        ids = torch.from_numpy(np.ascontiguousarray(tri["metadata"][:, 2], np.uint32).view(np.int32)).cuda()
        order = torch.zeros(n, dtype=torch.int32, device="cuda")
        nodes = torch.zeros((n - 1, 8), dtype=torch.float32, device="cuda")
    s.synchronize()
    N.check(lib.re_lbvh_build_static(pos.data_ptr(), ids.data_ptr(), n, order.data_ptr(), nodes.data_ptr(),
                                     C.c_void_p(s.cuda_stream)))
    s.synchronize()
    np.testing.assert_array_equal(order.cpu().numpy().view(np.uint32), want_order)
    got = nodes.cpu().numpy().view(N.LBVH_NODE_DTYPE).reshape(-1)
    np.testing.assert_array_equal(got.view(np.uint32), want_nodes.view(np.uint32))


def _karras_index_tiebreak(keys: np.ndarray):
    """Karras 2012 hierarchy over sorted 64-bit keys, equal keys split by
    sorted position (section 4): (left, right, first, last) per internal node,
    child codes with bit 31 marking a leaf."""
    n = len(keys)
    k = [int(x) for x in keys]

    def delta(i, j):
        if j < 0 or j >= n:
            return -1
        x = k[i] ^ k[j]
        return 64 + 32 - (i ^ j).bit_length() if x == 0 else 64 - x.bit_length()

    out = []
    for i in range(n - 1):
        d = 1 if delta(i, i + 1) - delta(i, i - 1) >= 0 else -1
        dmin = delta(i, i - d)
        lmax = 2
        while delta(i, i + lmax * d) > dmin:
            lmax <<= 1
        l, t = 0, lmax >> 1
        while t >= 1:
            if delta(i, i + (l + t) * d) > dmin:
                l += t
            t >>= 1
        j = i + l * d
        dnode = delta(i, j)
        s, t = 0, l
        while True:
            t = (t + 1) >> 1
            if delta(i, i + (s + t) * d) > dnode:
                s += t
            if t <= 1:
                break
        gamma = i + s * d + min(d, 0)
        first, last = min(i, j), max(i, j)
        lc = (N.LBVH_CHILD_LEAF | gamma) if first == gamma else gamma
        rc = (N.LBVH_CHILD_LEAF | (gamma + 1)) if last == gamma + 1 else gamma + 1
        out.append((lc, rc, first, last))
    return out


@pytest.mark.gpu
def test_duplicate_ids_and_codes_give_a_well_formed_hierarchy(native, oracle):
    """Triangles whose Morton codes and stable IDs are both equal (exact
    copies given the same ID) are split by sorted position: the same
    hierarchy as a restatement of Karras's index tie-break over the
    reference's Morton codes, every node with one parent, every internal box
    the exact bounds of its leaf range -- on two calls in a row."""
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    base = scenes.triangle_soup(3000, seed=21).triangles
    rng = np.random.default_rng(5)
    dup_src = rng.choice(len(base), 600, replace=False)
    tri = np.concatenate([base, base[dup_src]])
    ids = np.concatenate([np.arange(len(base), dtype=np.uint32), dup_src.astype(np.uint32)])
    # A further 200 triangles share an ID with another, different triangle.
    ids[rng.choice(len(base), 200, replace=False)] = rng.choice(len(base), 200).astype(np.uint32)
    tri["metadata"][:, 2] = ids
    n = len(tri)
    # Morton codes per triangle from the reference's own LBVH (unique IDs).
    v = np.ascontiguousarray(tri["positions"][:, :, :3].reshape(-1, 9), np.float32)
    nodes12 = np.zeros((2 * n, 12), np.float32)
    morton = np.zeros((n, 2), np.uint32)
    depth, status = C.c_uint32(0), C.c_int(0)
    uniq = np.arange(n, dtype=np.uint32)
    assert oracle.ref_lib().ref_lbvh_build(v.ctypes.data, uniq.ctypes.data, n, nodes12.ctypes.data, 2 * n,
                                           np.zeros(n, np.uint32).ctypes.data, morton.ctypes.data,
                                           C.byref(depth), C.byref(status)) > 0
    codes = np.zeros(n, np.uint64)
    codes[morton[:, 1]] = morton[:, 0]
    keys = (codes << np.uint64(32)) | ids.astype(np.uint64)
    want_order = np.argsort(keys, kind="stable").astype(np.uint32)
    sorted_keys = keys[want_order]
    assert len(np.unique(sorted_keys)) < n - 400  # the copies really collide
    want = _karras_index_tiebreak(sorted_keys)
    pos_sorted = np.ascontiguousarray(tri["positions"][:, :, :3], np.float32)[want_order]
    for call in range(2):
        order, nodes = _static_build(tri)
        np.testing.assert_array_equal(order, want_order, err_msg=f"call {call}: leaf order")
        np.testing.assert_array_equal(nodes["left"], [w[0] for w in want], err_msg=f"call {call}: left children")
        np.testing.assert_array_equal(nodes["right"], [w[1] for w in want], err_msg=f"call {call}: right children")
        parents = np.zeros(n - 1, np.int64)
        for lc, rc, _, _ in want:
            for c in (lc, rc):
                if not c & N.LBVH_CHILD_LEAF:
                    parents[c] += 1
        assert parents[0] == 0 and (parents[1:] == 1).all()
        for i, (_, _, first, last) in enumerate(want):
            span = pos_sorted[first:last + 1].reshape(-1, 3)
            np.testing.assert_array_equal(nodes["bounds_min"][i], span.min(axis=0), err_msg=f"node {i} lo")
            np.testing.assert_array_equal(nodes["bounds_max"][i], span.max(axis=0), err_msg=f"node {i} hi")
