"""Shared test helpers: scene flattening and oracle inputs."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np

from renderingengine_b200 import _native as N

ROOT = Path(__file__).resolve().parents[1]


def header_symbols() -> list[str]:
    text = (ROOT / "include" / "re_b200.h").read_text()
    return re.findall(r"RE_API\s+[\w\s\*]+?\b(re_\w+)\s*\(", text)


def host_sah(triangles: np.ndarray, bins: int = 16, leaf: int = 4):
    """Product host SAH build (no GPU): (nodes NODE_DTYPE, leaf_order, depth)."""
    lib = N.load()
    tri = np.ascontiguousarray(triangles, N.TRIANGLE_DTYPE)
    n = len(tri)
    nodes = np.zeros(max(1, 2 * n - 1), N.NODE_DTYPE)
    order = np.zeros(n, np.uint32)
    count = C.c_uint32(0)
    depth = C.c_uint32(0)
    N.check(lib.re_sah_build_host(N.ptr(tri), n, bins, leaf, N.ptr(nodes), len(nodes), C.byref(count),
                                  N.ptr(order), C.byref(depth)))
    return nodes[:count.value].copy(), order, depth.value


def tri_vertices(triangles: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(triangles["positions"][:, :, :3].reshape(-1, 9), np.float32)


def tri_keys(triangles: np.ndarray) -> np.ndarray:
    """(n, 4) uint32 oracle keys: instance, primitive, traversal ID, flags
    (bit0 double-sided, bit1 casts shadow)."""
    k = np.zeros((len(triangles), 4), np.uint32)
    k[:, 0] = triangles["identity"][:, 0]
    k[:, 1] = triangles["identity"][:, 1]
    k[:, 2] = triangles["metadata"][:, 2]
    ds = ((triangles["metadata"][:, 0] & N.GEOMETRY_FLAG_DOUBLE_SIDED) != 0) | \
         ((triangles["metadata"][:, 1] & N.MATERIAL_FLAG_DOUBLE_SIDED) != 0)
    cs = (triangles["metadata"][:, 3] & N.INSTANCE_FLAG_CASTS_SHADOW) != 0
    k[:, 3] = ds.astype(np.uint32) | (cs.astype(np.uint32) << 1)
    return k


def nodes_as_words(nodes: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(nodes).view(np.float32).reshape(-1, 12)


def software_rays(rays8: np.ndarray, mode: int = 0) -> np.ndarray:
    """SoftwareRayRecord words (m, 12) for SoftwareGpu::Trace."""
    m = rays8.shape[0]
    r = np.zeros((m, 12), np.float32)
    r[:, :8] = rays8
    q = r[:, 8:].view(np.uint32)
    q[:, 0] = np.arange(m, dtype=np.uint32)
    q[:, 1] = mode
    q[:, 2] = 0xFFFFFFFF
    return r


class OracleScene:
    """A scene flattened by the product host builder with oracle inputs in leaf order."""

    def __init__(self, scene_data, bins: int = 16, leaf: int = 4):
        self.data = scene_data
        self.nodes, self.order, self.depth = host_sah(scene_data.triangles, bins, leaf)
        leaf_tris = scene_data.triangles[self.order]
        self.leaf_triangles = leaf_tris
        self.tri_v = tri_vertices(leaf_tris)
        self.tri_key = tri_keys(leaf_tris)
        self.traversal_id = leaf_tris["metadata"][:, 2].copy()


def host_sah_oracle_inputs(oracle, sd):
    """Oracle render inputs over the reference's own binned-SAH hierarchy
    (Bvh<float> + FlattenCanonicalL3BinnedSah, oracle/_ref), or the product's
    host SAH builder where the reference library is absent; no GPU."""
    tri = sd.triangles
    if oracle.ref_available():
        nodes12, order, _ = oracle.ref_sah_build(tri_vertices(tri), np.ascontiguousarray(tri["metadata"][:, 2]))
        nodes = np.ascontiguousarray(nodes12).view(N.NODE_DTYPE).reshape(-1)
    else:
        nodes, order, _ = host_sah(tri)
    return oracle.OracleRenderInputs(sd, nodes, order)
