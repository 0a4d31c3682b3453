"""Scene ingestion: object-space SceneAbiV0 records (vertices, indices,
geometries, instances, materials) expanded on the GPU into world-space
CanonicalTraversalTriangle records (re_scene_expand_canonical, the GPU form
of BuildCanonicalTraversalScene, src/rt/gpu/CanonicalTraversalScene.cpp:69),
ready for Scene(...).  `instanced_heightfield` builds the traversal-bound
benchmark scene in instanced form: one heightfield mesh and one icosphere
mesh placed by per-instance transforms."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


def expand_canonical(vertices, indices, geometries, instances, materials, device: int = 0,
                     out_ptr: int | None = None, out_capacity: int = 0, stream: int | None = None):
    """Expands the scene; returns the TRIANGLE_DTYPE records (host), or the
    record count when `out_ptr` (device memory, `out_capacity` records) is
    given."""
    v = np.ascontiguousarray(vertices, N.VERTEX_V0_DTYPE)
    ix = np.ascontiguousarray(indices, np.uint32)
    g = np.ascontiguousarray(geometries, N.GEOMETRY_V0_DTYPE)
    inst = np.ascontiguousarray(instances, N.INSTANCE_V0_DTYPE)
    m = np.ascontiguousarray(materials, N.MATERIAL_V0_DTYPE)
    n = C.c_uint32(0)
    lib = N.load()
    if out_ptr is not None:
        N.check(lib.re_scene_expand_canonical(N.ptr(v), len(v), N.ptr(ix), len(ix), N.ptr(g), len(g), N.ptr(inst),
                                              len(inst), N.ptr(m), len(m), out_ptr, out_capacity, C.byref(n),
                                              N.MEMORY_DEVICE, device, stream))
        return int(n.value)
    out = np.zeros(max(expansion_count(g, inst), 1), N.TRIANGLE_DTYPE)
    N.check(lib.re_scene_expand_canonical(N.ptr(v), len(v), N.ptr(ix), len(ix), N.ptr(g), len(g), N.ptr(inst),
                                          len(inst), N.ptr(m), len(m), N.ptr(out), len(out), C.byref(n),
                                          N.MEMORY_HOST, device, stream))
    return out[:n.value]


def expansion_count(geometries, instances) -> int:
    """Triangles the expansion yields: one per started index triple of every
    geometry of every visible instance (ranges assumed valid)."""
    g = np.asarray(geometries, N.GEOMETRY_V0_DTYPE)
    per_geo = (g["index_range"][:, 1].astype(np.int64) + 2) // 3
    prefix = np.concatenate([[0], np.cumsum(per_geo)])
    total = 0
    for first, count, _, flags in np.asarray(instances, N.INSTANCE_V0_DTYPE)["metadata"].astype(np.int64):
        if flags & N.INSTANCE_FLAG_VISIBLE and first < len(g):
            total += int(prefix[min(first + count, len(g))] - prefix[first])
    return total


def _rows(mat: np.ndarray) -> np.ndarray:
    out = np.zeros((4, 4), np.float32)
    out[:3, :4] = mat[:3, :4]
    out[3] = (0, 0, 0, 1)
    return out


def instanced_heightfield(grid: int = 1024, spheres: int = 4096, subdivisions: int = 1, seed: int = 1,
                          per_instance: int = 4):
    """(vertices, indices, geometries, instances, materials) of a grid x grid
    heightfield (2 triangles per cell) plus `spheres` icospheres (20 x
    4^subdivisions triangles): `per_instance` copies of the icosphere mesh at
    fixed object-space offsets form one geometry each, and spheres /
    per_instance instances place them with random positions, uniform scales
    and rotations -- the benchmark's 2,424,832-triangle scene shape at the
    defaults.  (BuildCanonicalTraversalScene refuses scenes whose index count
    / 3 x instance count exceeds 2^32, so the instance count stays small.)"""
    rng = np.random.default_rng(seed)
    # Heightfield mesh in [0, 1]^2, heights from a few sines.
    xs = np.linspace(0.0, 1.0, grid + 1, dtype=np.float64)
    X, Z = np.meshgrid(xs, xs, indexing="xy")
    Y = 0.04 * np.sin(9.0 * X) * np.cos(7.0 * Z) + 0.02 * np.sin(23.0 * X + 5.0 * Z)
    hv = np.zeros((grid + 1) * (grid + 1), N.VERTEX_V0_DTYPE)
    hv["position"][:, 0], hv["position"][:, 1], hv["position"][:, 2] = X.ravel(), Y.ravel(), Z.ravel()
    hv["position"][:, 3] = 1.0
    hv["normal"][:, 1] = 1.0
    hv["texcoord0"][:, 0], hv["texcoord0"][:, 1] = X.ravel(), Z.ravel()
    r, c = np.meshgrid(np.arange(grid), np.arange(grid), indexing="ij")
    i0 = (r * (grid + 1) + c).ravel().astype(np.uint32)
    i1, i2, i3 = i0 + 1, i0 + grid + 1, i0 + grid + 2
    hidx = np.stack([i0, i2, i1, i1, i2, i3], axis=1).ravel().astype(np.uint32)
    # Icosphere mesh (unit radius).
    t = (1.0 + 5 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, np.float64) / np.linalg.norm(p) for p in verts]
    for _ in range(subdivisions):
        cache, nf = {}, []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                p = verts[a] + verts[b]
                verts.append(p / np.linalg.norm(p))
                cache[key] = len(verts) - 1
            return cache[key]
        for a, b, cc in faces:
            ab, bc, ca = mid(a, b), mid(b, cc), mid(cc, a)
            nf += [(a, ab, ca), (b, bc, ab), (cc, ca, bc), (ab, bc, ca)]
        faces = nf
    P = np.array(verts)
    offsets = [(0.0, 0.0, 0.0), (3.0, 0.0, 0.0), (0.0, 0.0, 3.0), (3.0, 0.0, 3.0)]
    copies = []
    for c in range(per_instance):
        sv = np.zeros(len(verts), N.VERTEX_V0_DTYPE)
        sv["position"][:, :3] = P + np.asarray(offsets[c % 4]) + np.array([0.0, 3.0 * (c // 4), 0.0])
        sv["position"][:, 3] = 1.0
        sv["normal"][:, :3] = P
        copies.append(sv)
    sidx = np.array(faces, np.uint32).ravel()
    vertices = np.concatenate([hv] + copies)
    indices = np.concatenate([hidx, sidx])
    geometries = np.zeros(1 + per_instance, N.GEOMETRY_V0_DTYPE)
    geometries[0]["index_range"] = (0, len(hidx), 0, 0)
    geometries[0]["identity"] = (0, 0, 0, 0)
    for c in range(per_instance):
        geometries[1 + c]["index_range"] = (len(hidx), len(sidx), len(hv) + c * len(verts), c * len(faces))
        geometries[1 + c]["identity"] = (1 + c, 1, 1, 0)
    materials = np.zeros(2, N.MATERIAL_V0_DTYPE)
    materials["metadata"][:, 0] = (5, 5)
    materials["metadata"][:, 2] = (0, 1)
    groups = spheres // per_instance
    instances = np.zeros(groups + 1, N.INSTANCE_V0_DTYPE)
    eye = np.eye(4, dtype=np.float32)
    instances[0]["object_to_world"] = eye
    instances[0]["world_to_object"] = eye
    instances[0]["metadata"] = (0, 1, 0, N.INSTANCE_FLAG_VISIBLE)
    for k in range(groups):
        s = rng.uniform(0.003, 0.012)
        a, b = rng.uniform(0, 2 * np.pi, 2)
        Rz = np.array([[np.cos(a), -np.sin(a), 0], [np.sin(a), np.cos(a), 0], [0, 0, 1]])
        Rx = np.array([[1, 0, 0], [0, np.cos(b), -np.sin(b)], [0, np.sin(b), np.cos(b)]])
        R = Rz @ Rx
        M = np.eye(4)
        M[:3, :3] = R * s
        M[:3, 3] = (rng.uniform(0, 1), rng.uniform(0.05, 0.15), rng.uniform(0, 1))
        Minv = np.linalg.inv(M)
        instances[k + 1]["object_to_world"] = _rows(M.astype(np.float32))
        instances[k + 1]["world_to_object"] = _rows(Minv.astype(np.float32))
        instances[k + 1]["metadata"] = (1, per_instance, k + 1, N.INSTANCE_FLAG_VISIBLE | (2 if k % 3 else 0))
    return vertices, indices, geometries, instances, materials
