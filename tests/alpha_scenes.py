"""Alpha-masked test scenes (GeometryFlagAlphaMask / MaterialFlagAlphaMask,
SceneAbiV0.hpp:20, 42) and the coverage data re_scene_set_alpha_masks takes:
GpuMaterialV0 records (alpha factor = base_color_factor.w, cutoff =
surface_params.w, alpha layer / sampler = texture_image_indices.x /
texture_sampler_indices.x) and an alpha atlas (layers, h, w)."""
from __future__ import annotations

import numpy as np

from renderingengine_b200 import _native as N
from renderingengine_b200 import scenes

INVALID = 0xFFFFFFFF
SAMPLER = 7
CHECKER = 8  # texels per side of the checkerboard layer


def v0_material(alpha_factor=1.0, cutoff=0.5, layer=INVALID, sampler=INVALID) -> np.ndarray:
    m = np.zeros(1, N.MATERIAL_V0_DTYPE)
    m["base_color_factor"] = [0.8, 0.8, 0.8, alpha_factor]
    m["surface_params"] = [0.0, 0.5, 1.0, cutoff]
    m["texture_image_indices"] = [layer, INVALID, INVALID, INVALID]
    m["texture_sampler_indices"] = [sampler, INVALID, INVALID, INVALID]
    m["metadata"] = [0, 2, 0, 0]
    return m


def atlas() -> np.ndarray:
    """Layer 0: an 8 x 8 checkerboard (alpha 1 where (i + j) is even, else
    0.2); layer 1: seeded value noise in [0, 1] at 64 x 64 (nearest-sampled
    from the same 64 x 64 grid for layer 0, which repeats each checker texel
    8 x 8 times)."""
    n = 64
    j, i = np.mgrid[0:n, 0:n]
    ch = np.where(((i // (n // CHECKER)) + (j // (n // CHECKER))) % 2 == 0, 1.0, 0.2)
    rng = np.random.default_rng(3)
    noise = scenes.value_noise(i / n, j / n, rng, octaves=3, base_frequency=4)
    return np.stack([ch, noise]).astype(np.float32)


def mask_flags(tri: np.ndarray, masked: np.ndarray, via_material: np.ndarray | None = None) -> None:
    """Sets the alpha-mask flag on `masked` triangles (geometry flag, or the
    material flag where via_material)."""
    vm = np.zeros(len(tri), bool) if via_material is None else via_material
    tri["metadata"][:, 0] |= np.where(masked & ~vm, 2, 0).astype(np.uint32)
    tri["metadata"][:, 1] |= np.where(masked & vm, 2, 0).astype(np.uint32)


def checker_quads() -> scenes.SceneData:
    """A unit quad in z = 0 (texcoords = (x, y)) masked by the checkerboard
    layer, and an unmasked backstop quad in z = -1."""
    q0 = scenes._quad((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1))
    q1 = scenes._quad((-1, -1, -1), (2, -1, -1), (2, 2, -1), (-1, 2, -1), (0, 0, 1))
    pos = np.asarray([np.stack(t) for t in q0 + q1], np.float64).astype(np.float32)
    tri = scenes.canonical_triangles(pos, None, np.zeros(4, np.uint32), np.arange(4, dtype=np.uint32),
                                     np.array([0, 0, 1, 1], np.uint32))
    tri["texcoords"][:, :, :2] = pos[:, :, :2]
    mask_flags(tri, np.array([True, True, False, False]), np.array([False, True, False, False]))
    mats = np.concatenate([scenes.material(scenes.LAMBERT, base=(0.8, 0.2, 0.2)),
                           scenes.material(scenes.LAMBERT, base=(0.2, 0.8, 0.2))])
    cam = scenes.Camera.look_at((0.5, 0.5, 2.0), (0.5, 0.5, 0.0), 40.0)
    sd = scenes.SceneData("checker-quads", tri, mats, scenes.sphere_light((0.5, 0.5, 3.0), 0.2, (20, 20, 20)),
                          np.zeros(0, scenes.FIXTURE_TRIANGLE_DTYPE), cam, fingerprint=0xA1FA)
    sd.extra = {"alpha": {"materials": np.concatenate([v0_material(1.0, 0.5, 0, SAMPLER), v0_material()]),
                          "atlas": atlas(), "sampler_id": SAMPLER}}
    return sd


def checker_expected(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """True where the checkerboard keeps the z = 0 quad (texel centres only)."""
    i = np.floor(x * CHECKER).astype(int)
    j = np.floor(y * CHECKER).astype(int)
    return (i + j) % 2 == 0


def foliage(seed: int = 2, leaves: int = 3000) -> scenes.SceneData:
    """A small heightfield with `leaves` alpha-masked leaf quads (noise
    layer, random texcoord windows, cutoffs U[0.3, 0.7]; half flagged on the
    geometry, half on the material; a quarter alpha-factor-only), for film
    parity with the oracle."""
    sd = scenes.heightfield_scene(grid=48, spheres=32, seed=seed)
    rng = np.random.default_rng(seed)
    c = np.stack([rng.uniform(0.05, 0.95, leaves), rng.uniform(0.05, 0.3, leaves), rng.uniform(0.05, 0.95, leaves)], 1)
    a = rng.normal(size=(leaves, 3))
    a /= np.linalg.norm(a, axis=1, keepdims=True)
    b = np.cross(a, rng.normal(size=(leaves, 3)))
    b /= np.linalg.norm(b, axis=1, keepdims=True)
    s = rng.uniform(0.01, 0.04, (leaves, 1))
    p = [c - a * s - b * s, c + a * s - b * s, c + a * s + b * s, c - a * s + b * s]
    pos = np.concatenate([np.stack([p[0], p[1], p[2]], 1), np.stack([p[0], p[2], p[3]], 1)]).astype(np.float32)
    n = len(pos)
    base_mat = len(sd.materials)
    mat_idx = (base_mat + np.tile(np.arange(leaves) % 4, 2)).astype(np.uint32)
    tri = scenes.canonical_triangles(pos, None, np.full(n, 9000, np.uint32), np.arange(n, dtype=np.uint32), mat_idx,
                                     first_traversal_id=len(sd.triangles))
    u0 = rng.uniform(0, 0.7, (leaves, 2))
    uv = [u0, u0 + [0.3, 0], u0 + [0.3, 0.3], u0 + [0, 0.3]]
    tri["texcoords"][:leaves, :, :2] = np.stack([uv[0], uv[1], uv[2]], 1)
    tri["texcoords"][leaves:, :, :2] = np.stack([uv[0], uv[2], uv[3]], 1)
    via_mat = np.tile(np.arange(leaves) % 2 == 1, 2)
    mask_flags(tri, np.ones(n, bool), via_mat)
    sd.triangles = np.concatenate([sd.triangles, tri])
    sd.materials = np.concatenate([sd.materials] + [scenes.material(scenes.METALLIC_ROUGHNESS, base=(0.2, 0.6, 0.2),
                                                                    roughness=0.6)] * 4)
    v0 = np.concatenate([v0_material()] * base_mat + [
        v0_material(1.0, 0.45, 1, SAMPLER), v0_material(0.9, 0.6, 1, SAMPLER), v0_material(0.8, 0.3, 1, SAMPLER),
        v0_material(0.7, 0.5)])
    sd.extra = dict(sd.extra or {}, alpha={"materials": v0, "atlas": atlas(), "sampler_id": SAMPLER})
    return sd
