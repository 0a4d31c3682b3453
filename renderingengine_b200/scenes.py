"""Seeded synthetic scenes in the reference's canonical record formats.

Every generator returns a :class:`SceneData` holding world-space
``re_canonical_triangle`` records (CanonicalTraversalTriangle), PBR material
records (PbrMaterialGpu), light records (PbrLightGpu), the emissive-triangle
fixture records the light sampler reads (FixtureTriangleGpu), and a camera.

Workloads (shapes and value distributions of the benchmark configurations):
  * ``cornell_reference`` -- the reference CPU fixture (36 triangles, light
    0.6 x 0.6 with radiance 17/15/12), the geometry of
    src/integrators/reference_cpu/CornellReference.cpp:234-310.
  * ``cornell_box`` -- the 640x360 workload: five walls and two boxes
    (34 triangles) plus a 0.25 x 0.25 emitting quad (17/12/4).
  * ``heightfield_scene`` -- 1024^2-cell heightfield (2,097,152 triangles,
    6-octave value noise, amplitude 0.2) + 4,096 icospheres (80 triangles,
    radii U[0.002, 0.02]); GGX materials, 10% rough dielectrics with
    Beer-Lambert attenuation; one spherical light.
  * ``add_emissive_triangles`` -- 10,000 emissive triangles for the many-light
    ReSTIR workload.
  * ``triangle_soup`` -- random triangles in the unit cube, edges <= 0.01.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from ._native import (GEOMETRY_FLAG_DOUBLE_SIDED, INSTANCE_FLAG_CASTS_SHADOW, INSTANCE_FLAG_VISIBLE,
                      LIGHT_DTYPE, MATERIAL_DTYPE, TRIANGLE_DTYPE)

# BSDF models / lobes (PbrBsdf.hlsli:55-80).
LAMBERT, GGX_CONDUCTOR, GGX_DIELECTRIC_REFLECTION, SMOOTH_GLASS, ROUGH_DIELECTRIC, METALLIC_ROUGHNESS = range(6)
LOBE_DIFFUSE, LOBE_GLOSSY, LOBE_SPECULAR, LOBE_REFLECTION, LOBE_TRANSMISSION = 1, 2, 4, 8, 16
LOBES_OPAQUE = LOBE_DIFFUSE | LOBE_GLOSSY | LOBE_REFLECTION
LOBES_DIELECTRIC = LOBE_GLOSSY | LOBE_SPECULAR | LOBE_REFLECTION | LOBE_TRANSMISSION
LOBES_ALL = 0x1F
PURE_EMITTER = 1
# Light types / flags (pbr_l6_types.hlsli:11-22).
LIGHT_SPHERE_AREA, LIGHT_EMISSIVE_TRIANGLE, LIGHT_ENVIRONMENT = 3, 4, 5
LIGHT_ENABLED, LIGHT_TWO_SIDED = 1, 2

FIXTURE_TRIANGLE_DTYPE = np.dtype([("p0", "<f4", 4), ("p1", "<f4", 4), ("p2", "<f4", 4),
                                   ("metadata", "<u4", 4)])  # material, primitive, instance, flags


@dataclass
class Camera:
    position: np.ndarray
    forward: np.ndarray
    right: np.ndarray
    up: np.ndarray
    tan_half_fov: float

    @staticmethod
    def look_at(eye, target, vfov_degrees: float, world_up=(0.0, 1.0, 0.0)) -> "Camera":
        eye = np.asarray(eye, np.float64)
        f = np.asarray(target, np.float64) - eye
        f /= np.linalg.norm(f)
        r = np.cross(f, np.asarray(world_up, np.float64))
        r /= np.linalg.norm(r)
        u = np.cross(r, f)
        return Camera(eye.astype(np.float32), f.astype(np.float32), r.astype(np.float32),
                      u.astype(np.float32), float(math.tan(math.radians(vfov_degrees) * 0.5)))


@dataclass
class SceneData:
    name: str
    triangles: np.ndarray                      # TRIANGLE_DTYPE
    materials: np.ndarray                      # MATERIAL_DTYPE
    lights: np.ndarray                         # LIGHT_DTYPE
    fixture_triangles: np.ndarray              # FIXTURE_TRIANGLE_DTYPE (emissive triangles)
    camera: Camera
    fingerprint: int = 1
    generation: int = 1
    extra: dict = field(default_factory=dict)

    @property
    def positions(self) -> np.ndarray:
        """(n, 3, 3) float32 world positions."""
        return self.triangles["positions"][:, :, :3]


# ---------------------------------------------------------------------------
# Record helpers
# ---------------------------------------------------------------------------
def canonical_triangles(pos: np.ndarray, normals: np.ndarray | None, instance: np.ndarray,
                        primitive: np.ndarray, material: np.ndarray,
                        first_traversal_id: int = 0, double_sided: bool = True) -> np.ndarray:
    n = pos.shape[0]
    t = np.zeros(n, TRIANGLE_DTYPE)
    t["positions"][:, :, :3] = pos
    t["positions"][:, :, 3] = 1.0
    if normals is None:
        g = np.cross(pos[:, 1] - pos[:, 0], pos[:, 2] - pos[:, 0])
        g /= np.maximum(np.linalg.norm(g, axis=1, keepdims=True), 1e-30)
        normals = np.repeat(g[:, None, :], 3, axis=1)
    t["normals"][:, :, :3] = normals
    t["identity"][:, 0] = instance
    t["identity"][:, 1] = primitive
    t["identity"][:, 2] = 0
    t["identity"][:, 3] = material
    t["metadata"][:, 0] = GEOMETRY_FLAG_DOUBLE_SIDED if double_sided else 0
    t["metadata"][:, 1] = 0
    t["metadata"][:, 2] = np.arange(first_traversal_id, first_traversal_id + n, dtype=np.uint32)
    t["metadata"][:, 3] = INSTANCE_FLAG_VISIBLE | INSTANCE_FLAG_CASTS_SHADOW
    return t


def material(model: int, base=(0.8, 0.8, 0.8), metallic=0.0, roughness=0.5, emission=(0, 0, 0),
             transmission=0.0, ior=1.5, attenuation=(1.0, 1.0, 1.0), attenuation_distance=0.0,
             lobes: int | None = None, pure_emitter: bool = False) -> np.ndarray:
    m = np.zeros(1, MATERIAL_DTYPE)
    base = np.asarray(base, np.float32)
    m["base_color_metallic"] = [*base, metallic]
    m["emissive_roughness"] = [*emission, roughness]
    m["transmission_ior"] = [transmission, ior, 0, 0]
    m["attenuation_color_distance"] = [*attenuation, attenuation_distance]
    f0 = 0.04 * (1.0 - metallic) + base * metallic  # glTF metallic-roughness F0
    m["f0"] = [*f0, 0]
    m["conductor_eta"] = [1, 1, 1, 0]
    if lobes is None:
        lobes = LOBES_OPAQUE if model in (LAMBERT, METALLIC_ROUGHNESS, GGX_CONDUCTOR,
                                          GGX_DIELECTRIC_REFLECTION) else LOBES_DIELECTRIC
    m["metadata"] = [model, lobes, 0, PURE_EMITTER if pure_emitter else 0]
    return m


def environment_light(radiance=(1.0, 1.0, 1.0), scale: float = 1.0, light_id: int = 0) -> np.ndarray:
    """An enabled environment light (PbrLightGpu type 5); its map is the
    scene's ``extra["environment"]`` (height, width, 4) linear RGBA."""
    l = np.zeros(1, LIGHT_DTYPE)
    l["radiance_scale"] = [*radiance, scale]
    l["identity"] = [LIGHT_ENVIRONMENT, LIGHT_ENABLED, light_id, 0xFFFFFFFF]
    l["payload"] = [0xFFFFFFFF, 0xFFFFFFFF, 0, 0xFFFFFFFF]
    return l


def sky_environment(width: int = 64, height: int = 32, seed: int = 0, sun=(0.35, 0.6), sun_radiance=400.0):
    """A seeded equirectangular sky: a vertical gradient, value-noise clouds
    and a small bright sun texel block at (u, v) = `sun`; (height, width, 4)."""
    rng = np.random.default_rng(seed)
    v = (np.arange(height) + 0.5) / height
    u = (np.arange(width) + 0.5) / width
    U, V = np.meshgrid(u, v)
    sky = np.stack([0.3 + 0.5 * (1 - V), 0.45 + 0.45 * (1 - V), 0.8 + 0.2 * (1 - V)], -1)
    clouds = value_noise(U, V, rng, octaves=4, base_frequency=4)[..., None]
    env = np.concatenate([sky * (0.4 + 0.8 * clouds), np.ones((height, width, 1))], -1)
    su, sv = int(sun[0] * width), int(sun[1] * height)
    env[max(sv - 1, 0):sv + 1, max(su - 1, 0):su + 1, :3] = sun_radiance
    return env.astype(np.float32)


def sphere_light(center, radius: float, radiance, scale: float = 1.0, light_id: int = 0) -> np.ndarray:
    l = np.zeros(1, LIGHT_DTYPE)
    l["position_range"] = [*center, 0.0]
    l["radiance_scale"] = [*radiance, scale]
    l["shape_params"] = [radius, 0, 0, 0]
    l["identity"] = [LIGHT_SPHERE_AREA, LIGHT_ENABLED, light_id, 0xFFFFFFFF]
    l["payload"] = [0xFFFFFFFF, 0xFFFFFFFF, 0, 0xFFFFFFFF]
    return l


def _emissive_light_records(tri_pos: np.ndarray, radiance: np.ndarray, fixture_offset: int,
                            instance: np.ndarray, primitive: np.ndarray, material_ids: np.ndarray,
                            first_light_id: int, two_sided: bool = False):
    n = tri_pos.shape[0]
    lights = np.zeros(n, LIGHT_DTYPE)
    fix = np.zeros(n, FIXTURE_TRIANGLE_DTYPE)
    fix["p0"][:, :3] = tri_pos[:, 0]
    fix["p1"][:, :3] = tri_pos[:, 1]
    fix["p2"][:, :3] = tri_pos[:, 2]
    fix["metadata"][:, 0] = material_ids
    fix["metadata"][:, 1] = primitive
    fix["metadata"][:, 2] = instance
    area = 0.5 * np.linalg.norm(np.cross(tri_pos[:, 1] - tri_pos[:, 0], tri_pos[:, 2] - tri_pos[:, 0]), axis=1)
    lights["radiance_scale"][:, :3] = radiance
    lights["radiance_scale"][:, 3] = 1.0
    lights["shape_params"][:, 2] = area
    lights["identity"][:, 0] = LIGHT_EMISSIVE_TRIANGLE
    lights["identity"][:, 1] = LIGHT_ENABLED | (LIGHT_TWO_SIDED if two_sided else 0)
    lights["identity"][:, 2] = np.arange(first_light_id, first_light_id + n)
    lights["identity"][:, 3] = primitive
    lights["payload"][:, 0] = np.arange(fixture_offset, fixture_offset + n)
    lights["payload"][:, 1] = 0xFFFFFFFF
    lights["payload"][:, 2] = 0
    lights["payload"][:, 3] = instance
    return lights, fix


# ---------------------------------------------------------------------------
# Cornell boxes
# ---------------------------------------------------------------------------
def _quad(v0, v1, v2, v3, normal):
    """Two triangles (v0 v1 v2), (v0 v2 v3), swapping v1/v3 so the winding
    normal faces `normal` (the AddQuad rule, CornellReference.cpp:184-201)."""
    v0, v1, v2, v3 = (np.asarray(v, np.float64) for v in (v0, v1, v2, v3))
    if not np.dot(np.cross(v1 - v0, v2 - v0), normal) > 0.0:
        v1, v3 = v3, v1
    return [(v0, v1, v2), (v0, v2, v3)]


def _box(lo, hi):
    (x0, y0, z0), (x1, y1, z1) = lo, hi
    p = {(i, j, k): (x1 if i else x0, y1 if j else y0, z1 if k else z0)
         for i in (0, 1) for j in (0, 1) for k in (0, 1)}
    tris = []
    tris += _quad(p[0, 0, 0], p[0, 0, 1], p[0, 1, 1], p[0, 1, 0], (-1, 0, 0))
    tris += _quad(p[1, 0, 0], p[1, 1, 0], p[1, 1, 1], p[1, 0, 1], (1, 0, 0))
    tris += _quad(p[0, 0, 0], p[1, 0, 0], p[1, 0, 1], p[0, 0, 1], (0, -1, 0))
    tris += _quad(p[0, 1, 0], p[0, 1, 1], p[1, 1, 1], p[1, 1, 0], (0, 1, 0))
    tris += _quad(p[0, 0, 0], p[0, 1, 0], p[1, 1, 0], p[1, 0, 0], (0, 0, -1))
    tris += _quad(p[0, 0, 1], p[1, 0, 1], p[1, 1, 1], p[0, 1, 1], (0, 0, 1))
    return tris


def _cornell(light_corner, light_size, light_radiance, green, name, include_light_in_count=True):
    X0, X1, Y0, Y1, ZF, ZB = -1.0, 1.0, -1.0, 1.0, -1.0, -3.0
    groups = []  # (triangles, material)
    groups.append((_quad((X0, Y0, ZF), (X1, Y0, ZF), (X1, Y0, ZB), (X0, Y0, ZB), (0, 1, 0)), 0))
    groups.append((_quad((X0, Y1, ZF), (X0, Y1, ZB), (X1, Y1, ZB), (X1, Y1, ZF), (0, -1, 0)), 0))
    groups.append((_quad((X0, Y0, ZB), (X1, Y0, ZB), (X1, Y1, ZB), (X0, Y1, ZB), (0, 0, 1)), 0))
    groups.append((_quad((X0, Y0, ZF), (X0, Y0, ZB), (X0, Y1, ZB), (X0, Y1, ZF), (1, 0, 0)), 1))
    groups.append((_quad((X1, Y0, ZF), (X1, Y1, ZF), (X1, Y1, ZB), (X1, Y0, ZB), (-1, 0, 0)), 2))
    c = np.asarray(light_corner, np.float64)
    eu = np.array([light_size, 0.0, 0.0])
    ev = np.array([0.0, 0.0, light_size])
    groups.append((_quad(c, c + eu, c + eu + ev, c + ev, (0, -1, 0)), 3))
    groups.append((_box((-0.72, -0.999, -2.55), (-0.10, -0.30, -1.72)), 0))
    groups.append((_box((0.16, -0.999, -2.75), (0.74, 0.22, -1.93)), 0))
    pos, mats = [], []
    for tris, m in groups:
        for t in tris:
            pos.append(np.stack(t))
            mats.append(m)
    pos = np.asarray(pos, np.float64).astype(np.float32)
    mats = np.asarray(mats, np.uint32)
    n = pos.shape[0]
    tri = canonical_triangles(pos, None, np.zeros(n, np.uint32), np.arange(n, dtype=np.uint32), mats)
    materials = np.concatenate([
        material(LAMBERT, base=(0.73, 0.73, 0.73)),
        material(LAMBERT, base=(0.63, 0.065, 0.05)),
        material(LAMBERT, base=green),
        material(LAMBERT, base=(0.0, 0.0, 0.0), emission=light_radiance, pure_emitter=True),
    ])
    emitter = np.nonzero(mats == 3)[0]
    lights, fix = _emissive_light_records(pos[emitter].astype(np.float32),
                                          np.tile(np.asarray(light_radiance, np.float32), (len(emitter), 1)),
                                          0, np.zeros(len(emitter), np.uint32), emitter.astype(np.uint32),
                                          np.full(len(emitter), 3, np.uint32), 0)
    cam = Camera.look_at((0.0, 0.0, 0.15), (0.0, 0.0, -1.0), 39.0)
    return SceneData(name, tri, materials, lights, fix, cam, fingerprint=0x434F524E454C4C,
                     extra={"emitter_triangles": emitter})


def cornell_reference() -> SceneData:
    """The reference CPU fixture (CornellReference.cpp:234-310): 36 triangles."""
    return _cornell((-0.30, 0.985, -2.30), 0.60, (17.0, 15.0, 12.0), (0.14, 0.45, 0.091), "cornell-reference")


def cornell_box() -> SceneData:
    """The 640x360 Cornell workload: 34 wall/box triangles + a 0.25^2 light quad."""
    return _cornell((-0.125, 0.985, -2.125), 0.25, (17.0, 12.0, 4.0), (0.14, 0.45, 0.09), "cornell")


# ---------------------------------------------------------------------------
# Heightfield + icospheres
# ---------------------------------------------------------------------------
def value_noise(xs: np.ndarray, zs: np.ndarray, rng: np.random.Generator, octaves: int = 6,
                base_frequency: int = 4) -> np.ndarray:
    """Seeded lattice value noise with smoothstep interpolation, summed over
    octaves with halving amplitude, normalised to [0, 1]."""
    total = np.zeros(np.broadcast(xs, zs).shape, np.float64)
    amp_sum = 0.0
    amp = 1.0
    for o in range(octaves):
        f = base_frequency << o
        lattice = rng.random((f + 1, f + 1))
        gx, gz = xs * f, zs * f
        ix = np.clip(np.floor(gx).astype(np.int64), 0, f - 1)
        iz = np.clip(np.floor(gz).astype(np.int64), 0, f - 1)
        tx, tz = gx - ix, gz - iz
        sx, sz = tx * tx * (3 - 2 * tx), tz * tz * (3 - 2 * tz)
        a = lattice[ix, iz] * (1 - sx) + lattice[ix + 1, iz] * sx
        b = lattice[ix, iz + 1] * (1 - sx) + lattice[ix + 1, iz + 1] * sx
        total += amp * (a * (1 - sz) + b * sz)
        amp_sum += amp
        amp *= 0.5
    return total / amp_sum


def _icosphere() -> tuple[np.ndarray, np.ndarray]:
    t = (1.0 + 5 ** 0.5) / 2.0
    v = np.array([(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
                  (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)], np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
         (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = list(map(tuple, v))
    cache = {}

    def mid(a, b):
        key = (min(a, b), max(a, b))
        if key not in cache:
            m = (np.asarray(verts[a]) + np.asarray(verts[b])) * 0.5
            verts.append(tuple(m / np.linalg.norm(m)))
            cache[key] = len(verts) - 1
        return cache[key]

    faces = []
    for a, b, c in f:
        ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
        faces += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
    return np.asarray(verts, np.float64), np.asarray(faces, np.int64)


def heightfield_scene(grid: int = 1024, spheres: int = 4096, seed: int = 1,
                      light_radiance=(30.0, 28.5, 25.5)) -> SceneData:
    rng = np.random.default_rng(seed)
    g = grid
    lin = np.linspace(0.0, 1.0, g + 1)
    X, Z = np.meshgrid(lin, lin, indexing="ij")
    H = 0.2 * value_noise(X, Z, rng)
    P = np.stack([X, H, Z], axis=-1)  # (g+1, g+1, 3)
    dhx = np.gradient(H, lin, axis=0)
    dhz = np.gradient(H, lin, axis=1)
    N = np.stack([-dhx, np.ones_like(H), -dhz], axis=-1)
    N /= np.linalg.norm(N, axis=-1, keepdims=True)
    i, j = np.meshgrid(np.arange(g), np.arange(g), indexing="ij")
    i, j = i.ravel(), j.ravel()
    # Cell corners a=(i,j) b=(i+1,j) c=(i+1,j+1) d=(i,j+1); winding (a, d, c)
    # and (a, c, b) gives +y facing normals.  Two triangles per cell, cells in
    # row-major order.
    ci = np.stack([np.stack([i, i, i + 1], 1), np.stack([i, i + 1, i + 1], 1)], 1).reshape(-1, 3)
    cj = np.stack([np.stack([j, j + 1, j + 1], 1), np.stack([j, j + 1, j], 1)], 1).reshape(-1, 3)
    hf_pos = P[ci, cj].astype(np.float32)
    hf_nrm = N[ci, cj].astype(np.float32)
    n_hf = hf_pos.shape[0]

    sv, sf = _icosphere()
    radii = rng.uniform(0.002, 0.02, spheres)
    cx = rng.uniform(0.02, 0.98, spheres)
    cz = rng.uniform(0.02, 0.98, spheres)
    # Height under the centre (bilinear on the vertex grid) + radius + lift.
    fx, fz = cx * g, cz * g
    ix, iz = np.minimum(fx.astype(np.int64), g - 1), np.minimum(fz.astype(np.int64), g - 1)
    tx, tz = fx - ix, fz - iz
    h = (H[ix, iz] * (1 - tx) * (1 - tz) + H[ix + 1, iz] * tx * (1 - tz) + H[ix, iz + 1] * (1 - tx) * tz
         + H[ix + 1, iz + 1] * tx * tz)
    cy = h + radii * rng.uniform(1.0, 3.0, spheres)
    centers = np.stack([cx, cy, cz], 1)
    sp_pos = (centers[:, None, None, :] + radii[:, None, None, None] * sv[sf][None]).astype(np.float32)
    sp_nrm = np.broadcast_to(sv[sf][None], sp_pos.shape).astype(np.float32)
    sp_pos = sp_pos.reshape(-1, 3, 3)
    sp_nrm = sp_nrm.reshape(-1, 3, 3)
    per = sf.shape[0]

    # Materials: 0 = terrain; 1 + k = sphere k.
    mats = [material(METALLIC_ROUGHNESS, base=(0.55, 0.5, 0.45), metallic=0.0, roughness=0.7)]
    rough = rng.uniform(0.05, 1.0, spheres)
    metal = rng.random(spheres) < 0.3
    dielectric = rng.random(spheres) < 0.1
    sigma = rng.uniform(0.0, 2.0, spheres)
    colors = rng.uniform(0.2, 0.95, (spheres, 3))
    for k in range(spheres):
        if dielectric[k]:
            att = np.exp(-sigma[k] * 1.0) * np.ones(3)
            mats.append(material(ROUGH_DIELECTRIC, base=(1, 1, 1), roughness=float(rough[k]),
                                 transmission=1.0, ior=1.5, attenuation=att, attenuation_distance=1.0))
        else:
            mats.append(material(METALLIC_ROUGHNESS, base=colors[k], metallic=1.0 if metal[k] else 0.0,
                                 roughness=float(rough[k])))
    materials = np.concatenate(mats)

    pos = np.concatenate([hf_pos, sp_pos])
    nrm = np.concatenate([hf_nrm, sp_nrm])
    inst = np.concatenate([np.zeros(n_hf, np.uint32), np.repeat(np.arange(1, spheres + 1, dtype=np.uint32), per)])
    prim = np.concatenate([np.arange(n_hf, dtype=np.uint32), np.tile(np.arange(per, dtype=np.uint32), spheres)])
    mat = np.concatenate([np.zeros(n_hf, np.uint32), np.repeat(np.arange(1, spheres + 1, dtype=np.uint32), per)])
    tri = canonical_triangles(pos, nrm, inst, prim, mat)
    lights = sphere_light((0.3, 0.9, 0.35), 0.08, light_radiance)
    cam = Camera.look_at((0.5, 0.55, -0.35), (0.5, 0.05, 0.55), 45.0)
    return SceneData(f"heightfield-{grid}-{spheres}", tri, materials, lights,
                     np.zeros(0, FIXTURE_TRIANGLE_DTYPE), cam, fingerprint=0x48460000 + seed,
                     extra={"heights": H.astype(np.float32), "grid": g, "dielectric": dielectric})


def add_emissive_triangles(scene: SceneData, count: int = 10000, seed: int = 7) -> SceneData:
    """Adds `count` emissive triangles (areas log-uniform in [1e-5, 1e-2],
    radiance log-uniform in [0.1, 100]) a little above seeded heightfield
    points, facing up, as both geometry and emissive-triangle lights."""
    rng = np.random.default_rng(seed)
    H = scene.extra["heights"]
    g = scene.extra["grid"]
    area = np.exp(rng.uniform(np.log(1e-5), np.log(1e-2), count))
    rad = np.exp(rng.uniform(np.log(0.1), np.log(100.0), count))
    hue = rng.uniform(0.5, 1.0, (count, 3))
    radiance = (rad[:, None] * hue).astype(np.float32)
    cx, cz = rng.uniform(0.05, 0.95, count), rng.uniform(0.05, 0.95, count)
    ix = np.minimum((cx * g).astype(np.int64), g - 1)
    iz = np.minimum((cz * g).astype(np.int64), g - 1)
    cy = np.maximum.reduce([H[ix, iz], H[ix + 1, iz], H[ix, iz + 1], H[ix + 1, iz + 1]]) + 0.004
    side = np.sqrt(4.0 * area / np.sqrt(3.0))  # equilateral triangle of the given area
    ang = rng.uniform(0, 2 * np.pi, count)
    verts = []
    for k in range(3):
        a = ang + k * 2 * np.pi / 3
        r = side / np.sqrt(3.0)
        verts.append(np.stack([cx + r * np.cos(a), cy, cz - r * np.sin(a)], 1))
    pos = np.stack(verts, 1).astype(np.float32)  # counter-clockwise seen from +y -> normal +y
    n0 = scene.triangles.shape[0]
    inst_id = int(scene.triangles["identity"][:, 0].max()) + 1
    m0 = scene.materials.shape[0]
    mats = np.zeros(count, MATERIAL_DTYPE)
    mats["emissive_roughness"][:, :3] = radiance
    mats["emissive_roughness"][:, 3] = 1.0
    mats["f0"][:, :3] = 0.04
    mats["metadata"][:, 0] = LAMBERT
    mats["metadata"][:, 1] = LOBES_OPAQUE
    mats["metadata"][:, 3] = PURE_EMITTER
    tri = canonical_triangles(pos, None, np.full(count, inst_id, np.uint32), np.arange(count, dtype=np.uint32),
                              np.arange(m0, m0 + count, dtype=np.uint32), first_traversal_id=n0)
    lights, fix = _emissive_light_records(pos, radiance, scene.fixture_triangles.shape[0],
                                          np.full(count, inst_id, np.uint32), np.arange(count, dtype=np.uint32),
                                          np.arange(m0, m0 + count, dtype=np.uint32), scene.lights.shape[0])
    return SceneData(scene.name + f"-{count}lights", np.concatenate([scene.triangles, tri]),
                     np.concatenate([scene.materials, mats]), np.concatenate([scene.lights, lights]),
                     np.concatenate([scene.fixture_triangles, fix]), scene.camera,
                     fingerprint=scene.fingerprint ^ 0x4C494748, extra=dict(scene.extra))


def triangle_soup(count: int = 500_000, seed: int = 3, max_edge: float = 0.01) -> SceneData:
    rng = np.random.default_rng(seed)
    c = rng.random((count, 3))
    # Random orthonormal frame per triangle; vertices on a circle of radius
    # <= max_edge / 2 at well-separated angles, so every edge is <= max_edge
    # and no triangle is degenerate.
    a = rng.normal(size=(count, 3))
    a /= np.linalg.norm(a, axis=1, keepdims=True)
    b = np.cross(a, rng.normal(size=(count, 3)))
    b /= np.linalg.norm(b, axis=1, keepdims=True)
    ang = rng.uniform(0, 2 * np.pi, (count, 1)) + np.array([0.0, 2.0, 4.0])[None, :] \
        + rng.uniform(-0.3, 0.3, (count, 3))
    r = rng.uniform(0.3, 1.0, (count, 3)) * (max_edge * 0.5)
    pos = (c[:, None, :] + (np.cos(ang) * r)[..., None] * a[:, None, :]
           + (np.sin(ang) * r)[..., None] * b[:, None, :]).astype(np.float32)
    tri = canonical_triangles(pos, None, np.zeros(count, np.uint32), np.arange(count, dtype=np.uint32),
                              np.zeros(count, np.uint32))
    materials = material(METALLIC_ROUGHNESS, base=(0.7, 0.7, 0.7), roughness=0.6)
    lights = sphere_light((0.5, 1.6, 0.5), 0.2, (20.0, 20.0, 20.0))
    cam = Camera.look_at((0.5, 0.5, -1.2), (0.5, 0.5, 0.5), 45.0)
    return SceneData(f"soup-{count}", tri, materials, lights, np.zeros(0, FIXTURE_TRIANGLE_DTYPE), cam,
                     fingerprint=0x534F5550 + seed)


# ---------------------------------------------------------------------------
# Ray batches
# ---------------------------------------------------------------------------
def pinhole_rays(camera: Camera, width: int, height: int, seed: int = 0, jitter: bool = True,
                 tmin: float = 1e-4) -> np.ndarray:
    """(width*height, 8) float32 primary rays (origin, tMin, direction, tMax)."""
    rng = np.random.default_rng(seed)
    x = (np.arange(width, dtype=np.float32)[None, :] + (rng.random((height, width), np.float32) if jitter else 0.5))
    y = (np.arange(height, dtype=np.float32)[:, None] + (rng.random((height, width), np.float32) if jitter else 0.5))
    sx = (x / width) * 2 - 1
    sy = -((y / height) * 2 - 1)
    aspect = width / height
    d = (camera.forward[None, None, :] + camera.right[None, None, :] * (sx * aspect * camera.tan_half_fov)[..., None]
         + camera.up[None, None, :] * (sy * camera.tan_half_fov)[..., None])
    d = d / np.linalg.norm(d, axis=-1, keepdims=True)
    rays = np.zeros((height * width, 8), np.float32)
    rays[:, :3] = camera.position
    rays[:, 3] = tmin
    rays[:, 4:7] = d.reshape(-1, 3)
    rays[:, 7] = 1e30
    return rays


def random_rays(lo, hi, count: int, seed: int = 0, tmin: float = 1e-6) -> np.ndarray:
    """Origins uniform in the box [lo, hi], uniformly random unit directions."""
    rng = np.random.default_rng(seed)
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    o = lo + rng.random((count, 3)) * (hi - lo)
    d = rng.normal(size=(count, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((count, 8), np.float32)
    rays[:, :3] = o
    rays[:, 3] = tmin
    rays[:, 4:7] = d
    rays[:, 7] = 1e30
    return rays


def to_ray_records(rays8: np.ndarray, path_ids: np.ndarray | None = None):
    from ._native import RAY_DTYPE
    n = rays8.shape[0]
    r = np.zeros(n, RAY_DTYPE)
    r["origin_tmin"] = rays8[:, :4]
    r["direction_tmax"] = rays8[:, 4:8]
    r["identity"][:, 0] = np.arange(n, dtype=np.uint32)
    r["identity"][:, 1] = np.arange(n, dtype=np.uint32) if path_ids is None else path_ids
    r["identity"][:, 3] = 0xFFFFFFFF
    return r
