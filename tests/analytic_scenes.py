"""Scenes whose converged images have a closed form, and that form computed
in double precision.

``glass_slab``: a camera looking down -z through a slab of smooth glass
(IOR 1.5, Beer-Lambert attenuation colour c at distance D, thickness d)
at a large one-sided emitter of radiance L behind it; nothing else.  A
camera path either reflects off the front face (and escapes: black), or
refracts in, travels s = d / cos(theta_t), and at each face reflects with
the exact dielectric Fresnel probability F or refracts; every refraction
multiplies the throughput by 1 / eta_rel^2 (radiance transport) and every
unit of in-medium distance by c^(1 / D).  The expected pixel value is

    E = L (1 - F)^2 sum_k F^(2k) c^((2k + 1) s / D)

over the internal round trips k the bounce limit leaves room for (the
emitter hit of round trip k is path vertex 2 + 2k), and the estimator's
second moment is L^2 (1 - F)^2 sum_k F^(2k) c^(2 (2k + 1) s / D): the
per-sample value is L c^((2k+1) s / D) with probability (1 - F)^2 F^(2k),
else 0.  Pixel footprints are integrated with an 8 x 8 midpoint grid."""
from __future__ import annotations

import numpy as np

from renderingengine_b200 import scenes

SLAB_Z0, SLAB_THICKNESS = -1.0, 0.3
EMITTER_Z = -2.5
IOR = 1.5
ATTENUATION = (0.55, 0.75, 0.9)
ATTENUATION_DISTANCE = 0.8
RADIANCE = (2.0, 1.5, 1.0)


def glass_slab() -> scenes.SceneData:
    S = 20.0
    z0, z1 = SLAB_Z0, SLAB_Z0 - SLAB_THICKNESS
    tris = scenes._box((-S, -S, z1), (S, S, z0))
    mats = [0] * len(tris)
    e = 60.0
    tris += scenes._quad((-e, -e, EMITTER_Z), (e, -e, EMITTER_Z), (e, e, EMITTER_Z), (-e, e, EMITTER_Z), (0, 0, 1))
    mats += [1, 1]
    pos = np.asarray([np.stack(t) for t in tris], np.float64).astype(np.float32)
    mats = np.asarray(mats, np.uint32)
    n = len(pos)
    tri = scenes.canonical_triangles(pos, None, np.zeros(n, np.uint32), np.arange(n, dtype=np.uint32), mats)
    materials = np.concatenate([
        scenes.material(scenes.SMOOTH_GLASS, base=(1, 1, 1), transmission=1.0, ior=IOR, attenuation=ATTENUATION,
                        attenuation_distance=ATTENUATION_DISTANCE),
        scenes.material(scenes.LAMBERT, base=(0, 0, 0), emission=RADIANCE, pure_emitter=True),
    ])
    em = np.nonzero(mats == 1)[0]
    lights, fix = scenes._emissive_light_records(pos[em], np.tile(np.asarray(RADIANCE, np.float32), (len(em), 1)),
                                                 0, np.zeros(len(em), np.uint32), em.astype(np.uint32),
                                                 np.full(len(em), 1, np.uint32), 0)
    cam = scenes.Camera.look_at((0.0, 0.0, 0.0), (0.0, 0.0, -1.0), 30.0)
    return scenes.SceneData("glass-slab", tri, materials, lights, fix, cam, fingerprint=0x534C4142)


def fresnel_dielectric(cos_i: np.ndarray, eta_i: float, eta_t: float) -> np.ndarray:
    """Exact unpolarised dielectric Fresnel reflectance."""
    ci = np.minimum(np.abs(cos_i), 1.0)
    st2 = (eta_i / eta_t) ** 2 * np.maximum(0.0, 1 - ci * ci)
    ct = np.sqrt(np.maximum(0.0, 1 - st2))
    rpar = (eta_t * ci - eta_i * ct) / (eta_t * ci + eta_i * ct)
    rper = (eta_i * ci - eta_t * ct) / (eta_i * ci + eta_t * ct)
    return np.where(st2 >= 1, 1.0, 0.5 * (rpar ** 2 + rper ** 2))


def glass_slab_expectation(camera: scenes.Camera, width: int, height: int, max_depth: int, sub: int = 8):
    """(mean, second moment) per pixel and channel, (h*w, 3) float64."""
    c = np.asarray(ATTENUATION, np.float64)
    L = np.asarray(RADIANCE, np.float64)
    fwd, right, up = (np.asarray(v, np.float64) for v in (camera.forward, camera.right, camera.up))
    t = camera.tan_half_fov
    aspect = width / height
    ys, xs = np.mgrid[0:height, 0:width]
    off = (np.arange(sub) + 0.5) / sub
    mean = np.zeros((height * width, 3))
    second = np.zeros((height * width, 3))
    kmax = (max_depth - 3) // 2
    for jy in off:
        for jx in off:
            sx = (xs.ravel() + jx) / width * 2 - 1
            sy = -((ys.ravel() + jy) / height * 2 - 1)
            d = fwd + right * (sx * aspect * t)[:, None] + up * (sy * t)[:, None]
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            cos1 = np.abs(d[:, 2])
            F = fresnel_dielectric(cos1, 1.0, IOR)
            sin2 = np.sqrt(np.maximum(0.0, 1 - cos1 ** 2)) / IOR
            cos2 = np.sqrt(1 - sin2 ** 2)
            s = SLAB_THICKNESS / cos2
            for k in range(kmax + 1):
                p = (1 - F) ** 2 * F ** (2 * k)
                a = c[None, :] ** (((2 * k + 1) * s / ATTENUATION_DISTANCE)[:, None])
                mean += (p[:, None] * a * L)
                second += (p[:, None] * (a * L) ** 2)
    n = sub * sub
    return mean / n, second / n


# ---------------------------------------------------------------------------
# White furnace: a plane under a constant environment.
# ---------------------------------------------------------------------------
FURNACE_NORMAL = np.array([0.0, 0.6, 0.8])  # unit


def furnace_plane(material: np.ndarray) -> scenes.SceneData:
    """A large square of `material` with normal FURNACE_NORMAL through the
    origin, seen by a camera on its front side, under a constant white
    environment (radiance 1) radiated by an environment light.  Every ray
    the plane reflects escapes, so a pixel's expected value is the
    material's directional albedo at that pixel's outgoing direction."""
    n = FURNACE_NORMAL / np.linalg.norm(FURNACE_NORMAL)
    t = np.cross(n, [1.0, 0.0, 0.0])
    t /= np.linalg.norm(t)
    b = np.cross(n, t)
    S = 50.0
    c = [(-S, -S), (S, -S), (S, S), (-S, S)]
    v = [t * x + b * y for x, y in c]
    tris = scenes._quad(v[0], v[1], v[2], v[3], n)
    pos = np.asarray([np.stack(q) for q in tris], np.float64).astype(np.float32)
    tri = scenes.canonical_triangles(pos, np.repeat(np.repeat(n[None, None, :], 3, 1), 2, 0).astype(np.float32),
                                     np.zeros(2, np.uint32), np.arange(2, dtype=np.uint32), np.zeros(2, np.uint32))
    lights = scenes.environment_light()
    cam = scenes.Camera.look_at(n * 2.0 + t * 0.3, np.zeros(3), 40.0)
    env = np.ones((8, 16, 4), np.float32)
    return scenes.SceneData("furnace", tri, material, lights, np.zeros(0, scenes.FIXTURE_TRIANGLE_DTYPE), cam,
                            fingerprint=0x46555247, extra={"environment": env})


def pixel_directions(camera: scenes.Camera, width: int, height: int, sub: int = 4) -> np.ndarray:
    """(h*w, sub*sub, 3) unit camera-ray directions over each pixel's footprint
    (midpoint grid), with the renderer's pinhole mapping."""
    fwd, right, up = (np.asarray(v, np.float64) for v in (camera.forward, camera.right, camera.up))
    tt, aspect = camera.tan_half_fov, width / height
    ys, xs = np.mgrid[0:height, 0:width]
    off = (np.arange(sub) + 0.5) / sub
    out = np.zeros((height * width, sub * sub, 3))
    k = 0
    for jy in off:
        for jx in off:
            sx = (xs.ravel() + jx) / width * 2 - 1
            sy = -((ys.ravel() + jy) / height * 2 - 1)
            d = fwd + right * (sx * aspect * tt)[:, None] + up * (sy * tt)[:, None]
            out[:, k] = d / np.linalg.norm(d, axis=1, keepdims=True)
            k += 1
    return out


def directional_albedo(oracle, material: np.ndarray, wo: np.ndarray, theta_steps: int = 128, phi_steps: int = 256):
    """FP64 directional albedo sum_i f(wo, wi) |cos| dOmega of `material`
    (PbrMaterialGpu record) on the furnace plane, per outgoing direction
    (n, 3), by midpoint quadrature in (theta, phi) (dOmega = sin theta
    dtheta dphi) of the reference's own EvaluateBsdfL6
    (ReferenceBsdf.hpp:922) over the hemisphere of FURNACE_NORMAL; (n, 3)."""
    import bsdf_cases as B
    n = FURNACE_NORMAL / np.linalg.norm(FURNACE_NORMAL)
    t = np.cross(n, [1.0, 0.0, 0.0])
    t /= np.linalg.norm(t)
    b = np.cross(n, t)
    th = 0.5 * np.pi * (np.arange(theta_steps) + 0.5) / theta_steps
    ph = 2 * np.pi * (np.arange(phi_steps) + 0.5) / phi_steps
    tt, pp = np.meshgrid(th, ph, indexing="ij")
    s, zz = np.sin(tt), np.cos(tt)
    wi = (s * np.cos(pp))[..., None] * t + (s * np.sin(pp))[..., None] * b + zz[..., None] * n
    wi = wi.reshape(-1, 3)
    dw = (s * (0.5 * np.pi / theta_steps) * (2 * np.pi / phi_steps)).reshape(-1)
    m = material[0]
    out = np.zeros((len(wo), 3))
    for i, w in enumerate(wo):
        q = np.zeros(len(wi), B.QUERY_DTYPE)
        q["geometric_normal"] = n
        q["shading_normal"] = n
        q["tangent"] = t
        q["eta_incident"], q["eta_transmitted"] = 1.0, m["transmission_ior"][1]
        q["base_color"] = m["base_color_metallic"][:3]
        q["metallic"] = m["base_color_metallic"][3]
        q["f0"] = m["f0"][:3]
        q["perceptual_roughness"] = m["emissive_roughness"][3]
        q["conductor_eta"] = m["conductor_eta"][:3]
        q["transmission"] = m["transmission_ior"][0]
        q["conductor_k"] = m["conductor_k"][:3]
        q["model"], q["allowed_lobes"], q["use_complex_conductor_fresnel"] = m["metadata"][:3]
        q["wo"] = w
        q["wi"] = wi
        r = B.reference_probe(oracle, q)
        ok = (r["eval_valid"] == 1) & (r["eval_measure"] == 1)
        cos = np.abs(wi @ n)
        out[i] = (np.where(ok[:, None], r["eval_value"], 0.0) * (cos * dw)[:, None]).sum(0)
    return out


FURNACE_MATERIALS = {
    "lambert": lambda: scenes.material(scenes.LAMBERT, base=(0.8, 0.55, 0.3)),
    "ggx-conductor": lambda: _conductor(),
    "metallic-roughness": lambda: scenes.material(scenes.METALLIC_ROUGHNESS, base=(0.9, 0.6, 0.2), metallic=0.5,
                                                   roughness=0.3),
    "ggx-dielectric-reflection": lambda: scenes.material(scenes.GGX_DIELECTRIC_REFLECTION, roughness=0.35),
}


def _conductor():
    m = scenes.material(scenes.GGX_CONDUCTOR, base=(0.9, 0.7, 0.5), roughness=0.45)
    m["f0"] = [0.9, 0.7, 0.5, 0.0]
    return m
