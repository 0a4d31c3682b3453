"""Seeded generators of the multi-view and multi-request workloads: the
batch of many camera views over scenes of very different sizes, and the
Poisson request stream over a pool of synthetic scenes.  Pure numpy; the
scenes themselves come from `scenes`.

Batch: 64 views over four scenes (the Cornell box; the 2,424,832-triangle
heightfield + icosphere scene; the same with 10,000 emissive triangles,
rendered with ReSTIR DI; a 500,000-triangle random soup in the unit cube),
resolutions uniform over {256x256, 512x512, 1280x720, 1920x1080}, samples
per pixel uniform over {1, 4, 16}, maximum bounce 6.

Serving: Poisson arrivals at 200 requests/s over 16 scenes of 10k-5M
triangles (heightfields and soups, sizes log-spaced), resolution uniform over
{256x256, 1280x720, 1920x1080}, spp uniform over {1, 8, 64}, ReSTIR DI with
probability 0.5.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import scenes

BATCH_RESOLUTIONS = ((256, 256), (512, 512), (1280, 720), (1920, 1080))
BATCH_SPP = (1, 4, 16)
BATCH_DEPTH = 6
SERVE_RESOLUTIONS = ((256, 256), (1280, 720), (1920, 1080))
SERVE_SPP = (1, 8, 64)
SERVE_RATE = 200.0
SERVE_DEPTH = 6
# ReSTIR settings of the many-light configuration: 32 RIS candidates,
# temporal M-cap 20, one spatial pass of 5 neighbours in a 30-pixel disk.
RESTIR_MANY_LIGHTS = dict(candidates=32, max_m=20, spatial_neighbors=5, neighbor_mode=1, disk_radius=30.0)


@dataclass
class ViewSpec:
    scene: int          # index into the batch's scene list
    width: int
    height: int
    spp: int
    camera: scenes.Camera
    seed: int
    restir: bool

    @property
    def pixels(self) -> int:
        return self.width * self.height


def jittered_camera(cam: scenes.Camera, rng: np.random.Generator, scale: float) -> scenes.Camera:
    """The camera moved by a seeded offset of size ~`scale`, looking at the
    point one unit ahead of the original camera."""
    target = cam.position.astype(np.float64) + cam.forward.astype(np.float64)
    eye = cam.position.astype(np.float64) + rng.normal(0.0, scale, 3)
    vfov = np.degrees(2.0 * np.arctan(cam.tan_half_fov))
    return scenes.Camera.look_at(eye, target, float(vfov))


def batch_scenes(heightfield: scenes.SceneData | None = None):
    """[(SceneData, light_selection, restir, camera jitter scale)] of the batch."""
    hf = heightfield if heightfield is not None else scenes.heightfield_scene()
    return [
        (scenes.cornell_box(), 0, False, 0.05),
        (hf, 0, False, 0.02),
        (scenes.add_emissive_triangles(hf, count=10000), 1, True, 0.02),
        (scenes.triangle_soup(500_000), 0, False, 0.02),
    ]


def batch_views(scene_list, count: int = 64, seed: int = 0x5EED64) -> list[ViewSpec]:
    rng = np.random.default_rng(seed)
    out = []
    for v in range(count):
        k = v % len(scene_list)
        sd, _, restir, jitter = scene_list[k]
        w, h = BATCH_RESOLUTIONS[int(rng.integers(0, len(BATCH_RESOLUTIONS)))]
        spp = BATCH_SPP[int(rng.integers(0, len(BATCH_SPP)))]
        cam = jittered_camera(sd.camera, rng, jitter)
        out.append(ViewSpec(k, w, h, spp, cam, 0x10000 + v, restir))
    return out


@dataclass
class SceneRecipe:
    kind: str           # "heightfield" or "soup"
    triangles: int      # requested size
    seed: int

    def build(self) -> scenes.SceneData:
        if self.kind == "soup":
            return scenes.triangle_soup(self.triangles, seed=self.seed)
        # A grid of g x g cells gives 2 g^2 triangles, plus icospheres of 80.
        spheres = min(4096, max(8, self.triangles // 400))
        g = max(8, int(round(np.sqrt(max(self.triangles - 80 * spheres, 128) / 2.0))))
        return scenes.heightfield_scene(grid=g, spheres=spheres, seed=self.seed)


def serving_pool(count: int = 16, lo: float = 1e4, hi: float = 5e6, seed: int = 0x5E12) -> list[SceneRecipe]:
    """`count` scenes with sizes log-spaced in [lo, hi], alternating
    heightfields and random soups."""
    sizes = np.exp(np.linspace(np.log(lo), np.log(hi), count)).round().astype(np.int64)
    return [SceneRecipe("heightfield" if k % 2 == 0 else "soup", int(n), seed + k) for k, n in enumerate(sizes)]


@dataclass
class RequestSpec:
    arrival: float      # seconds after the stream starts
    scene: int          # index into the pool
    width: int
    height: int
    spp: int
    restir: bool
    seed: int

    @property
    def samples(self) -> int:
        return self.width * self.height * self.spp


def request_stream(count: int, pool_size: int = 16, rate: float = SERVE_RATE, seed: int = 0xA11) -> list[RequestSpec]:
    """The first `count` requests of the seeded Poisson stream (the stream is
    the same prefix whatever `count` is)."""
    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    for i in range(count):
        t += float(rng.exponential(1.0 / rate))
        scene = int(rng.integers(0, pool_size))
        w, h = SERVE_RESOLUTIONS[int(rng.integers(0, len(SERVE_RESOLUTIONS)))]
        spp = SERVE_SPP[int(rng.integers(0, len(SERVE_SPP)))]
        restir = bool(rng.random() < 0.5)
        out.append(RequestSpec(t, scene, w, h, spp, restir, 0x20000 + i))
    return out


def camera_path(camera: scenes.Camera, frames: int, seed: int = 0xC2, radius: float = 0.08) -> list:
    """A seeded smooth camera path: the eye moves on a wobbling arc of
    `radius` around its start (two seeded sinusoids per axis), looking at
    the point one unit ahead of the start camera."""
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.3, 1.0, (2, 3)) * radius
    freq = rng.uniform(0.5, 2.0, (2, 3))
    phase = rng.uniform(0.0, 2.0 * np.pi, (2, 3))
    target = camera.position.astype(np.float64) + camera.forward.astype(np.float64)
    vfov = float(np.degrees(2.0 * np.arctan(camera.tan_half_fov)))
    out = []
    for k in range(frames):
        t = k / max(frames - 1, 1) * 2.0 * np.pi
        off = (amp * np.sin(freq * t + phase)).sum(0)
        out.append(scenes.Camera.look_at(camera.position.astype(np.float64) + off, target, vfov))
    return out


def fifo_latencies(arrivals, durations) -> tuple[np.ndarray, float]:
    """Completion latencies of requests served one at a time in arrival
    order, each taking its measured duration; returns (latencies, makespan
    from the first arrival to the last completion)."""
    a = np.asarray(arrivals, np.float64)
    d = np.asarray(durations, np.float64)
    done = np.empty_like(a)
    free = -np.inf
    for i in range(len(a)):
        start = max(a[i], free)
        free = start + d[i]
        done[i] = free
    return done - a, float(done[-1] - a[0]) if len(a) else 0.0
