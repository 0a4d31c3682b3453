"""Host mirror of the wavefront runtime over the C ABI.

``CudaWavefrontRuntime`` follows the frame interface of ``Wave2Runtime``
(include/renderers/Wave2Runtime.hpp:95-131): ``SetScene`` once per scene,
``UpdateFrame`` + ``RecordFrame`` per frame, ``CollectCompletedFrame`` after
the frame's work completes.  The frame record is the reference's
``MegakernelFrameConstantsGpu`` (304 bytes) byte for byte.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .scenes import Camera, SceneData
from .traversal import Scene
from ._native import FrameTelemetry, RendererDesc, RendererTuning

FRAME_DTYPE = np.dtype([
    ("camera_position_tan_half_fov", "<f4", 4), ("camera_forward_aspect", "<f4", 4),
    ("camera_right_lens_radius", "<f4", 4), ("camera_up_exposure", "<f4", 4),
    ("image", "<u4", 4), ("trace", "<u4", 4), ("sampling", "<u4", 4), ("environment", "<u4", 4),
    ("distribution", "<u4", 4), ("russian_roulette", "<f4", 4), ("scene_center_radius", "<f4", 4),
    ("environment_to_world", "<f4", (3, 4)), ("world_to_environment", "<f4", (3, 4)),
    ("traversal", "<u4", 4), ("output", "<u4", 4)])
assert FRAME_DTYPE.itemsize == 304

ESTIMATOR_BSDF_ONLY, ESTIMATOR_NEE, ESTIMATOR_MIS, ESTIMATOR_RESTIR = 0, 1, 2, 3
SHADOW_PHYSICAL = 2
(FILM_MEAN, FILM_SAMPLE, FILM_CAMERA_EMISSION, FILM_DIRECT_DIFFUSE, FILM_DIRECT_SPECULAR,
 FILM_INDIRECT_DIFFUSE, FILM_INDIRECT_SPECULAR, FILM_PRIMARY_POSITION, FILM_PRIMARY_NORMAL,
 FILM_PRIMARY_ALBEDO, FILM_PRIMARY_IDENTITY) = range(11)
# Wave2Runtime's Russian-roulette / epsilon defaults (Wave2Runtime.cpp:1410).
DEFAULT_RR = (3.0, 0.05, 0.95, 1.0e-4)


def frame_constants(camera: Camera, width: int, height: int, sample_index: int, max_depth: int,
                    seed: int = 0x5EED, estimator: int = ESTIMATOR_MIS, light_selection: int = 0,
                    rr=DEFAULT_RR, stream_tag: int = 0, scene_radius: float = 1.0) -> np.ndarray:
    f = np.zeros(1, FRAME_DTYPE)
    f["camera_position_tan_half_fov"] = [*camera.position, camera.tan_half_fov]
    f["camera_forward_aspect"] = [*camera.forward, width / height]
    f["camera_right_lens_radius"] = [*camera.right, 0.0]
    f["camera_up_exposure"] = [*camera.up, 1.0]
    f["image"] = [width, height, sample_index, max_depth]
    f["sampling"] = [seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF, light_selection, estimator]
    f["environment"] = [0xFFFFFFFF, 0, 0, 0]
    f["russian_roulette"] = rr
    f["scene_center_radius"] = [0, 0, 0, scene_radius]
    f["traversal"] = [1, 0, 0, 0]
    f["output"] = [stream_tag, 0xFFFFFFFF, 0, SHADOW_PHYSICAL]
    return f


def camera_matrices(frame: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """re_camera_matrices: (view-projection, world-to-view), row-major 4x4
    float32, in the reconstruction module's conventions."""
    f = np.ascontiguousarray(frame, FRAME_DTYPE)
    vp = np.zeros((4, 4), np.float32)
    w2v = np.zeros((4, 4), np.float32)
    N.check(N.load().re_camera_matrices(N.ptr(f), N.ptr(vp), N.ptr(w2v)))
    return vp, w2v


def plan_launches(scene_slots, pixel_counts, launch_paths: int) -> tuple[np.ndarray, int]:
    """re_plan_launches: the launch index of every view (each scene's views
    cut into chunks of at most `launch_paths` paths, chunks placed first-fit
    into launches of at most `launch_paths` paths) and the launch count."""
    slots = np.ascontiguousarray(scene_slots, np.uint32)
    pixels = np.ascontiguousarray(pixel_counts, np.uint32)
    out = np.zeros(len(slots), np.uint32)
    n = C.c_uint32()
    N.check(N.load().re_plan_launches(N.ptr(slots), N.ptr(pixels), len(slots), launch_paths, N.ptr(out),
                                      C.byref(n)))
    return out, int(n.value)


@dataclass
class Telemetry:
    path_rays: int
    shadow_rays: int
    fatal_mask: int
    non_finite: int
    negative_pdf: int
    frames_accumulated: int
    active_per_bounce: list
    shadow_per_bounce: list
    gpu_ms: float
    total_path_rays: int
    total_shadow_rays: int


class Renderer:
    """One wavefront renderer (path state + queues + film resident in HBM)."""

    def __init__(self, max_width: int, max_height: int, max_depth: int = 8, device: int = 0):
        self.lib = N.load()
        h = C.c_void_p()
        N.check(self.lib.re_renderer_create(C.byref(RendererDesc(max_width, max_height, max_depth, device)),
                                            C.byref(h)))
        self.handle = h
        self.scene: Scene | None = None
        self.scene_data: SceneData | None = None

    def close(self):
        if self.handle:
            self.lib.re_renderer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_tuning(self, fuse: bool = False, graph: bool = True, blocks_per_sm: int = 0, block: int = 128,
                   shade_variant: int = 4, refill: int = 0, traversal: int = 3):
        self.tuning = dict(fuse=fuse, graph=graph, blocks_per_sm=blocks_per_sm, block=block,
                           shade_variant=shade_variant, refill=refill, traversal=traversal)
        N.check(self.lib.re_renderer_set_tuning(self.handle, C.byref(RendererTuning(
            block, blocks_per_sm, int(fuse), int(graph), shade_variant, refill, traversal))))

    def set_environment(self, texels: np.ndarray | None, slot: int = 0):
        """Equirectangular linear-RGBA environment map (height, width, 4) of a
        scene slot (re_renderer_set_environment); unbinds the slot first."""
        if getattr(self, "_slots", {}).get(slot) is not None or (slot == 0 and self.scene is not None):
            self.unbind_scene(slot)
            if slot == 0:
                self.scene = self.scene_data = None
        if texels is None:
            N.check(self.lib.re_renderer_set_environment(self.handle, slot, None, 0, 0))
            return
        t = np.ascontiguousarray(texels, np.float32)
        h, w = t.shape[:2]
        N.check(self.lib.re_renderer_set_environment(self.handle, slot, N.ptr(t), w, h))
        self._env_shape = getattr(self, "_env_shape", {})
        self._env_shape[slot] = (w, h)

    def environment_tables(self, slot: int = 0):
        """(row alias entries (h, 4), column alias entries (h * w, 4),
        integrated luminance); entries are (q, pmf, alias bits, item bits)."""
        w, h = self._env_shape[slot]
        rows = np.zeros((h, 4), np.float32)
        cols = np.zeros((h * w, 4), np.float32)
        integ = C.c_double(0.0)
        N.check(self.lib.re_renderer_environment_tables(self.handle, slot, N.ptr(rows), N.ptr(cols), C.byref(integ)))
        return rows, cols, integ.value

    def set_scene(self, scene: Scene, data: SceneData, light_selection: int = 0, scene_radius: float = 1.0):
        env = data.extra.get("environment") if data.extra else None
        if env is not None:
            self.set_environment(env, 0)
        self._mat = np.ascontiguousarray(data.materials)
        self._lights = np.ascontiguousarray(data.lights)
        self._fix = np.ascontiguousarray(data.fixture_triangles)
        N.check(self.lib.re_renderer_set_scene(
            self.handle, scene.handle, N.ptr(self._mat), len(self._mat),
            N.ptr(self._lights) if len(self._lights) else None, len(self._lights),
            N.ptr(self._fix) if len(self._fix) else None, len(self._fix), light_selection, scene_radius))
        self.scene = scene
        self.scene_data = data

    # -- batched views: many cameras / scenes in one launch --------------------
    def bind_scene(self, slot: int, scene: Scene, data: SceneData, light_selection: int = 0,
                   scene_radius: float = 1.0):
        """Binds a resident scene to a slot (re_renderer_bind_scene)."""
        env = data.extra.get("environment") if data.extra else None
        if env is not None:
            self.set_environment(env, slot)
        keep = (np.ascontiguousarray(data.materials), np.ascontiguousarray(data.lights),
                np.ascontiguousarray(data.fixture_triangles))
        mat, lights, fix = keep
        N.check(self.lib.re_renderer_bind_scene(
            self.handle, slot, scene.handle, N.ptr(mat), len(mat), N.ptr(lights) if len(lights) else None,
            len(lights), N.ptr(fix) if len(fix) else None, len(fix), light_selection, scene_radius))
        self._slots = getattr(self, "_slots", {})
        self._slots[slot] = (scene, data, keep)
        if slot == 0:
            self.scene, self.scene_data = scene, data

    def unbind_scene(self, slot: int):
        N.check(self.lib.re_renderer_unbind_scene(self.handle, slot))
        getattr(self, "_slots", {}).pop(slot, None)

    def render_views(self, views: list, stream: int | None = None):
        """One sample of every view; views are dicts with keys frame (frame
        constants), slot, offset, accumulate (bool) and key (int)."""
        self._vframes = [np.ascontiguousarray(v["frame"], FRAME_DTYPE) for v in views]
        arr = (N.ViewDesc * len(views))()
        for k, v in enumerate(views):
            arr[k] = N.ViewDesc(N.ptr(self._vframes[k]), v.get("slot", 0), v.get("offset", 0),
                                int(v.get("accumulate", False)), 0, v.get("key", k))
        self._vdesc = arr
        N.check(self.lib.re_renderer_render_views(self.handle, arr, len(views), stream))

    def read_view(self, plane: int, offset: int, pixels: int) -> np.ndarray:
        out = np.zeros((pixels, 4), np.float32)
        N.check(self.lib.re_renderer_read_view(self.handle, plane, offset, pixels, N.ptr(out), N.MEMORY_HOST, None))
        return out

    def export_reconstruction(self, current: np.ndarray, previous: np.ndarray | None = None, offset: int = 0,
                              slot: int = 0, gbuffer_ptr: int | None = None, signal_ptr: int | None = None,
                              stream: int | None = None):
        """re_renderer_export_reconstruction for the view rendered with frame
        constants `current` (motion to `previous`).  With device pointers
        the records are written there; otherwise returns host arrays
        (GBUFFER_DTYPE, SIGNAL_DTYPE)."""
        cur = np.ascontiguousarray(current, FRAME_DTYPE)
        prev = None if previous is None else np.ascontiguousarray(previous, FRAME_DTYPE)
        if gbuffer_ptr is not None:
            N.check(self.lib.re_renderer_export_reconstruction(self.handle, slot, offset, N.ptr(cur), N.ptr(prev),
                                                               gbuffer_ptr, signal_ptr, N.MEMORY_DEVICE, stream))
            return None
        n = int(cur["image"][0, 0]) * int(cur["image"][0, 1])
        gb = np.zeros(n, N.GBUFFER_DTYPE)
        sig = np.zeros(n, N.SIGNAL_DTYPE)
        N.check(self.lib.re_renderer_export_reconstruction(self.handle, slot, offset, N.ptr(cur), N.ptr(prev),
                                                           N.ptr(gb), N.ptr(sig), N.MEMORY_HOST, stream))
        return gb, sig

    def release_view(self, key: int):
        N.check(self.lib.re_renderer_release_view(self.handle, key))

    @property
    def capacity(self) -> int:
        c = C.c_uint32()
        N.check(self.lib.re_renderer_path_capacity(self.handle, C.byref(c)))
        return int(c.value)

    def render(self, frame: np.ndarray, accumulate: bool = True, stream: int | None = None):
        self._frame = np.ascontiguousarray(frame, FRAME_DTYPE)
        N.check(self.lib.re_renderer_render(self.handle, N.ptr(self._frame), int(accumulate), stream))

    def read_async(self, plane: int, out: np.ndarray, offset: int = 0, stream: int | None = None) -> None:
        """Starts reading `len(out)` pixels of a film plane into `out` (a
        (pixels, 4) float32 array, best in pinned memory) after the work
        queued on `stream`, without waiting (re_renderer_read_view_async);
        `out` must stay alive until wait_reads()."""
        assert out.dtype == np.float32 and out.ndim == 2 and out.shape[1] == 4 and out.flags["C_CONTIGUOUS"]
        N.check(self.lib.re_renderer_read_view_async(self.handle, plane, offset, len(out), out.ctypes.data, stream))

    def wait_reads(self) -> None:
        """Blocks until every read started by read_async has landed."""
        N.check(self.lib.re_renderer_wait_reads(self.handle))

    def restir_debug(self, mode: int, pixels: int) -> tuple[np.ndarray, np.ndarray]:
        """RestirDebugV3 of the last frame's published reservoirs
        (re_renderer_restir_debug): (records as (pixels, 16) uint32 --
        identity, generation, scalar bits, state -- and the (pixels, 4)
        float32 view of `mode`)."""
        rec = np.zeros((pixels, 16), np.uint32)
        img = np.zeros((pixels, 4), np.float32)
        N.check(self.lib.re_renderer_restir_debug(self.handle, mode, pixels, N.ptr(rec), N.ptr(img), N.MEMORY_HOST,
                                                  None))
        return rec, img

    def read(self, plane: int, pixels: int) -> np.ndarray:
        out = np.zeros((pixels, 4), np.float32)
        N.check(self.lib.re_renderer_read_film(self.handle, plane, N.ptr(out), pixels, N.MEMORY_HOST, None))
        return out

    def film_pointer(self, plane: int) -> int:
        p = C.c_void_p()
        N.check(self.lib.re_renderer_film_pointer(self.handle, plane, C.byref(p)))
        return p.value

    def profile(self, frame: np.ndarray) -> dict:
        """Per-stage times and traversal test counts of one frame (film untouched)."""
        self._pframe = np.ascontiguousarray(frame, FRAME_DTYPE)
        p = N.StageProfile()
        N.check(self.lib.re_renderer_profile(self.handle, N.ptr(self._pframe), C.byref(p)))
        depth = int(self._pframe["image"][0, 3])
        out = {"raygen_ms": p.raygen_ms, "resolve_ms": p.resolve_ms, "restir_ms": p.restir_ms}
        for name in ("intersect_ms", "shade_ms", "shadow_ms", "rays", "shadows", "intersect_node_tests",
                     "intersect_triangle_tests", "shadow_node_tests", "shadow_triangle_tests",
                     "intersect_node_bytes", "shadow_node_bytes"):
            out[name] = list(getattr(p, name))[:depth]
        return out

    # -- ReSTIR DI (frames rendered with estimator=ESTIMATOR_RESTIR_PRIMARY) --
    def set_restir(self, **kw) -> None:
        """re_renderer_set_restir over re_restir_default_config, fields as
        keywords (candidates, spatial_neighbors, max_m, max_history_age,
        temporal, neighbor_mode, disk_radius, normal_cos, relative_depth,
        position_distance, estimator: 0 biased, 1 reference correction)."""
        c = N.RestirConfig()
        N.check(self.lib.re_restir_default_config(C.byref(c)))
        for k, v in kw.items():
            if not hasattr(c, k):
                raise KeyError(k)
            setattr(c, k, v)
        N.check(self.lib.re_renderer_set_restir(self.handle, C.byref(c)))

    def restir_reset(self) -> None:
        N.check(self.lib.re_renderer_restir_reset(self.handle))

    def restir_statistics(self) -> dict:
        st = N.RestirStatistics()
        N.check(self.lib.re_renderer_restir_statistics(self.handle, C.byref(st)))
        return {name: getattr(st, name) for name, _ in N.RestirStatistics._fields_}

    def restir_read(self, plane: int, pixels: int) -> np.ndarray:
        """Copies a ReSTIR plane of the last frame: reservoirs as (pixels, 64)
        uint32 words, surfaces as (pixels, 24) words, direct as (2, pixels, 4)
        float32, reasons as (pixels,) uint32."""
        words = {N.RESTIR_PUBLISHED: 64, N.RESTIR_TEMPORAL: 64, N.RESTIR_SURFACES: 24, N.RESTIR_DIRECT: 8,
                 N.RESTIR_REASONS: 1}[plane]
        out = np.empty(pixels * words, np.uint32)
        N.check(self.lib.re_renderer_restir_read(self.handle, plane, N.ptr(out), out.nbytes, N.MEMORY_HOST, None))
        if plane == N.RESTIR_DIRECT:
            return out.view(np.float32).reshape(2, pixels, 4)
        if plane == N.RESTIR_REASONS:
            return out
        return out.reshape(pixels, words)

    def collect(self, check: bool = True) -> Telemetry:
        t = FrameTelemetry()
        code = self.lib.re_renderer_collect(self.handle, C.byref(t))
        if check:
            N.check(code)
        return Telemetry(t.path_rays, t.shadow_rays, t.fatal_mask, t.non_finite, t.negative_pdf,
                         t.frames_accumulated, list(t.active_per_bounce), list(t.shadow_per_bounce), t.gpu_ms,
                         t.total_path_rays, t.total_shadow_rays)


class CudaWavefrontRuntime:
    """Wave2Runtime-shaped frame interface for the cuda-wavefront architecture."""

    def __init__(self, max_width: int, max_height: int, max_depth: int = 8, device: int = 0):
        self.renderer = Renderer(max_width, max_height, max_depth, device)
        self.device = device
        self._frame = None
        self._scene = None

    def SetScene(self, data: SceneData, build_kind: int = N.BUILD_FLATTENED_SAH,  # noqa: N802
                 light_selection: int = 0, scene_radius: float = 1.0) -> None:
        self._scene = Scene(data.triangles, data.fingerprint, data.generation, build_kind, device=self.device)
        self.renderer.set_scene(self._scene, data, light_selection, scene_radius)

    def UpdateFrame(self, camera: Camera, width: int, height: int, sample_index: int, max_depth: int,  # noqa: N802
                    **kw) -> None:
        self._frame = frame_constants(camera, width, height, sample_index, max_depth, **kw)

    def RecordFrame(self, accumulate: bool = True, stream: int | None = None) -> None:  # noqa: N802
        self.renderer.render(self._frame, accumulate, stream)

    def CollectCompletedFrame(self) -> Telemetry:  # noqa: N802
        return self.renderer.collect()
