"""Host-side mirror of the reference traversal interface over the C ABI.

``CudaTraversalBackend`` mirrors ``IGpuTraversalBackend``
(include/rt/gpu/IGpuTraversalBackend.hpp:72-84): ``Descriptor``,
``BuildOrUpdateScene``, ``RecordTraceClosestBatch`` and ``RecordTraceAnyBatch``
return a :class:`GpuTraversalStatus` (code + message, truthy on success) with
the reference's status-code values.  Batch offsets are record indices, and a
batch whose scene fingerprint/generation does not match the resident scene is
rejected with ``MissingScene``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N


@dataclass
class GpuTraversalStatus:
    code: int = N.SUCCESS
    message: str = ""

    def __bool__(self) -> bool:
        return self.code == N.SUCCESS

    @property
    def name(self) -> str:
        return N.STATUS_NAMES.get(self.code, str(self.code))


@dataclass
class GpuTraversalBackendDescriptor:
    stable_token: str = "cuda-software-bvh"
    display_name: str = "CUDA sm_100a flattened BVH"
    supports_closest: bool = True
    supports_any: bool = True
    requires_acceleration_structure: bool = True


@dataclass
class GpuSceneBuildRequest:
    triangles: np.ndarray                  # TRIANGLE_DTYPE
    scene_fingerprint: int = 0
    scene_generation: int = 0
    topology_changed: bool = True
    build_kind: int = N.BUILD_FLATTENED_SAH
    sah_bins: int = 16
    max_leaf_size: int = 4
    nodes: np.ndarray | None = None        # optional caller-flattened NODE_DTYPE
    device: int = 0


@dataclass
class GpuTraceBatch:
    rays: np.ndarray                       # RAY_DTYPE (host) or device pointer (int)
    hits: np.ndarray                       # HIT_DTYPE (host) or device pointer (int)
    scene_fingerprint: int = 0
    ray_offset: int = 0
    hit_offset: int = 0
    ray_count: int = 0
    scene_generation: int = 0
    stream: int | None = None


def _status(code: int) -> GpuTraversalStatus:
    if code == N.SUCCESS:
        return GpuTraversalStatus()
    msg = N.load().re_last_error()
    return GpuTraversalStatus(code, msg.decode() if msg else "")


class Scene:
    """A resident scene (BVH + triangles in HBM)."""

    def __init__(self, triangles: np.ndarray, fingerprint: int, generation: int = 1,
                 build_kind: int = N.BUILD_FLATTENED_SAH, sah_bins: int = 16, max_leaf_size: int = 4,
                 nodes: np.ndarray | None = None, device: int = 0):
        lib = N.load()
        self._tri = np.ascontiguousarray(triangles, N.TRIANGLE_DTYPE)
        self._nodes = None if nodes is None else np.ascontiguousarray(nodes, N.NODE_DTYPE)
        desc = N.SceneDesc(N.ptr(self._tri), len(self._tri), N.ptr(self._nodes),
                           0 if self._nodes is None else len(self._nodes), build_kind, sah_bins,
                           max_leaf_size, fingerprint, generation, device)
        handle = C.c_void_p()
        N.check(lib.re_scene_create(C.byref(desc), C.byref(handle)))
        self.handle = handle
        self.fingerprint = fingerprint
        self.generation = generation

    @classmethod
    def from_device(cls, records_ptr: int, count: int, fingerprint: int, generation: int = 1,
                    device: int = 0) -> "Scene":
        """A GPU-LBVH scene from `count` CanonicalTraversalTriangle records in
        device memory (re_scene_create_from_device), e.g. the output of
        ingest.expand_canonical; the records are not kept."""
        self = cls.__new__(cls)
        self._tri = None
        self._nodes = None
        desc = N.SceneDesc(records_ptr, count, None, 0, N.BUILD_LBVH, 16, 4, fingerprint, generation, device)
        handle = C.c_void_p()
        N.check(N.load().re_scene_create_from_device(C.byref(desc), C.byref(handle)))
        self.handle = handle
        self.fingerprint = fingerprint
        self.generation = generation
        return self

    def set_alpha_masks(self, alpha: dict) -> None:
        """Coverage data of the scene's alpha-masked triangles
        (re_scene_set_alpha_masks): alpha = dict(materials = GpuMaterialV0
        records, atlas = (layers, height, width) float32 alpha, sampler_id)."""
        mats = np.ascontiguousarray(alpha.get("materials", np.zeros(0, N.MATERIAL_V0_DTYPE)), N.MATERIAL_V0_DTYPE)
        atlas = np.ascontiguousarray(alpha.get("atlas", np.zeros((0, 1, 1), np.float32)), np.float32)
        layers, h, w = atlas.shape
        self._alpha_keep = (mats, atlas)
        N.check(N.load().re_scene_set_alpha_masks(self.handle, N.ptr(mats) if len(mats) else None, len(mats),
                                                  N.ptr(atlas) if atlas.size else None, w, h, layers,
                                                  int(alpha.get("sampler_id", 0xFFFFFFFF))))

    def close(self) -> None:
        if self.handle:
            N.load().re_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> N.SceneInfo:
        info = N.SceneInfo()
        N.check(N.load().re_scene_info_get(self.handle, C.byref(info)))
        return info

    def export_flat(self) -> tuple[np.ndarray, np.ndarray]:
        info = self.info()
        nodes = np.zeros(info.node_count, N.NODE_DTYPE)
        order = np.zeros(info.triangle_count, np.uint32)
        N.check(N.load().re_scene_export_flat(self.handle, N.ptr(nodes), len(nodes), N.ptr(order), len(order)))
        return nodes, order

    def _batch(self, rays, hits, memory, stream, count=None, ray_offset=0, hit_offset=0):
        if memory == N.MEMORY_HOST:
            count = len(rays) - ray_offset if count is None else count
            return N.TraceBatch(N.ptr(rays), N.ptr(hits), ray_offset, hit_offset, count, memory,
                                self.fingerprint, self.generation, 0, stream)
        return N.TraceBatch(rays, hits, ray_offset, hit_offset, count, memory, self.fingerprint,
                            self.generation, 0, stream)

    def trace(self, rays: np.ndarray, any_hit: bool = False, counters: bool = False):
        """Traces a host RAY_DTYPE array; returns the HIT_DTYPE array (and
        counters when requested)."""
        rays = np.ascontiguousarray(rays, N.RAY_DTYPE)
        hits = np.zeros(len(rays), N.HIT_DTYPE)
        b = self._batch(rays, hits, N.MEMORY_HOST, None)
        lib = N.load()
        if counters:
            c = N.TraversalCounters()
            N.check(lib.re_trace_counted(self.handle, C.byref(b), int(any_hit), C.byref(c)))
            return hits, {f: getattr(c, f) for f, _ in N.TraversalCounters._fields_}
        fn = lib.re_trace_any if any_hit else lib.re_trace_closest
        N.check(fn(self.handle, C.byref(b)))
        return hits

    def trace_device(self, rays_ptr: int, hits_ptr: int, count: int, any_hit: bool = False,
                     stream: int | None = None) -> None:
        b = self._batch(rays_ptr, hits_ptr, N.MEMORY_DEVICE, stream, count)
        lib = N.load()
        N.check((lib.re_trace_any if any_hit else lib.re_trace_closest)(self.handle, C.byref(b)))


class CudaTraversalBackend:
    """IGpuTraversalBackend over the sm_100a kernels."""

    def __init__(self):
        N.load()
        self.scene: Scene | None = None

    def Descriptor(self) -> GpuTraversalBackendDescriptor:  # noqa: N802 (reference naming)
        return GpuTraversalBackendDescriptor()

    def BuildOrUpdateScene(self, request: GpuSceneBuildRequest) -> GpuTraversalStatus:  # noqa: N802
        if request.scene_fingerprint == 0 or request.scene_generation == 0:
            return GpuTraversalStatus(N.INVALID_ARGUMENT, "scene fingerprint and generation must be non-zero")
        if (self.scene is not None and not request.topology_changed
                and self.scene.fingerprint == request.scene_fingerprint
                and self.scene.generation == request.scene_generation):
            return GpuTraversalStatus()
        try:
            new = Scene(request.triangles, request.scene_fingerprint, request.scene_generation,
                        request.build_kind, request.sah_bins, request.max_leaf_size, request.nodes,
                        request.device)
        except N.NativeError as e:
            return GpuTraversalStatus(e.code, str(e))
        if self.scene is not None:
            self.scene.close()
        self.scene = new
        return GpuTraversalStatus()

    def _record(self, batch: GpuTraceBatch, any_hit: bool) -> GpuTraversalStatus:
        if self.scene is None:
            return GpuTraversalStatus(N.MISSING_SCENE, "no scene has been built")
        lib = N.load()
        host = isinstance(batch.rays, np.ndarray)
        if host:
            if batch.ray_offset + batch.ray_count > len(batch.rays) or \
                    batch.hit_offset + batch.ray_count > len(batch.hits):
                return GpuTraversalStatus(N.INVALID_ARGUMENT, "batch range exceeds the ray/hit buffers")
            b = N.TraceBatch(N.ptr(batch.rays), N.ptr(batch.hits), batch.ray_offset, batch.hit_offset,
                             batch.ray_count, N.MEMORY_HOST, batch.scene_fingerprint, batch.scene_generation, 0,
                             batch.stream)
        else:
            b = N.TraceBatch(batch.rays, batch.hits, batch.ray_offset, batch.hit_offset, batch.ray_count,
                             N.MEMORY_DEVICE, batch.scene_fingerprint, batch.scene_generation, 0, batch.stream)
        fn = lib.re_trace_any if any_hit else lib.re_trace_closest
        return _status(fn(self.scene.handle, C.byref(b)))

    def RecordTraceClosestBatch(self, batch: GpuTraceBatch) -> GpuTraversalStatus:  # noqa: N802
        return self._record(batch, False)

    def RecordTraceAnyBatch(self, batch: GpuTraceBatch) -> GpuTraversalStatus:  # noqa: N802
        return self._record(batch, True)
