"""Render server: continuous batching of render requests (the C ABI's
re_server_*).  Scenes are registered once as host records; requests arrive
over time and are rendered one sample per launch together with every other
admitted request, against an HBM budget with least-recently-used scene
eviction."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .scenes import SceneData
from .wavefront import FRAME_DTYPE


@dataclass
class RequestStatus:
    state: int
    samples_done: int
    error: int
    arrival_time: float
    admit_time: float
    completion_time: float

    @property
    def latency(self) -> float:
        return self.completion_time - self.arrival_time


class RenderServer:
    def __init__(self, hbm_budget_bytes: int, path_capacity: int, max_depth: int = 8, device: int = 0,
                 max_batch_views: int = 256, build_kind: int = N.BUILD_LBVH, restir: bool = True,
                 launch_paths: int = 0, backfill_window: int = N.BACKFILL_DEFAULT, **restir_config):
        self.lib = N.load()
        rc = N.RestirConfig()
        N.check(self.lib.re_restir_default_config(C.byref(rc)))
        for k, v in restir_config.items():
            setattr(rc, k, v)
        desc = N.ServerDesc(hbm_budget_bytes, path_capacity, max_depth, device, max_batch_views, build_kind,
                            int(restir), rc, launch_paths, backfill_window)
        self.handle = C.c_void_p()
        N.check(self.lib.re_server_create(C.byref(desc), C.byref(self.handle)))
        self._pixels: dict[int, int] = {}

    def close(self):
        if self.handle:
            self.lib.re_server_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def clock(self) -> float:
        return float(self.lib.re_server_clock(self.handle))

    def register_scene(self, key: int, data: SceneData, light_selection: int = 0, scene_radius: float = 1.0):
        tri = np.ascontiguousarray(data.triangles, N.TRIANGLE_DTYPE)
        mat = np.ascontiguousarray(data.materials)
        lights = np.ascontiguousarray(data.lights)
        fix = np.ascontiguousarray(data.fixture_triangles)
        N.check(self.lib.re_server_register_scene(
            self.handle, key, N.ptr(tri), len(tri), N.ptr(mat), len(mat), N.ptr(lights) if len(lights) else None,
            len(lights), N.ptr(fix) if len(fix) else None, len(fix), light_selection, scene_radius))

    def submit(self, scene_key: int, frame: np.ndarray, spp: int, arrival_time: float = 0.0) -> int:
        fc = np.ascontiguousarray(frame, FRAME_DTYPE)
        req = N.RenderRequest()
        req.scene_key = scene_key
        C.memmove(req.frame, fc.ctypes.data, 304)
        req.spp = spp
        req.arrival_time = arrival_time
        rid = C.c_uint64()
        N.check(self.lib.re_server_submit(self.handle, C.byref(req), C.byref(rid)))
        self._pixels[rid.value] = int(fc["image"][0, 0]) * int(fc["image"][0, 1])
        return int(rid.value)

    def pump(self, max_steps: int = 1 << 30, max_wait: float = 0.0) -> int:
        steps = C.c_uint32()
        N.check(self.lib.re_server_pump(self.handle, max_steps, max_wait, C.byref(steps)))
        return int(steps.value)

    def drain(self):
        N.check(self.lib.re_server_drain(self.handle))

    def poll(self, rid: int) -> RequestStatus:
        st = N.RequestStatus()
        N.check(self.lib.re_server_poll(self.handle, rid, C.byref(st)))
        return RequestStatus(st.state, st.samples_done, st.error, st.arrival_time, st.admit_time,
                             st.completion_time)

    def result(self, rid: int) -> np.ndarray:
        n = self._pixels[rid]
        out = np.zeros((n, 4), np.float32)
        N.check(self.lib.re_server_read_result(self.handle, rid, N.ptr(out), n))
        return out

    def release(self, rid: int):
        N.check(self.lib.re_server_release(self.handle, rid))
        self._pixels.pop(rid, None)

    def stats(self) -> dict:
        st = N.ServerStats()
        N.check(self.lib.re_server_stats_get(self.handle, C.byref(st)))
        return {name: getattr(st, name) for name, _ in N.ServerStats._fields_}
