"""SVGF / A-Trous reconstruction on the GPU, mirroring the reference's
``rendering::reconstruction`` interface (reconstruction/include/reconstruction/
Svgf.hpp:30-75, Types.hpp:100-202): ``SvgfReconstruction`` with ``Process``,
``SelectOutput``, ``SetConfig`` and ``Reset``; ``ComputeRmse`` /
``ComputePsnr``.  Everything runs through the C ABI of ``libre_b200.so``;
there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import enum
import math
from dataclasses import dataclass, fields

import numpy as np

from . import _native as N

GBUFFER_DTYPE = N.GBUFFER_DTYPE
SIGNAL_DTYPE = N.SIGNAL_DTYPE


class ResetTrigger(enum.IntFlag):
    """ResetTrigger (Types.hpp:130-140)."""
    NONE = 0
    CAMERA_CUT = 1 << 0
    FIELD_OF_VIEW = 1 << 1
    RESOLUTION = 1 << 2
    SCENE = 1 << 3
    BACKEND = 1 << 4
    TRANSPORT = 1 << 5
    RECONSTRUCTION_PARAMETERS = 1 << 6
    SHADER_RELOAD = 1 << 7


class RejectReason(enum.IntFlag):
    """RejectReason (Types.hpp:100-113)."""
    NONE = 0
    NO_HISTORY = 1 << 0
    RESET = 1 << 1
    SCREEN_BOUNDS = 1 << 2
    INVALID_CURRENT = 1 << 3
    INVALID_HISTORY = 1 << 4
    NON_FINITE = 1 << 5
    DEPTH = 1 << 6
    NORMAL = 1 << 7
    MATERIAL_ID = 1 << 8
    OBJECT_ID = 1 << 9
    INVALID_MOTION = 1 << 10


class ReconstructionOutput(enum.IntEnum):
    """ReconstructionOutput (Types.hpp:155-166)."""
    RAW = 0
    TEMPORAL = 1
    ATROUS = 2
    SVGF = 3
    MOTION = 4
    HISTORY_LENGTH = 5
    MOMENTS = 6
    VARIANCE = 7
    HISTORY_ACCEPTANCE = 8
    REJECT_REASONS = 9


def requires_temporal_reset(trigger: int) -> bool:
    """RequiresTemporalReset (Types.hpp:151-153)."""
    return int(trigger) != 0


@dataclass
class SvgfConfig:
    """SvgfConfig with its Validation / Temporal / Variance / ATrous parts
    flattened (Types.hpp:164-202); the defaults are the reference's."""
    relative_depth_threshold: float = 0.02
    absolute_depth_threshold: float = 0.01
    normal_cosine_threshold: float = 0.9063078  # cos(25 degrees)
    require_material_id: bool = True
    require_object_id: bool = True
    max_history_length: int = 32
    minimum_color_alpha: float = 0.05
    minimum_moments_alpha: float = 0.10
    short_history_length: int = 4
    spatial_radius: int = 3
    minimum_variance: float = 1.0e-6
    atrous_iterations: int = 4
    phi_depth: float = 1.0
    phi_normal: float = 64.0
    phi_luminance: float = 4.0
    minimum_albedo: float = 1.0e-3
    demodulate_specular: bool = True

    def to_native(self) -> N.SvgfConfig:
        c = N.SvgfConfig()
        for f in fields(self):
            setattr(c, f.name, getattr(self, f.name))
        return c

    @classmethod
    def from_native(cls, c: N.SvgfConfig) -> "SvgfConfig":
        out = cls()
        for f in fields(cls):
            v = getattr(c, f.name)
            setattr(out, f.name, bool(v) if f.type in ("bool", bool) else v)
        return out


PLANE_RAW, PLANE_TEMPORAL, PLANE_ATROUS, PLANE_SVGF = 0, 1, 2, 3
PLANE_HISTORY_LENGTH, PLANE_MOMENTS, PLANE_VARIANCE, PLANE_ACCEPTED, PLANE_REJECT = 4, 5, 6, 7, 8
_PLANE_LAYOUT = {
    PLANE_RAW: (SIGNAL_DTYPE, ()), PLANE_TEMPORAL: (SIGNAL_DTYPE, ()), PLANE_ATROUS: (SIGNAL_DTYPE, ()),
    PLANE_SVGF: (SIGNAL_DTYPE, ()), PLANE_HISTORY_LENGTH: (np.uint32, ()), PLANE_MOMENTS: (np.float32, (2,)),
    PLANE_VARIANCE: (np.float32, ()), PLANE_ACCEPTED: (np.uint32, ()), PLANE_REJECT: (np.uint32, ()),
}


@dataclass
class ReconstructionFrame:
    """ReconstructionFrame (Svgf.hpp:19-29) as (height, width) host arrays."""
    raw: np.ndarray
    temporal: np.ndarray
    atrous: np.ndarray
    svgf: np.ndarray
    history_length: np.ndarray
    moments: np.ndarray
    variance: np.ndarray
    accepted_history: np.ndarray
    reject_reasons: np.ndarray


class SvgfReconstruction:
    """SvgfReconstruction (Svgf.hpp:52-75) with its history ping-pong
    resident in HBM.  ``process`` takes host numpy arrays (GBUFFER_DTYPE,
    SIGNAL_DTYPE, shape (height, width)) or, through ``process_device``,
    device pointers."""

    def __init__(self, width: int, height: int, frames_in_flight: int = 2, config: SvgfConfig | None = None,
                 device: int = 0):
        self._lib = N.load()
        self._h = C.c_void_p()
        cfg = (config or SvgfConfig()).to_native()
        N.check(self._lib.re_svgf_create(width, height, frames_in_flight, C.byref(cfg), device, C.byref(self._h)))
        self.width, self.height = width, height

    def close(self) -> None:
        if self._h:
            self._lib.re_svgf_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def config(self) -> SvgfConfig:
        c = N.SvgfConfig()
        N.check(self._lib.re_svgf_get_config(self._h, C.byref(c)))
        return SvgfConfig.from_native(c)

    def set_config(self, config: SvgfConfig) -> None:
        c = config.to_native()
        N.check(self._lib.re_svgf_set_config(self._h, C.byref(c)))

    def reset(self, width: int, height: int) -> None:
        N.check(self._lib.re_svgf_reset(self._h, width, height))

    def process(self, gbuffer: np.ndarray, raw_signal: np.ndarray, frame_index: int,
                reset_trigger: int = 0, read: bool = True) -> ReconstructionFrame | None:
        gb = np.ascontiguousarray(gbuffer, GBUFFER_DTYPE)
        sig = np.ascontiguousarray(raw_signal, SIGNAL_DTYPE)
        if gb.shape != sig.shape or gb.ndim != 2:
            raise ValueError("GBuffer and raw signal extents must match")
        h, w = gb.shape
        inp = N.SvgfFrameInputs(N.ptr(gb), N.ptr(sig), w, h, N.MEMORY_HOST, int(reset_trigger), frame_index)
        N.check(self._lib.re_svgf_process(self._h, C.byref(inp), None))
        self.width, self.height = w, h
        return self.frame() if read else None

    def process_device(self, gbuffer_ptr: int, signal_ptr: int, width: int, height: int, frame_index: int,
                       reset_trigger: int = 0, stream: int | None = None) -> None:
        inp = N.SvgfFrameInputs(gbuffer_ptr, signal_ptr, width, height, N.MEMORY_DEVICE, int(reset_trigger),
                                frame_index)
        N.check(self._lib.re_svgf_process(self._h, C.byref(inp), stream))
        self.width, self.height = width, height

    def read(self, plane: int) -> np.ndarray:
        dtype, tail = _PLANE_LAYOUT[plane]
        out = np.empty((self.height, self.width) + tail, dtype)
        N.check(self._lib.re_svgf_read(self._h, plane, N.ptr(out), out.nbytes, N.MEMORY_HOST, None))
        return out

    def plane_pointer(self, plane: int) -> int:
        p = C.c_void_p()
        N.check(self._lib.re_svgf_plane_pointer(self._h, plane, C.byref(p)))
        return int(p.value)

    def frame(self) -> ReconstructionFrame:
        return ReconstructionFrame(
            raw=self.read(PLANE_RAW), temporal=self.read(PLANE_TEMPORAL), atrous=self.read(PLANE_ATROUS),
            svgf=self.read(PLANE_SVGF), history_length=self.read(PLANE_HISTORY_LENGTH),
            moments=self.read(PLANE_MOMENTS), variance=self.read(PLANE_VARIANCE),
            accepted_history=self.read(PLANE_ACCEPTED), reject_reasons=self.read(PLANE_REJECT))

    def select_output(self, output: int, gbuffer: np.ndarray | None = None) -> np.ndarray:
        """SelectOutput (Svgf.cpp:754-822) of the last processed frame as a
        (height, width, 3) float32 image."""
        gb = None if gbuffer is None else np.ascontiguousarray(gbuffer, GBUFFER_DTYPE)
        out = np.empty((self.height, self.width, 3), np.float32)
        N.check(self._lib.re_svgf_select_output(self._h, N.ptr(gb), N.MEMORY_HOST, int(output), N.ptr(out),
                                                N.MEMORY_HOST, None))
        return out


def compute_rmse(candidate: np.ndarray, reference: np.ndarray) -> float:
    """ComputeRmse (Svgf.cpp:824-833) on the GPU; (h, w, 3) host images."""
    import torch

    a = torch.from_numpy(np.ascontiguousarray(candidate, np.float32)).cuda()
    b = torch.from_numpy(np.ascontiguousarray(reference, np.float32)).cuda()
    if a.shape != b.shape:
        raise ValueError("RMSE images must have matching extents")
    out = C.c_float()
    N.check(N.load().re_image_rmse(a.data_ptr(), b.data_ptr(), a.numel() // 3, C.byref(out), None))
    return float(out.value)


def compute_psnr(candidate: np.ndarray, reference: np.ndarray, peak: float = 1.0) -> float:
    """ComputePsnr (Svgf.cpp:835-841)."""
    if not peak > 0.0:
        raise ValueError("PSNR peak value must be positive")
    rmse = compute_rmse(candidate, reference)
    if rmse <= np.finfo(np.float32).eps:
        return math.inf
    return float(np.float32(20.0) * np.float32(math.log10(np.float32(peak) / np.float32(rmse))))
