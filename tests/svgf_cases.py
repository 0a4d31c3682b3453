"""Inputs for the SVGF parity tests: the scenarios of the reference's L8
tests (reconstruction/tests/ReconstructionTests.cpp:52-77, 222-407) and
seeded multi-frame sequences with camera motion, disocclusion, invalid and
non-finite pixels, resets and resolution changes."""
from __future__ import annotations

import numpy as np

from renderingengine_b200 import _native as N

GB = N.GBUFFER_DTYPE
SIG = N.SIGNAL_DTYPE
VALID = N.GBUFFER_VALID | N.GBUFFER_MOTION_VALID


def config(**kw) -> N.SvgfConfig:
    """re_svgf_config with the reference defaults (Types.hpp:164-202)."""
    c = N.SvgfConfig(0.02, 0.01, 0.9063078, 1, 1, 32, 0.05, 0.10, 4, 3, 1.0e-6, 4, 1.0, 64.0, 4.0, 1.0e-3, 1)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def valid_gbuffer(h: int, w: int, object_id: int = 7) -> np.ndarray:
    """ValidGBuffer (ReconstructionTests.cpp:46-58) over an h x w image."""
    g = np.zeros((h, w), GB)
    g["linear_depth"] = 5.0
    g["world_normal"] = (0.0, 0.0, 1.0)
    g["diffuse_albedo"] = 1.0
    g["specular_albedo"] = 1.0
    g["expected_previous_linear_depth"] = 5.0
    g["material_id"] = 3
    g["object_id"] = object_id
    g["flags"] = VALID
    return g


def uniform_signal(h: int, w: int, value: float) -> np.ndarray:
    s = np.zeros((h, w), SIG)
    s["diffuse"] = value
    return s


def checkerboard(n: int = 16):
    """TestVarianceBootstrapAndDenoisingMetric inputs: 0.5 / 1.5 diffuse."""
    g = valid_gbuffer(n, n)
    s = np.zeros((n, n), SIG)
    yy, xx = np.mgrid[0:n, 0:n]
    s["diffuse"] = np.where(((xx + yy) & 1) == 0, 0.5, 1.5).astype(np.float32)[..., None]
    return g, s


def sequence(w: int, h: int, frames: int, seed: int, hostile: bool = True):
    """Seeded frames [(gbuffer, signal, frame_index, reset_trigger)].

    A handful of objects (distinct object / material IDs, tilted depth
    planes, varied normals) under a camera that pans by a fractional number
    of pixels per frame, one object moving on its own; a fraction of pixels
    invalid, motion-invalid or (with `hostile`) non-finite; noisy diffuse and
    specular signals over varied albedos.  Frame indices skip once (history
    unavailable) and one frame carries a camera-cut trigger."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    n_obj = 5
    cx = rng.uniform(0, w, n_obj)
    cy = rng.uniform(0, h, n_obj)
    rad = rng.uniform(0.15, 0.45, n_obj) * min(w, h)
    base_depth = rng.uniform(1.0, 40.0, n_obj)
    slope = rng.uniform(-0.05, 0.05, (n_obj, 2))
    nrm = rng.normal(size=(n_obj, 3)).astype(np.float32)
    nrm[:, 2] = np.abs(nrm[:, 2]) + 1.0
    dalb = rng.uniform(0.0, 1.2, (n_obj, 3)).astype(np.float32)
    salb = rng.uniform(0.0, 1.0, (n_obj, 3)).astype(np.float32)
    mats = rng.integers(0, 3, n_obj)
    pan = rng.uniform(-1.5, 1.5, 2)
    own = rng.uniform(-2.0, 2.0, 2)
    out = []
    frame_index = int(rng.integers(0, 3))
    for f in range(frames):
        shift = pan * f
        ids = np.full((h, w), 0xFFFFFFFF, np.uint32)
        depth = np.full((h, w), 100.0, np.float32)
        obj = np.full((h, w), -1, np.int64)
        for k in range(n_obj):
            ox, oy = cx[k] + shift[0], cy[k] + shift[1]
            if k == 0:
                ox += own[0] * f
                oy += own[1] * f
            inside = (xx - ox) ** 2 + (yy - oy) ** 2 < rad[k] ** 2
            d = base_depth[k] + slope[k, 0] * (xx - ox) + slope[k, 1] * (yy - oy)
            closer = inside & (d < depth)
            depth[closer] = d[closer]
            obj[closer] = k
        g = np.zeros((h, w), GB)
        hit = obj >= 0
        k = np.where(hit, obj, 0)
        g["linear_depth"] = np.where(hit, depth, 0.0)
        jitter = rng.normal(scale=0.02, size=(h, w, 3)).astype(np.float32)
        g["world_normal"] = np.where(hit[..., None], nrm[k] + jitter, (0.0, 0.0, 1.0))
        g["diffuse_albedo"] = np.where(hit[..., None], dalb[k], 0.0)
        g["specular_albedo"] = np.where(hit[..., None], salb[k], 0.0)
        g["material_id"] = np.where(hit, mats[k], 0xFFFFFFFF)
        g["object_id"] = np.where(hit, k + 10, 0xFFFFFFFF)
        mv = np.empty((h, w, 2), np.float32)
        mv[..., 0] = -pan[0] / w
        mv[..., 1] = -pan[1] / h
        mv[obj == 0, 0] -= own[0] / w
        mv[obj == 0, 1] -= own[1] / h
        g["motion"] = mv
        g["expected_previous_linear_depth"] = g["linear_depth"] * np.float32(1.0 + rng.uniform(-0.01, 0.01))
        flags = np.where(hit, VALID, 0).astype(np.uint32)
        flags[rng.random((h, w)) < 0.01] &= ~np.uint32(N.GBUFFER_MOTION_VALID)
        flags[rng.random((h, w)) < 0.01] = 0
        g["flags"] = flags
        s = np.zeros((h, w), SIG)
        noise = rng.exponential(1.0, (h, w, 3)).astype(np.float32)
        s["diffuse"] = g["diffuse_albedo"] * noise * np.float32(0.8)
        s["specular"] = g["specular_albedo"] * rng.exponential(0.3, (h, w, 3)).astype(np.float32)
        if hostile:
            bad = rng.random((h, w))
            s["diffuse"][bad < 0.003] = np.nan
            s["specular"][(bad >= 0.003) & (bad < 0.005)] = np.inf
            s["diffuse"][(bad >= 0.005) & (bad < 0.006)] = 3.0e38
            g["linear_depth"][(bad >= 0.006) & (bad < 0.007)] = np.nan
            g["world_normal"][(bad >= 0.007) & (bad < 0.008)] = 0.0
            g["expected_previous_linear_depth"][(bad >= 0.008) & (bad < 0.009)] = -1.0
            g["diffuse_albedo"][(bad >= 0.009) & (bad < 0.010)] = np.nan
            g["motion"][(bad >= 0.010) & (bad < 0.011)] = np.nan
        trigger = 0
        if f == frames // 2:
            trigger = 1  # CameraCut
        out.append((g, s, frame_index, trigger))
        frame_index += 2 if f == 1 else 1  # one skipped index: no history
    return out


def bits(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a).view(np.uint32)
