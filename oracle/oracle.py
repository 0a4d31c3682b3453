"""TEST INFRASTRUCTURE ONLY -- ctypes access to the CPU oracles.

Two libraries:
  * ``oracle/_build/liboracle.so`` -- our CPU restatement of the hot path
    (``oracle_*.cpp``), each function citing the reference file:line it follows.
  * ``oracle/_ref/libref_oracle.so`` -- the reference's own CPU sources compiled
    unmodified with a thin shim (``ref_shim.cpp``).  Built where the reference
    tree exists; the built file travels with the repository snapshot.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
arm may import this module.  The product library never links or loads it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "_build" / "liboracle.so"
REF_LIB = HERE / "_ref" / "libref_oracle.so"

_P = C.c_void_p
_U32 = C.c_uint32

_ORACLE_SIGS = {
    "oracle_trace": (None, [_P, _U32, _P, _P, _P, _U32, _U32, _U32, _U32, _P, _P, _P, _P, _P]),
    "oracle_render": (None, [_P, _U32, _P, _P, _P, _P, _P, _P, _U32, _P, _U32, _P, _U32, _U32, C.c_float, _P,
                             _P, _U32, _U32, _P, _P]),
    "oracle_render_env": (None, [_P, _U32, _P, _P, _P, _P, _P, _P, _U32, _P, _U32, _P, _U32, _U32, C.c_float, _P,
                                 _P, _U32, _U32, _P, _P, _P, _U32, _U32, _P]),
    "oracle_trace_alpha": (None, [_P, _U32, _P, _P, _P, _U32, _U32, _U32, _U32, _P, _P, _P, _P, _P, _P]),
    "oracle_environment_tables": (None, [_P, _U32, _U32, _P, _P, _P]),
    "oracle_counter_random": (C.c_float, [_U32, _U32, _U32, _U32, _U32, _U32]),
    "oracle_light_distribution": (C.c_int, [_P, _U32, _U32, C.c_float, _P]),
    "oracle_svgf_create": (_P, [_U32, _U32, _U32, _P]),
    "oracle_svgf_destroy": (None, [_P]),
    "oracle_svgf_set_config": (C.c_int, [_P, _P]),
    "oracle_svgf_process": (C.c_int, [_P, _P, _P, _U32, _U32, C.c_uint64, _U32, _P]),
    "oracle_image_rmse": (C.c_float, [_P, _P, C.c_uint64]),
    "oracle_motion_vector": (None, [_P, _P, _P, _P, _P, _P, _P]),
    "oracle_restir_ris": (C.c_int, [_P, _P, _U32, _U32, _P, _P]),
    "oracle_restir_spatial_gate": (None, [_P, _P, _P, _U32, _P, _P]),
    "oracle_restir_temporal_gate": (None, [_P, _P, _P, _P, _P, _U32, _P, _P]),
    "oracle_bsdf_probe": (None, [_P, _U32, _P]),
    "oracle_bsdf_probe64": (None, [_P, _U32, _P]),
    "oracle_ggx_vndf": (None, [_P, _P, _P, _U32, _P]),
    "oracle_restir_frame": (None, [_P, _U32, _P, _P, _P, _U32, _P, _U32, _U32, C.c_float, _P, _P, _P, _P, _P, _P,
                                   _P, _P, _P, _P, _U32]),
}

# Frame record of oracle_render (oracle_pbr.cpp, struct Frame).
FRAME_DTYPE = np.dtype([("cam_pos", "<f4", 3), ("tan_half_fov", "<f4"), ("fwd", "<f4", 3), ("aspect", "<f4"),
                        ("right", "<f4", 3), ("pad0", "<f4"), ("up", "<f4", 3), ("pad1", "<f4"),
                        ("width", "<u4"), ("height", "<u4"), ("sample", "<u4"), ("max_depth", "<u4"),
                        ("seed_lo", "<u4"), ("seed_hi", "<u4"), ("estimator", "<u4"), ("stream", "<u4"),
                        ("rr_start", "<f4"), ("rr_min", "<f4"), ("rr_max", "<f4"), ("eps", "<f4"),
                        ("env_xf", "<f4", 24)])
PLANES = ("sample", "camera_emission", "direct_diffuse", "direct_specular", "indirect_diffuse",
          "indirect_specular", "primary_position", "primary_normal")
_REF_SIGS = {
    "ref_sah_build": (C.c_int, [_P, _P, _U32, _U32, _P, _U32, _P, _P, _P]),
    "ref_trace": (None, [_P, _U32, _P, _P, _U32, _P, _U32, _U32, _U32, _U32, _P, _P]),
    "ref_lbvh_build": (C.c_int, [_P, _P, _U32, _P, _U32, _P, _P, _P, _P]),
    "ref_canonical_expand": (C.c_int, [_P, _U32, _P, _U32, _P, _U32, _P, _U32, _P, _U32, _P, _U32, C.c_char_p,
                                       _U32]),
    "ref_cornell": (C.c_double, [_U32, _U32, _U32, _U32, C.c_uint64, _U32, _P, _P]),
    "ref_counter_random": (C.c_float, [_U32, _U32, _U32, _U32, C.c_uint64]),
    "ref_philox": (None, [_P, _P, _P]),
    "ref_alias_table": (C.c_int, [_P, _U32, _P]),
    "ref_light_distribution": (C.c_int, [_P, _U32, _U32, C.c_float, _P, _P]),
    "ref_l3_parity_corpus": (None, [_U32, _P, _P, _P, _P, _P]),
    "ref_svgf_create": (_P, [_U32, _U32, _U32, _P]),
    "ref_svgf_destroy": (None, [_P]),
    "ref_svgf_set_config": (C.c_int, [_P, _P]),
    "ref_svgf_process": (C.c_int, [_P, _P, _P, _U32, _U32, C.c_uint64, _U32, _P]),
    "ref_svgf_select": (C.c_int, [_P, _P, _U32, _U32, _U32, _P]),
    "ref_image_rmse": (C.c_float, [_P, _P, _U32, _U32]),
    "ref_image_psnr": (C.c_float, [_P, _P, _U32, _U32, C.c_float]),
    "ref_motion_vector": (None, [_P, _P, _P, _P, _P, _P, _P]),
    "ref_restir_ris": (C.c_int, [_P, _P, _U32, _U32, _P, _P]),
    "ref_restir_validate_spatial": (None, [_P, _P, _P, _U32, _P, _U32, _P]),
    "ref_restir_validate_temporal": (None, [_P, _P, _P, _P, _U32, _P, _U32, _P]),
    "ref_bsdf_probe": (None, [_P, _U32, _P]),
    "ref_env_distribution": (C.c_int, [_U32, _U32, _P, _P, _P, _P, _P]),
    "ref_light_distribution_env": (C.c_int, [_P, _U32, _U32, C.c_float, C.c_double, _P, _P]),
    "ref_ggx_vndf": (None, [_P, _P, _P, _U32, _P]),
}

_oracle = None
_ref = None


def reference_root() -> Path | None:
    """The reference tree to compile _ref from: $RE_REFERENCE_ROOT, else the
    container's read-only checkout when it exists (GPU machines have none and
    use the prebuilt library)."""
    env = os.environ.get("RE_REFERENCE_ROOT")
    for cand in ([Path(env)] if env else []) + [Path("/root/reference/RenderingEngine")]:
        if cand.is_dir():
            return cand
    return None


def build() -> None:
    """Compiles the oracle restatement and, when the reference tree is present, _ref."""
    ref = reference_root()
    subprocess.run(["make", "-s", "-C", str(HERE), "all"] + ([f"REF={ref}"] if ref else []), check=True)


def _bind(path: Path, sigs: dict) -> C.CDLL:
    lib = C.CDLL(str(path))
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def oracle_lib() -> C.CDLL:
    global _oracle
    if _oracle is None:
        if not ORACLE_LIB.exists():
            build()
        _oracle = _bind(ORACLE_LIB, _ORACLE_SIGS)
    return _oracle


def ref_available() -> bool:
    return REF_LIB.exists()


def ref_lib() -> C.CDLL:
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            raise FileNotFoundError(f"{REF_LIB} was not built (reference tree absent)")
        _ref = _bind(REF_LIB, _REF_SIGS)
    return _ref


def _p(a):
    return None if a is None else a.ctypes.data


# ---------------------------------------------------------------------------
# Traversal
# ---------------------------------------------------------------------------
class _AlphaData(C.Structure):
    _fields_ = [("tc", _P), ("materials", _P), ("atlas", _P), ("material_count", _U32), ("width", _U32),
                ("height", _U32), ("layers", _U32), ("sampler_id", _U32)]


def alpha_data(leaf_triangles: np.ndarray, alpha: dict | None):
    """Oracle alpha-mask data for leaf-ordered CanonicalTraversalTriangle
    records and a scene's alpha description (dict: materials = GpuMaterialV0
    records, atlas = (layers, h, w) float32, sampler_id); None when no
    triangle is masked.  Returns (struct, keep-alive arrays)."""
    masked = ((leaf_triangles["metadata"][:, 0] & 2) != 0) | ((leaf_triangles["metadata"][:, 1] & 2) != 0)
    if not masked.any():
        return None, ()
    n = len(leaf_triangles)
    tc = np.zeros((n, 8), np.float32)
    tc[:, 0:2] = leaf_triangles["texcoords"][:, 0, :2]
    tc[:, 2:4] = leaf_triangles["texcoords"][:, 1, :2]
    tc[:, 4:6] = leaf_triangles["texcoords"][:, 2, :2]
    tc[:, 6] = leaf_triangles["identity"][:, 3].view(np.float32)
    a = alpha or {}
    mats_in = a.get("materials")
    nm = 0 if mats_in is None else len(mats_in)
    mats = np.zeros((max(nm, 1), 4), np.float32)
    if nm:
        mats[:nm, 0] = mats_in["base_color_factor"][:, 3]
        mats[:nm, 1] = mats_in["surface_params"][:, 3]
        mats[:nm, 2] = mats_in["texture_image_indices"][:, 0].view(np.float32)
        mats[:nm, 3] = mats_in["texture_sampler_indices"][:, 0].view(np.float32)
    atlas = np.ascontiguousarray(a.get("atlas", np.zeros((0, 1, 1), np.float32)), np.float32)
    layers, h, w = atlas.shape if atlas.ndim == 3 else (0, 1, 1)
    atl = atlas if atlas.size else np.zeros(1, np.float32)
    st = _AlphaData(_p(tc), _p(mats), _p(atl), nm if alpha is not None else 0, w, h, layers,
                    int(a.get("sampler_id", 0xFFFFFFFF)))
    return st, (tc, mats, atl)


def trace(nodes: np.ndarray, tri_v: np.ndarray, tri_key: np.ndarray, rays: np.ndarray,
          any_hit: bool = False, shadow: bool = False, threads: int = 8, alpha=None):
    """Restated traversal.  nodes: flat 48-byte records; tri_v: (n, 9) float32
    in leaf order; tri_key: (n, 4) uint32 (instance, primitive, traversal, flags);
    rays: (m, 8) float32.  Returns dict of tri, t, u, v, front, status, counters."""
    m = rays.shape[0]
    out_tri = np.empty(m, np.uint32)
    tuv = np.empty((m, 3), np.float32)
    front = np.empty(m, np.uint32)
    status = np.empty(m, np.uint32)
    cnt = np.zeros(2, np.uint64)
    oracle_lib().oracle_trace_alpha(_p(nodes), len(nodes), _p(np.ascontiguousarray(tri_v, np.float32)),
                                    _p(np.ascontiguousarray(tri_key, np.uint32)),
                                    _p(np.ascontiguousarray(rays, np.float32)), m, int(any_hit), int(shadow),
                                    threads, _p(out_tri), _p(tuv), _p(front), _p(status), _p(cnt),
                                    None if alpha is None else C.byref(alpha))
    return {"tri": out_tri, "t": tuv[:, 0], "u": tuv[:, 1], "v": tuv[:, 2], "front": front,
            "status": status, "node_tests": int(cnt[0]), "tri_tests": int(cnt[1])}


def ref_sah_build(tri_v: np.ndarray, ids: np.ndarray, max_leaf: int = 4):
    n = tri_v.shape[0]
    cap = 2 * n + 1
    nodes = np.zeros((cap, 12), np.float32)
    order = np.zeros(n, np.uint32)
    depth = C.c_uint32(0)
    status = C.c_int(0)
    cnt = ref_lib().ref_sah_build(_p(np.ascontiguousarray(tri_v, np.float32)),
                                  _p(np.ascontiguousarray(ids, np.uint32)), n, max_leaf,
                                  _p(nodes), cap, _p(order), C.byref(depth), C.byref(status))
    if cnt < 0:
        raise RuntimeError(f"reference SAH build failed with status {status.value}")
    return nodes[:cnt].copy(), order, depth.value


def ref_trace(nodes12: np.ndarray, prim_v: np.ndarray, prim_ids: np.ndarray, rays12: np.ndarray,
              any_hit: bool = False, stack_capacity: int = 64, threads: int = 1):
    """SoftwareGpu::Trace.  rays12: (m, 12) float32 view of SoftwareRayRecord
    (query words as raw bits).  Returns (hits (m, 8) uint32 view, counters)."""
    m = rays12.shape[0]
    hits = np.zeros((m, 8), np.uint32)
    cnt = np.zeros(11, np.uint64)
    ref_lib().ref_trace(_p(np.ascontiguousarray(nodes12, np.float32)), nodes12.shape[0],
                        _p(np.ascontiguousarray(prim_v, np.float32)),
                        _p(np.ascontiguousarray(prim_ids, np.uint32)), prim_v.shape[0],
                        _p(np.ascontiguousarray(rays12)), m, int(any_hit), stack_capacity, threads,
                        _p(hits), _p(cnt))
    return hits, cnt


def ref_l3_parity_corpus(ray_count: int):
    tris = np.zeros((18, 9), np.float32)
    ids = np.zeros(18, np.uint32)
    rays = np.zeros((ray_count, 8), np.float32)
    bid = np.zeros(ray_count, np.uint32)
    bt = np.zeros(ray_count, np.float64)
    ref_lib().ref_l3_parity_corpus(ray_count, _p(tris), _p(ids), _p(rays), _p(bid), _p(bt))
    return tris, ids, rays, bid, bt


def ref_cornell(width: int, height: int, spp: int, bounces: int, seed: int, threads: int = 0):
    px = np.zeros(width * height * 3, np.float32)
    stats = np.zeros(4, np.uint64)
    ms = ref_lib().ref_cornell(width, height, spp, bounces, seed, threads, _p(px), _p(stats))
    if ms < 0:
        raise RuntimeError("reference Cornell render failed")
    return px.reshape(height, width, 3), {"scene_hash": int(stats[0]), "rays": int(stats[1]),
                                          "shadow_rays": int(stats[2]), "non_finite": int(stats[3]),
                                          "ms": ms}


# ---------------------------------------------------------------------------
# Wavefront PBR integrator
# ---------------------------------------------------------------------------
class OracleRenderInputs:
    """Leaf-ordered oracle buffers for a scene flattened into `nodes` / `order`."""

    def __init__(self, scene_data, nodes: np.ndarray, order: np.ndarray):
        t = scene_data.triangles[order]
        self.nodes = np.ascontiguousarray(nodes)
        self.tri_v = np.ascontiguousarray(t["positions"][:, :, :3].reshape(-1, 9), np.float32)
        self.tri_n = np.ascontiguousarray(t["normals"][:, :, :3].reshape(-1, 9), np.float32)
        key = np.zeros((len(t), 4), np.uint32)
        key[:, 0] = t["identity"][:, 0]
        key[:, 1] = t["identity"][:, 1]
        key[:, 2] = t["metadata"][:, 2]
        ds = ((t["metadata"][:, 0] & (1 << 2)) != 0) | ((t["metadata"][:, 1] & 1) != 0)
        cs = (t["metadata"][:, 3] & 2) != 0
        am = ((t["metadata"][:, 0] & 2) != 0) | ((t["metadata"][:, 1] & 2) != 0)
        key[:, 3] = ds.astype(np.uint32) | (cs.astype(np.uint32) << 1) | (am.astype(np.uint32) << 2)
        self.alpha, self._alpha_keep = alpha_data(t, (scene_data.extra or {}).get("alpha"))
        self.tri_key = key
        self.tri_ids = np.ascontiguousarray(t["identity"], np.uint32)
        # Emitter map: (instance, primitive) of emissive-triangle lights.
        em = np.full(len(t), 0xFFFFFFFF, np.uint32)
        L = scene_data.lights
        tri_lights = np.nonzero(L["identity"][:, 0] == 4)[0]
        if len(tri_lights):
            lk = (L["payload"][tri_lights, 3].astype(np.uint64) << np.uint64(32)) | L["identity"][tri_lights, 3]
            tk = (t["identity"][:, 0].astype(np.uint64) << np.uint64(32)) | t["identity"][:, 1]
            lut = dict(zip(lk.tolist(), tri_lights.tolist()))
            hit = np.isin(tk, lk)
            em[hit] = [lut[k] for k in tk[hit].tolist()]
        self.emitter = em
        self.materials = np.ascontiguousarray(scene_data.materials)
        self.lights = np.ascontiguousarray(scene_data.lights)
        self.fixtures = np.ascontiguousarray(scene_data.fixture_triangles)
        env = (scene_data.extra or {}).get("environment")
        self.environment = None if env is None else np.ascontiguousarray(env, np.float32)


def oracle_frame(frame_constants: np.ndarray) -> np.ndarray:
    """Maps a 304-byte MegakernelFrameConstantsGpu record to the oracle Frame."""
    fc = frame_constants[0]
    f = np.zeros(1, FRAME_DTYPE)
    f["cam_pos"] = fc["camera_position_tan_half_fov"][:3]
    f["tan_half_fov"] = fc["camera_position_tan_half_fov"][3]
    f["fwd"] = fc["camera_forward_aspect"][:3]
    f["aspect"] = fc["camera_forward_aspect"][3]
    f["right"] = fc["camera_right_lens_radius"][:3]
    f["up"] = fc["camera_up_exposure"][:3]
    f["width"], f["height"], f["sample"], f["max_depth"] = fc["image"]
    f["seed_lo"], f["seed_hi"] = fc["sampling"][0], fc["sampling"][1]
    f["estimator"] = fc["sampling"][3]
    f["stream"] = fc["output"][0]
    f["rr_start"], f["rr_min"], f["rr_max"], f["eps"] = fc["russian_roulette"]
    xf = np.concatenate([fc["environment_to_world"].reshape(-1), fc["world_to_environment"].reshape(-1)])
    if not np.any(xf.reshape(6, 4)[:, :3]):  # all zero: identity, as the renderer reads it
        xf = np.tile(np.array([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0], np.float32), 2)
    f["env_xf"] = xf
    return f


def render(inputs: OracleRenderInputs, frame_constants: np.ndarray, light_selection: int = 0,
           scene_radius: float = 1.0, pixels: np.ndarray | None = None, threads: int = 8):
    """One sample per pixel.  Returns (planes dict of (n, 4) arrays, path rays, shadow rays)."""
    f = oracle_frame(frame_constants)
    w, h = int(f["width"][0]), int(f["height"][0])
    n = w * h if pixels is None else len(pixels)
    px = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
    out = np.zeros((len(PLANES) + 7, n, 4), np.float32)
    counts = np.zeros(2, np.uint64)
    env = getattr(inputs, "environment", None)
    oracle_lib().oracle_render_env(
        _p(inputs.nodes), len(inputs.nodes), _p(inputs.tri_v), _p(inputs.tri_key), _p(inputs.tri_n),
        _p(inputs.tri_ids), _p(inputs.emitter), _p(inputs.materials), len(inputs.materials),
        _p(inputs.lights) if len(inputs.lights) else None, len(inputs.lights),
        _p(inputs.fixtures) if len(inputs.fixtures) else None, len(inputs.fixtures), light_selection,
        scene_radius, _p(f), _p(px), n, threads, _p(out), _p(counts),
        None if env is None else _p(env), 0 if env is None else env.shape[1], 0 if env is None else env.shape[0],
        None if getattr(inputs, "alpha", None) is None else C.byref(inputs.alpha))
    planes = {name: out[i] for i, name in enumerate(PLANES)}
    # GpuPrimarySurfaceV2 per pixel as 24 words (float lanes; identity as bits).
    planes["surface"] = np.ascontiguousarray(out[len(PLANES):len(PLANES) + 6].transpose(1, 0, 2).reshape(n, 24))
    # libm transcendentals (sin, cos, pow, acos, atan2) the pixel's path
    # evaluated: where CUDA's and glibc's results may differ in the last bit.
    planes["libm_calls"] = out[len(PLANES) + 6][:, 0].astype(np.int64)
    return planes, int(counts[0]), int(counts[1])


def environment_tables(env: np.ndarray):
    """The oracle's environment importance tables for an (h, w, 4) map:
    (row entries (h, 4), column entries (h * w, 4), integrated luminance);
    entries (q, pmf, alias bits, item bits) as float32 lanes."""
    e = np.ascontiguousarray(env, np.float32)
    h, w = e.shape[:2]
    rows = np.zeros((h, 4), np.float32)
    cols = np.zeros((h * w, 4), np.float32)
    integ = C.c_double(0.0)
    oracle_lib().oracle_environment_tables(_p(e), w, h, _p(rows), _p(cols), C.byref(integ))
    return rows, cols, integ.value


def ref_environment_tables(env: np.ndarray):
    """The reference's BuildEnvironmentDistribution over the map's luminance
    (0.2126 r + 0.7152 g + 0.0722 b in float, as Wave2Runtime computes it):
    (rows, columns, integrated luminance, fallback) with entries as float32
    lanes like environment_tables()."""
    e = np.ascontiguousarray(env, np.float32)
    h, w = e.shape[:2]
    lum = (np.float32(0.2126) * e[..., 0] + np.float32(0.7152) * e[..., 1]).astype(np.float32)
    lum = np.ascontiguousarray((lum + np.float32(0.0722) * e[..., 2]).astype(np.float32).reshape(-1))
    rows = np.zeros((h, 4), np.float32)
    cols = np.zeros((h * w, 4), np.float32)
    integ = C.c_double(0.0)
    fb = C.c_int(0)
    if ref_lib().ref_env_distribution(w, h, _p(lum), _p(rows), _p(cols), C.byref(integ), C.byref(fb)) != 0:
        raise ValueError("reference rejected the environment")
    return rows, cols, integ.value, bool(fb.value)


def counter_random(pixel, sample, dim, stream, seed_lo, seed_hi) -> float:
    return oracle_lib().oracle_counter_random(pixel, sample, dim, stream, seed_lo, seed_hi)


def light_distribution(lights: np.ndarray, selection: int, scene_radius: float = 1.0) -> np.ndarray:
    out = np.zeros((max(1, len(lights)), 4), np.float32)
    n = oracle_lib().oracle_light_distribution(_p(np.ascontiguousarray(lights)), len(lights), selection,
                                               scene_radius, _p(out))
    return out[:n]


def ref_light_distribution(lights: np.ndarray, selection: int, scene_radius: float = 1.0):
    alias = np.zeros((max(1, len(lights)), 4), np.uint32)
    pmf = np.zeros(max(1, len(lights)), np.float32)
    n = ref_lib().ref_light_distribution(_p(np.ascontiguousarray(lights)), len(lights), selection, scene_radius,
                                         _p(alias), _p(pmf))
    if n < 0:
        raise RuntimeError("reference light distribution failed")
    return alias[:n], pmf[:len(lights)]


# ---------------------------------------------------------------------------
# SVGF / A-Trous: the restatement (oracle_svgf.cpp) and the reference's own
# SvgfReconstruction (ref_svgf.cpp) behind one interface.  Inputs are
# (height, width) arrays of the C ABI's re_gbuffer_pixel / re_signal_pixel
# records; the config is any ctypes structure with re_svgf_config's layout.
# ---------------------------------------------------------------------------
class _SvgfOutputs(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("raw", "temporal", "atrous", "svgf", "history_length", "moments",
                                          "variance", "accepted", "reject")]


class _SvgfBase:
    _prefix = ""

    def __init__(self, width: int, height: int, frames_in_flight: int, config):
        self._lib = self._library()
        self._h = getattr(self._lib, self._prefix + "svgf_create")(width, height, frames_in_flight,
                                                                   C.byref(config))
        if not self._h:
            raise ValueError("invalid SVGF configuration")

    def close(self):
        if self._h:
            getattr(self._lib, self._prefix + "svgf_destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_config(self, config) -> None:
        if getattr(self._lib, self._prefix + "svgf_set_config")(self._h, C.byref(config)) != 0:
            raise ValueError("invalid SVGF configuration")

    def process(self, gbuffer: np.ndarray, signal: np.ndarray, frame_index: int, reset_trigger: int = 0) -> dict:
        gb = np.ascontiguousarray(gbuffer)
        sig = np.ascontiguousarray(signal)
        assert gb.dtype.itemsize == 64 and sig.dtype.itemsize == 24 and gb.shape == sig.shape
        h, w = gb.shape
        planes = {
            "raw": np.zeros((h, w, 6), np.float32), "temporal": np.zeros((h, w, 6), np.float32),
            "atrous": np.zeros((h, w, 6), np.float32), "svgf": np.zeros((h, w, 6), np.float32),
            "history_length": np.zeros((h, w), np.uint32), "moments": np.zeros((h, w, 2), np.float32),
            "variance": np.zeros((h, w), np.float32), "accepted": np.zeros((h, w), np.uint32),
            "reject": np.zeros((h, w), np.uint32)}
        outs = _SvgfOutputs(*[a.ctypes.data for a in planes.values()])
        rc = getattr(self._lib, self._prefix + "svgf_process")(self._h, gb.ctypes.data, sig.ctypes.data, w, h,
                                                                frame_index, reset_trigger, C.byref(outs))
        if rc != 0:
            raise ValueError("SVGF process failed")
        return planes


class OracleSvgf(_SvgfBase):
    """CPU restatement of SvgfReconstruction (oracle_svgf.cpp)."""
    _prefix = "oracle_"

    @staticmethod
    def _library():
        return oracle_lib()


class RefSvgf(_SvgfBase):
    """The reference's own SvgfReconstruction (reconstruction/src/Svgf.cpp)."""
    _prefix = "ref_"

    @staticmethod
    def _library():
        return ref_lib()

    def select_output(self, gbuffer: np.ndarray, output: int) -> np.ndarray:
        gb = np.ascontiguousarray(gbuffer)
        h, w = gb.shape
        out = np.zeros((h, w, 3), np.float32)
        if self._lib.ref_svgf_select(self._h, gb.ctypes.data, w, h, output, out.ctypes.data) != 0:
            raise ValueError("SelectOutput failed")
        return out


def image_rmse(a: np.ndarray, b: np.ndarray) -> float:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return float(oracle_lib().oracle_image_rmse(a.ctypes.data, b.ctypes.data, a.size // 3))


def ref_image_rmse(a: np.ndarray, b: np.ndarray) -> float:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return float(ref_lib().ref_image_rmse(a.ctypes.data, b.ctypes.data, a.shape[1], a.shape[0]))


def ref_image_psnr(a: np.ndarray, b: np.ndarray, peak: float = 1.0) -> float:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return float(ref_lib().ref_image_psnr(a.ctypes.data, b.ctypes.data, a.shape[1], a.shape[0], peak))


def _motion(fn, position, cur_vp, prev_vp, prev_w2v, cur_jitter=(0.0, 0.0), prev_jitter=(0.0, 0.0)):
    args = [np.ascontiguousarray(x, np.float32) for x in (position, cur_vp, prev_vp, prev_w2v, cur_jitter,
                                                          prev_jitter)]
    out = np.zeros(8, np.float32)
    fn(*[a.ctypes.data for a in args], out.ctypes.data)
    return out


def motion_vector(*args, **kw) -> np.ndarray:
    """(currentUv, previousUv, motion, expectedPreviousDepth, valid)."""
    return _motion(oracle_lib().oracle_motion_vector, *args, **kw)


def ref_motion_vector(*args, **kw) -> np.ndarray:
    return _motion(ref_lib().ref_motion_vector, *args, **kw)


# ---------------------------------------------------------------------------
# ReSTIR DI (oracle_pbr.cpp: oracle_restir_frame)
# ---------------------------------------------------------------------------
RESTIR_PARAMS_DTYPE = np.dtype([
    ("candidates", "<u4"), ("neighbors", "<u4"), ("max_m", "<u4"), ("max_age", "<u4"),
    ("history_enabled", "<u4"), ("neighbor_mode", "<u4"), ("scene_gen", "<u4"), ("light_gen", "<u4"),
    ("camera_gen", "<u4"), ("resolution_gen", "<u4"), ("history_gen", "<u4"), ("frame_lo", "<u4"),
    ("frame_hi", "<u4"), ("prev_valid", "<u4"), ("candidate_source", "<u4"), ("light_count", "<u4"),
    ("prev_light_count", "<u4"), ("estimator", "<u4"), ("pad", "<u4", 2),
    ("normal_cos", "<f4"), ("rel_depth", "<f4"), ("position_dist", "<f4"), ("disk_radius", "<f4"),
    ("prev_pos", "<f4", 3), ("prev_tan", "<f4"), ("prev_fwd", "<f4", 3), ("prev_aspect", "<f4"),
    ("prev_right", "<f4", 4), ("prev_up", "<f4", 4)])
assert RESTIR_PARAMS_DTYPE.itemsize == 160

RESTIR_DEFAULTS = dict(candidates=8, spatial_neighbors=5, max_m=32, max_history_age=20, temporal=1,
                       neighbor_mode=0, disk_radius=30.0, normal_cos=0.8, relative_depth=0.05,
                       position_distance=0.02, estimator=0)


class OracleRestir:
    """ReSTIR DI state across frames on the CPU, with the GPU renderer's
    bookkeeping: scene / light generation 1 after one scene bind, camera
    generation bumped by every configuration change and reset, resolution
    generation bumped when the extent changes, the previous frame's camera
    for the reprojection."""

    def __init__(self, inputs: "OracleRenderInputs", light_selection: int = 0, scene_radius: float = 1.0,
                 scene_gen: int = 1, **config):
        self.inp = inputs
        self.light_selection = light_selection
        self.scene_radius = scene_radius
        self.scene_gen = scene_gen
        self.camera_gen = 1
        self.resolution_gen = 1
        self.cfg = dict(RESTIR_DEFAULTS)
        self.last_wh = (0, 0)
        self.prev_frame = None
        self.prev_light_count = 0
        self.prev_surface = None
        self.prev_published = None
        if config:
            self.set_config(**config)

    def set_config(self, **config):
        self.cfg.update(config)
        self.camera_gen += 1

    def reset(self):
        self.camera_gen += 1

    def params(self, fc: np.ndarray) -> np.ndarray:
        f = fc[0]
        w, h = int(f["image"][0]), int(f["image"][1])
        rp = np.zeros(1, RESTIR_PARAMS_DTYPE)
        c = self.cfg
        rp["candidates"] = c["candidates"]
        rp["neighbors"] = c["spatial_neighbors"]
        rp["max_m"] = c["max_m"]
        rp["max_age"] = c["max_history_age"]
        rp["history_enabled"] = c["temporal"]
        rp["neighbor_mode"] = c["neighbor_mode"]
        rp["scene_gen"] = rp["light_gen"] = self.scene_gen
        rp["camera_gen"] = self.camera_gen
        rp["resolution_gen"] = self.resolution_gen + (1 if (w, h) != self.last_wh else 0)
        rp["history_gen"] = 1
        rp["frame_lo"] = f["image"][2]
        rp["frame_hi"] = 0
        rp["prev_valid"] = 1 if self.prev_frame is not None else 0
        rp["candidate_source"] = 2 if self.light_selection == 1 else 1
        rp["light_count"] = len(self.inp.lights)
        rp["prev_light_count"] = self.prev_light_count
        rp["normal_cos"] = c["normal_cos"]
        rp["rel_depth"] = c["relative_depth"]
        rp["position_dist"] = c["position_distance"]
        rp["disk_radius"] = c["disk_radius"]
        rp["estimator"] = c.get("estimator", 0)
        if self.prev_frame is not None:
            pf = self.prev_frame[0]
            rp["prev_pos"] = pf["camera_position_tan_half_fov"][:3]
            rp["prev_tan"] = pf["camera_position_tan_half_fov"][3]
            rp["prev_fwd"] = pf["camera_forward_aspect"][:3]
            rp["prev_aspect"] = pf["camera_forward_aspect"][3]
            rp["prev_right"][0, :3] = pf["camera_right_lens_radius"][:3]
            rp["prev_up"][0, :3] = pf["camera_up_exposure"][:3]
        return rp

    def frame(self, fc: np.ndarray, surface: np.ndarray, prev_surface: np.ndarray | None = None,
              prev_published: np.ndarray | None = None, threads: int = 8) -> dict:
        """One ReSTIR frame over `surface` (n x 24 words).  The previous
        surfaces / published reservoirs default to this object's own."""
        f = fc[0]
        w, h = int(f["image"][0]), int(f["image"][1])
        n = w * h
        rp = self.params(fc)
        ps = prev_surface if prev_surface is not None else self.prev_surface
        pp = prev_published if prev_published is not None else self.prev_published
        if ps is None or ps.shape[0] != n:
            ps = np.zeros((n, 24), np.float32)
        if pp is None or pp.shape[0] != n:
            pp = np.zeros((n, 64), np.uint32)
        cur = np.ascontiguousarray(surface).view(np.uint32).reshape(n, 24)
        ps = np.ascontiguousarray(ps).view(np.uint32).reshape(n, 24)
        pp = np.ascontiguousarray(pp, np.uint32).reshape(n, 64)
        temporal = np.zeros((n, 64), np.uint32)
        published = np.zeros((n, 64), np.uint32)
        direct = np.zeros((2, n, 4), np.float32)
        reasons = np.zeros(n, np.uint32)
        stats = np.zeros(12, np.uint32)
        ofr = oracle_frame(fc)
        inp = self.inp
        oracle_lib().oracle_restir_frame(
            _p(inp.nodes), len(inp.nodes), _p(inp.tri_v), _p(inp.tri_key),
            _p(inp.lights) if len(inp.lights) else None, len(inp.lights),
            _p(inp.fixtures) if len(inp.fixtures) else None, len(inp.fixtures), self.light_selection,
            self.scene_radius, _p(ofr), _p(rp), _p(cur), _p(ps), _p(pp), _p(temporal), _p(published),
            _p(direct), _p(reasons), _p(stats), threads)
        # Commit like a rendered GPU frame.
        self.resolution_gen = int(rp["resolution_gen"][0])
        self.last_wh = (w, h)
        self.prev_frame = fc.copy()
        self.prev_light_count = len(inp.lights)
        self.prev_surface = cur.copy()
        self.prev_published = published.copy()
        return {"temporal": temporal, "published": published, "direct": direct, "reasons": reasons,
                "stats": stats}


def restir_spatial_gate(center: np.ndarray, neighbor: np.ndarray, neighbor_valid: np.ndarray,
                        rp: np.ndarray) -> np.ndarray:
    """Reason code (RestirRejectionReason) of each (centre, neighbour) pair
    of the spatial pass; surfaces are n x 24 GpuPrimarySurfaceV2 words."""
    c = np.ascontiguousarray(center, np.float32).view(np.uint32).reshape(-1, 24)
    b = np.ascontiguousarray(neighbor, np.float32).view(np.uint32).reshape(-1, 24)
    v = np.ascontiguousarray(neighbor_valid, np.uint32)
    out = np.zeros(len(c), np.uint32)
    oracle_lib().oracle_restir_spatial_gate(_p(c), _p(b), _p(v), len(c), _p(np.ascontiguousarray(rp)), _p(out))
    return out


def restir_temporal_gate(current: np.ndarray, history_surface: np.ndarray, history: np.ndarray,
                         reproj: np.ndarray, reprojected_depth: np.ndarray, rp: np.ndarray) -> np.ndarray:
    """Reason code of each temporal history (oracle_pbr.cpp temporal_gate);
    history is n x 64 GpuRestirReservoirV3 words."""
    c = np.ascontiguousarray(current).view(np.uint32).reshape(-1, 24)
    h = np.ascontiguousarray(history_surface).view(np.uint32).reshape(-1, 24)
    r = np.ascontiguousarray(history, np.uint32).reshape(-1, 64)
    out = np.zeros(len(c), np.uint32)
    oracle_lib().oracle_restir_temporal_gate(_p(c), _p(h), _p(r), _p(np.ascontiguousarray(reproj, np.uint32)),
                                             _p(np.ascontiguousarray(reprojected_depth, np.float32)), len(c),
                                             _p(np.ascontiguousarray(rp)), _p(out))
    return out


def ref_restir_validate(kind: str, geo: np.ndarray, ids: np.ndarray, gen: np.ndarray, thresholds, max_age: int,
                        flags: np.ndarray | None = None) -> np.ndarray:
    """RejectionReason bitmask of the reference's ValidateSpatialNeighbor
    (kind "spatial") or ValidateTemporalHistory ("temporal") per case
    (ref_restir.cpp for the packing of geo / ids / flags)."""
    g = np.ascontiguousarray(geo, np.float32)
    w = np.ascontiguousarray(ids, np.uint32)
    gn = np.ascontiguousarray(gen, np.uint32)
    th = np.asarray(thresholds, np.float32)
    out = np.zeros(len(g), np.uint32)
    if kind == "spatial":
        ref_lib().ref_restir_validate_spatial(_p(g), _p(w), _p(gn), len(g), _p(th), max_age, _p(out))
    else:
        ref_lib().ref_restir_validate_temporal(_p(g), _p(w), _p(np.ascontiguousarray(flags, np.uint32)), _p(gn),
                                               len(g), _p(th), max_age, _p(out))
    return out


def restir_ris(terms: np.ndarray, u: np.ndarray, max_m: int):
    """(selected index or -1, weightSum, W, M) of the float reservoir update."""
    t = np.ascontiguousarray(terms, np.float32)
    uu = np.ascontiguousarray(u, np.float32)
    out = np.zeros(2, np.float32)
    m = np.zeros(1, np.uint32)
    sel = oracle_lib().oracle_restir_ris(_p(t), _p(uu), len(uu), max_m, _p(out), _p(m))
    return sel, float(out[0]), float(out[1]), int(m[0])


def ref_restir_ris(terms: np.ndarray, u: np.ndarray, max_m: int):
    """The reference's UpdateReservoir / ClampReservoirM / FinalizeReservoir."""
    t = np.ascontiguousarray(terms, np.float32)
    uu = np.ascontiguousarray(u, np.float32)
    out = np.zeros(2, np.float64)
    m = np.zeros(1, np.uint32)
    sel = ref_lib().ref_restir_ris(_p(t), _p(uu), len(uu), max_m, _p(out), _p(m))
    return sel, float(out[0]), float(out[1]), int(m[0])


def linear_rgb_hash(image: np.ndarray) -> int:
    """Restatement of HashLinearRgbPixels (src/rt/cpu/ImageOutput.cpp:343-380):
    64-bit FNV-1a over the tag b"RERGB" 1 3 0, width and height as
    little-endian uint32, then every component's float32 bits little-endian
    with -0 folded to +0.  Pure Python over the bytes: small images only."""
    img = np.ascontiguousarray(image, np.float32)
    h, w = img.shape[:2]
    flat = img.reshape(-1).copy()
    flat[flat == 0.0] = 0.0
    data = b"RERGB\x01\x03\x00" + int(w).to_bytes(4, "little") + int(h).to_bytes(4, "little") + \
        flat.view("<u4").tobytes()
    value, mask = 0xCBF29CE484222325, (1 << 64) - 1
    for b in data:
        value = ((value ^ b) * 0x100000001B3) & mask
    return value


def restir_debug(words: np.ndarray, mode: int, max_m: int, max_age: int):
    """Restatement of RestirDebugV3 (resources/shaders/restir/RestirDebugV3.comp.hlsl:33-121)
    over published GpuRestirReservoirV3 records given as (n, 64) uint32 words:
    (records (n, 16) uint32 = identity, generation, scalar bits, state;
    view (n, 4) float32 for `mode`), in float32 arithmetic."""
    u = np.ascontiguousarray(words, np.uint32).reshape(-1, 64)
    f = u.view(np.float32)
    n = len(u)
    f32 = np.float32
    sel_identity, sel_generation, sel_source = u[:, 16:20], u[:, 20:24], u[:, 28:32]
    weight, terms, state, prov, h_reproj = f[:, 32:36], f[:, 36:40], u[:, 40:44], u[:, 44:48], u[:, 60:64]
    fz = lambda v: np.where(np.isfinite(v), v, f32(0)).astype(f32)
    rec = np.zeros((n, 16), np.uint32)
    rec[:, 0:2] = sel_identity[:, 0:2]
    rec[:, 2:4] = prov[:, 0:2]
    rec[:, 4:8] = sel_generation
    rec[:, 8:11] = fz(weight[:, 0:3]).view(np.uint32)
    rec[:, 11] = fz(terms[:, 3]).view(np.uint32)
    rec[:, 12:16] = state
    finite = np.isfinite(f[:, 32:40]).all(axis=1) & np.isfinite(f[:, 0:16]).all(axis=1)
    a = np.where(finite, f32(1), f32(0))
    flag = lambda bit: np.where((state[:, 2] & bit) != 0, f32(1), f32(0))
    img = np.zeros((n, 4), f32)
    img[:, 3] = a
    if mode == 0:
        img[:, 0] = state[:, 0].astype(f32) / f32(max(max_m, 1))
        img[:, 1] = state[:, 1].astype(f32) / f32(max(max_age, 1))
        img[:, 2] = flag(2)
    elif mode == 1:
        v = fz(np.concatenate([weight[:, 0:3], terms[:, 3:4]], axis=1))
        x = np.maximum(v[:, 0:3], f32(0))
        img[:, 0:3] = x / (f32(1) + x)
        img[:, 3] = v[:, 3]
    elif mode <= 5:
        if mode == 2:
            xyz = [sel_identity[:, 0], sel_identity[:, 1], sel_generation[:, 0]]
            xyz = [c.astype(f32) for c in xyz]
        elif mode == 3:
            xyz = [prov[:, 0].astype(f32), prov[:, 2].astype(f32), sel_source[:, 0].astype(f32)]
        elif mode == 4:
            xyz = [prov[:, 1].astype(f32), flag(4), flag(8)]
        else:
            xyz = [state[:, 3].astype(f32), h_reproj[:, 0].astype(f32), prov[:, 2].astype(f32)]
        for k, (c, m) in enumerate(zip(xyz, (f32(0.6180339), f32(0.381966), f32(0.7548777)))):
            x = np.maximum(c, f32(0)) * m
            img[:, k] = x - np.floor(x)
    else:
        w_y, t_w = weight[:, 1], terms[:, 3]
        ok = ((state[:, 2] & 32) != 0) & (w_y > 0) & np.isfinite(w_y) & np.isfinite(t_w)
        with np.errstate(all="ignore"):
            vis = np.clip(np.where(ok, t_w / np.where(ok, w_y, f32(1)), f32(0)), f32(0), f32(1)).astype(f32)
        img[:, 0] = vis
        img[:, 1] = flag(32)
        img[:, 2] = flag(64)
    return rec, img
