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
}
_REF_SIGS = {
    "ref_sah_build": (C.c_int, [_P, _P, _U32, _U32, _P, _U32, _P, _P, _P]),
    "ref_trace": (None, [_P, _U32, _P, _P, _U32, _P, _U32, _U32, _U32, _U32, _P, _P]),
    "ref_lbvh_build": (C.c_int, [_P, _P, _U32, _P, _U32, _P, _P, _P, _P]),
    "ref_cornell": (C.c_double, [_U32, _U32, _U32, _U32, C.c_uint64, _U32, _P, _P]),
    "ref_counter_random": (C.c_float, [_U32, _U32, _U32, _U32, C.c_uint64]),
    "ref_philox": (None, [_P, _P, _P]),
    "ref_alias_table": (C.c_int, [_P, _U32, _P]),
    "ref_light_distribution": (C.c_int, [_P, _U32, _U32, C.c_float, _P, _P]),
    "ref_l3_parity_corpus": (None, [_U32, _P, _P, _P, _P, _P]),
}

_oracle = None
_ref = None


def build() -> None:
    """Compiles the oracle restatement and, when the reference tree is present, _ref."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)


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
def trace(nodes: np.ndarray, tri_v: np.ndarray, tri_key: np.ndarray, rays: np.ndarray,
          any_hit: bool = False, shadow: bool = False, threads: int = 8):
    """Restated traversal.  nodes: flat 48-byte records; tri_v: (n, 9) float32
    in leaf order; tri_key: (n, 4) uint32 (instance, primitive, traversal, flags);
    rays: (m, 8) float32.  Returns dict of tri, t, u, v, front, status, counters."""
    m = rays.shape[0]
    out_tri = np.empty(m, np.uint32)
    tuv = np.empty((m, 3), np.float32)
    front = np.empty(m, np.uint32)
    status = np.empty(m, np.uint32)
    cnt = np.zeros(2, np.uint64)
    oracle_lib().oracle_trace(_p(nodes), len(nodes), _p(np.ascontiguousarray(tri_v, np.float32)),
                              _p(np.ascontiguousarray(tri_key, np.uint32)),
                              _p(np.ascontiguousarray(rays, np.float32)), m, int(any_hit), int(shadow),
                              threads, _p(out_tri), _p(tuv), _p(front), _p(status), _p(cnt))
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
