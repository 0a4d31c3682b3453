"""Benchmark of the B200 wavefront path-tracing hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload trace|frame]

Prints ONE JSON line on rank 0.  Multi-GPU runs (torchrun, one rank per GPU)
are replicas with no data-path collective: every rank renders its own copy of
the workload; `value` is the aggregate over ranks of the work done divided by
the maximum per-rank device time ("scaling": "weak").

`--impl reference` times the reference's own CPU implementation of the same
path (oracle/_ref, compiled from the unmodified reference sources) on the host
cores, on a bounded sample of the workload per step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s & samples/s on 1 B200, batched/served vs plain; p50/p99 request latency"


# ---------------------------------------------------------------------------
# Clock sampling during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


# DRAM bytes (read + write) of the 8 k_intersect launches of one frame of the
# frame workload, by hierarchy and node layout, from one ncu capture each of
# this command with --tuning b200_frame_lbvh (dram__bytes_read.sum +
# dram__bytes_write.sum, mean of two frames that agree within 0.6 %), with the
# source revision the capture ran.  Not measured by the run itself: ncu is not
# available inside it.  Layouts without a capture report null.
INTERSECT_DRAM_BYTES_PER_FRAME = {
    ("lbvh", "four-wide"): (573.9e6, "ncu capture, source of commit ad76b66, k_intersect<64, 4, 512>"),
    ("sah", "four-wide"): (498.3e6, "ncu capture, source of commit ad76b66, k_intersect<64, 2, 512>"),
}
NODE_LAYOUT = {0: "child-pair", 1: "child-pair", 2: "four-wide", 4: "four-wide", 5: "eight-wide",
               6: "eight-wide-compressed", 7: "four-wide-conservative", 8: "four-wide-conservative"}


def intersect_layout(build: str, traversal: int) -> str:
    """Node layout the frame's Intersect launches fetch: mode 3 picks the
    four-wide loop per launch on either hierarchy."""
    return NODE_LAYOUT.get(traversal, "four-wide")


def frame_kernels(tuning: dict, depth: int) -> int:
    """Kernels one frame launches (all of them this library's): RayGen,
    per bounce Intersect (unless fused into Shade), the Shade form's kernels
    and TraceShadow, then Resolve."""
    shade = {0: 1, 1: 1, 2: 1, 3: 2, 4: 2, 5: 3, 6: 3, 7: 3}[tuning.get("shade_variant", 4)]
    per_bounce = (0 if tuning.get("fuse") else 1) + shade + 1
    return 2 + depth * per_bounce


def measured_peak_hbm() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def measure_l2_gbs(device_bytes: int = 24 << 20, repeats: int = 100) -> float:
    """L2 bandwidth of this GPU, measured in the run: a device-to-device copy
    of a 24 MiB buffer (read + write 48 MiB, resident in the 126 MB L2 after
    the first pass), best of three timed batches of `repeats` copies, bytes
    read + written over CUDA-event time."""
    import torch
    a = torch.empty(device_bytes // 4, dtype=torch.float32, device="cuda").uniform_()
    b = torch.empty_like(a)
    for _ in range(5):
        b.copy_(a)
    best = float("inf")
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(repeats):
            b.copy_(a)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / repeats)
    del a, b
    return 2.0 * device_bytes / (best / 1e3) / 1e9


# ---------------------------------------------------------------------------
# Workloads
# ---------------------------------------------------------------------------
class TraceWorkload:
    """Closest-hit traversal of the 1080p camera rays of the 2,424,832-triangle
    heightfield + icosphere scene (flattened SAH), one batch per step."""

    name = "trace-closest 1920x1080 camera rays, heightfield 1024^2 + 4096 icospheres (2,424,832 tris)"

    def __init__(self, device: int, build: str = "sah"):
        import torch

        from renderingengine_b200 import _native as N
        from renderingengine_b200 import scenes
        from renderingengine_b200.traversal import Scene
        self.N = N
        self.torch = torch
        self.sd = heightfield()
        self.scene = Scene(self.sd.triangles, self.sd.fingerprint, 1, device=device)
        self.rays8 = scenes.pinhole_rays(self.sd.camera, 1920, 1080, seed=1)
        self.rays = scenes.to_ray_records(self.rays8)
        self.n = len(self.rays)
        self.d_rays = torch.from_numpy(self.rays.view(np.uint8).copy()).cuda()
        self.d_hits = torch.zeros(self.n * N.HIT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
        # Pinned host buffers for the end-to-end leg.
        self.h_rays = torch.from_numpy(self.rays.view(np.uint8).copy()).pin_memory()
        self.h_hits = torch.zeros(self.n * N.HIT_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
        info = self.scene.info()
        self.node_bytes, self.tri_bytes = info.node_bytes, info.triangle_bytes
        _, self.counters = self.scene.trace(self.rays, counters=True)

    def units_per_step(self) -> int:
        return self.n

    def step_device(self, stream) -> None:
        self.scene.trace_device(self.d_rays.data_ptr(), self.d_hits.data_ptr(), self.n,
                                stream=stream.cuda_stream)

    def step_e2e(self) -> None:
        rays = self.h_rays.numpy().view(self.N.RAY_DTYPE)
        hits = self.h_hits.numpy().view(self.N.HIT_DTYPE)
        b = self.N.TraceBatch(rays.ctypes.data, hits.ctypes.data, 0, 0, self.n, self.N.MEMORY_HOST,
                              self.scene.fingerprint, self.scene.generation, 0, None)
        import ctypes as C
        self.N.check(self.N.load().re_trace_closest(self.scene.handle, C.byref(b)))

    def bytes_per_step(self) -> tuple[int, int]:
        return self.n * self.N.RAY_DTYPE.itemsize, self.n * self.N.HIT_DTYPE.itemsize

    def algorithmic_bytes(self) -> int:
        c = self.counters
        node_fetches = (c["node_tests"] - self.n) // 2  # one 64 B child-pair record per interior visit
        return node_fetches * self.node_bytes + c["triangle_tests"] * self.tri_bytes

    def cpu_reference(self, sample: int, threads: int):
        """SoftwareGpu::Trace (reference CPU mirror) over `sample` rays of the
        same batch with `threads` host threads; returns (rays, seconds)."""
        if not hasattr(self, "_cpu"):
            nodes, order = self.scene.export_flat()
            self._cpu = CpuTraceArm(self.sd, nodes, order, self.rays8)
        return self._cpu.run(sample, threads)


def frame_workload_name(build: str) -> str:
    return ("wavefront frame 1920x1080 1spp maxbounce 8, heightfield 1024^2 + 4096 icospheres "
            "(2,424,832 tris), NEE+MIS, " + ("GPU LBVH (30-bit Morton)" if build == "lbvh"
                                             else "flattened binned SAH (16 bins, leaf <= 4)"))


class FrameWorkload:
    """One wavefront path-tracing frame per step: the 2,424,832-triangle
    heightfield + icosphere scene, 1920x1080, 1 spp, maximum bounce 8, NEE +
    MIS, one spherical light; film accumulated progressively.  Hierarchy: the
    GPU LBVH (30-bit Morton codes) of the traversal-bound configuration, or
    the reference's flattened binned SAH (`build="sah"`)."""

    def __init__(self, device: int, build: str = "lbvh"):
        import torch

        from renderingengine_b200 import _native as N
        from renderingengine_b200 import scenes
        from renderingengine_b200.traversal import Scene
        from renderingengine_b200.wavefront import FILM_SAMPLE, Renderer, frame_constants
        self.N, self.torch, self.FILM_SAMPLE = N, torch, FILM_SAMPLE
        self.frame_constants = frame_constants
        self.w, self.h, self.depth = 1920, 1080, 8
        self.sd = heightfield()
        kind = N.BUILD_LBVH if build == "lbvh" else N.BUILD_FLATTENED_SAH
        self.build = build
        self.name = frame_workload_name(build)
        self.scene = Scene(self.sd.triangles, self.sd.fingerprint, 1, kind, device=device)
        self.r = Renderer(self.w, self.h, self.depth, device)
        self.r.set_scene(self.scene, self.sd)
        self.frame = 0
        self.n = self.w * self.h
        # Two pinned film buffers: the read of frame k lands while frame k + 1
        # renders (re_renderer_read_view_async keeps two reads in flight).
        self.h_film = [torch.zeros(self.n * 16, dtype=torch.uint8).pin_memory() for _ in range(2)]
        info = self.scene.info()
        self.node_bytes, self.tri_bytes = info.node_bytes, info.triangle_bytes
        self.run_profile()

    def run_profile(self) -> None:
        """Per-stage CUDA-event times and traversal counts of one frame under
        the renderer's current tuning (taken again once the run's tuning is
        set): the first pass loads the kernels (lazy module loading), then
        the fastest of three warm passes (the counts are identical)."""
        self.r.profile(self._fc(0))
        self.prof = min((self.r.profile(self._fc(0)) for _ in range(3)), key=lambda p: sum(p["intersect_ms"]))
        self.rays_per_frame = sum(self.prof["rays"]) + sum(self.prof["shadows"])

    def _fc(self, sample):
        return self.frame_constants(self.sd.camera, self.w, self.h, sample, self.depth)

    def units_per_step(self) -> int:
        return self.rays_per_frame

    def reset_counts(self):
        self.r.render(self._fc(self.frame), accumulate=False)
        self.frame += 1
        self.r.collect()

    def step_device(self, stream) -> None:
        self.r.render(self._fc(self.frame), accumulate=True, stream=stream.cuda_stream)
        self.frame += 1

    def measured_units(self) -> tuple[int, int]:
        t = self.r.collect()
        return t.total_path_rays + t.total_shadow_rays, t.frames_accumulated

    def step_e2e(self) -> None:
        """One frame through the public API: the frame record uploaded from
        pinned memory inside render(), then its film sample plane read to
        pinned host memory asynchronously, overlapping the next frame; the
        caller's device synchronize after the last step waits for the last
        read."""
        self.r.render(self._fc(self.frame), accumulate=True)
        out = self.h_film[self.frame & 1].numpy().view(np.float32).reshape(self.n, 4)
        self.frame += 1
        self.r.read_async(self.FILM_SAMPLE, out)

    def finish_e2e(self) -> None:
        self.r.wait_reads()

    def bytes_per_step(self) -> tuple[int, int]:
        return 304, self.n * 16

    def roofline_stage(self):
        """(algorithmic bytes, seconds) of the Intersect stage over all bounces."""
        p = self.prof
        nb = 0
        # Node records the traversal fetched (child pairs or wide nodes, as
        # tuned) plus one triangle record per triangle test.
        for node_bytes, tt in zip(p["intersect_node_bytes"], p["intersect_triangle_tests"]):
            nb += node_bytes + tt * self.tri_bytes
        return nb, sum(p["intersect_ms"]) / 1e3, len(p["rays"])

    def cpu_reference(self, sample: int, threads: int):
        """FP32 CPU port of the same frame (oracle) on `sample` pixels."""
        if not hasattr(self, "_cpu"):
            nodes, order = self.scene.export_flat()
            self._cpu = CpuFrameArm(self.sd, nodes, order, self._fc(0))
        return self._cpu.run(sample, threads)


# ---------------------------------------------------------------------------
# CPU legs: the reference's own CPU code (oracle/_ref) or the FP32 port of the
# frame (oracle/oracle_pbr.cpp) over a given flattened hierarchy.  Neither
# touches the GPU or the product library.
# ---------------------------------------------------------------------------
class CpuTraceArm:
    def __init__(self, sd, nodes, order, rays8):
        leaf = sd.triangles[order]
        self.nodes12 = np.ascontiguousarray(nodes).view(np.float32).reshape(-1, 12)
        self.tv = np.ascontiguousarray(leaf["positions"][:, :, :3].reshape(-1, 9), np.float32)
        self.ids = np.ascontiguousarray(leaf["metadata"][:, 2])
        self.rays8 = rays8

    def run(self, sample: int, threads: int):
        from oracle import oracle as O
        sel = np.random.default_rng(0).choice(len(self.rays8), sample, replace=False)
        r = np.zeros((sample, 12), np.float32)
        r[:, :8] = self.rays8[sel]
        q = r[:, 8:].view(np.uint32)
        q[:, 0] = np.arange(sample)
        q[:, 2] = 0xFFFFFFFF
        t0 = time.perf_counter()
        O.ref_trace(self.nodes12, self.tv, self.ids, r, stack_capacity=128, threads=threads)
        return sample, time.perf_counter() - t0


class CpuFrameArm:
    def __init__(self, sd, nodes, order, fc):
        from oracle import oracle as O
        self.inputs = O.OracleRenderInputs(sd, nodes, order)
        self.fc = fc
        self.n = int(fc["image"][0][0]) * int(fc["image"][0][1])

    def run(self, sample: int, threads: int):
        from oracle import oracle as O
        px = np.random.default_rng(0).choice(self.n, sample, replace=False).astype(np.uint32)
        t0 = time.perf_counter()
        _, rays, shadows = O.render(self.inputs, self.fc, pixels=px, threads=threads)
        return rays + shadows, time.perf_counter() - t0


def reference_hierarchy(sd, build: str):
    """The scene's flattened hierarchy from the reference's own CPU builders
    (oracle/_ref): SoftwareGpu::BuildKarrasLbvh for the LBVH, Bvh<float>
    binned SAH + FlattenCanonicalL3BinnedSah for the SAH.  Returns (nodes as
    48-byte SoftwareNodeRecord words, leaf order as source indices)."""
    import ctypes as C

    from oracle import oracle as O
    from renderingengine_b200._native import NODE_DTYPE
    tri = sd.triangles
    v = np.ascontiguousarray(tri["positions"][:, :, :3].reshape(-1, 9), np.float32)
    ids = np.ascontiguousarray(tri["metadata"][:, 2], np.uint32)
    if build == "sah":
        nodes12, order, _ = O.ref_sah_build(v, ids)
        return np.ascontiguousarray(nodes12).view(NODE_DTYPE).reshape(-1), order
    n = len(tri)
    nodes12 = np.zeros((2 * n, 12), np.float32)
    prim_ids = np.zeros(n, np.uint32)
    morton = np.zeros((n, 2), np.uint32)
    depth, status = C.c_uint32(0), C.c_int(0)
    cnt = O.ref_lib().ref_lbvh_build(v.ctypes.data, ids.ctypes.data, n, nodes12.ctypes.data, 2 * n,
                                     prim_ids.ctypes.data, morton.ctypes.data, C.byref(depth), C.byref(status))
    if cnt <= 0:
        raise RuntimeError(f"reference LBVH build failed with status {status.value}")
    return np.ascontiguousarray(nodes12[:cnt]).view(NODE_DTYPE).reshape(-1), morton[:, 1].copy()


WORKLOADS = {"trace": TraceWorkload, "frame": FrameWorkload}

_HEIGHTFIELD = None


def heightfield():
    """The 2,424,832-triangle heightfield + icosphere scene, generated once."""
    global _HEIGHTFIELD
    if _HEIGHTFIELD is None:
        from renderingengine_b200 import scenes
        _HEIGHTFIELD = scenes.heightfield_scene()
    return _HEIGHTFIELD


def _pct(x, q):
    return round(float(np.percentile(np.asarray(x, np.float64), q)) * 1e3, 3) if len(x) else None


# ---------------------------------------------------------------------------
# Batched views vs the plain single-view launch
# ---------------------------------------------------------------------------
def run_batched(device: int, warmup: int, steps: int, save_tuning: str | None = None) -> dict:
    """64 camera views over four scenes (36 to 2,434,832 triangles), each to
    its own sample count, rendered (a) batched: all views resident in one
    path pool; sample k of every view that still needs one is rendered in
    the planner's launches (each scene's views together, at most a path
    budget picked by a short sweep), each launch one persistent kernel per
    stage and bounce replayed from a CUDA graph; (b) plain: the same views
    one after another, one launch per sample, on single-view renderers.
    Both produce the same films (checked below on the non-ReSTIR views);
    samples/s = pixels x spp over device time."""
    import torch

    from renderingengine_b200 import _native as N
    from renderingengine_b200 import workloads as W
    from renderingengine_b200.traversal import Scene
    from renderingengine_b200.wavefront import FILM_MEAN, Renderer, frame_constants, plan_launches
    sl = W.batch_scenes(heightfield())
    views = W.batch_views(sl)
    objs = [Scene(sd.triangles, sd.fingerprint, 1, N.BUILD_LBVH, device=device) for sd, _, _, _ in sl]
    fcs, offs, off = [], [], 0
    for v in views:
        sel = sl[v.scene][1]
        est = N.ESTIMATOR_RESTIR_PRIMARY if v.restir else 2
        fcs.append([frame_constants(v.camera, v.width, v.height, k, W.BATCH_DEPTH, seed=v.seed, estimator=est,
                                    light_selection=sel) for k in range(v.spp)])
        offs.append(off)
        off += v.pixels
    total_paths = off
    samples = sum(v.pixels * v.spp for v in views)
    max_spp = max(v.spp for v in views)
    rb = Renderer(16384, (total_paths + 16383) // 16384, W.BATCH_DEPTH, device)
    rb.set_restir(**W.RESTIR_MANY_LIGHTS)
    for k, (sd, sel, _, _) in enumerate(sl):
        rb.bind_scene(k, objs[k], sd, light_selection=sel)
    plain = []
    for k, (sd, sel, restir, _) in enumerate(sl):
        r = Renderer(1920, 1080, W.BATCH_DEPTH, device)
        r.set_scene(objs[k], sd, light_selection=sel)
        r.set_restir(**W.RESTIR_MANY_LIGHTS)
        plain.append(r)
    stream = torch.cuda.Stream()
    launches = [0]
    budget = [8 << 20]

    def batched_step():
        # Sample k of every view that still needs one, in the planner's
        # launches (each scene's views together, at most `budget` paths).
        for k in range(max_spp):
            live = [i for i, v in enumerate(views) if v.spp > k]
            plan, count = plan_launches([views[i].scene for i in live], [views[i].pixels for i in live], budget[0])
            for l in range(count):
                vs = [dict(frame=fcs[i][k], slot=views[i].scene, offset=offs[i], accumulate=k > 0, key=i)
                      for i, pl in zip(live, plan) if pl == l]
                rb.render_views(vs, stream=stream.cuda_stream)
                launches[0] += 1

    def plain_step():
        for i, v in enumerate(views):
            r = plain[v.scene]
            for k in range(v.spp):
                r.render(fcs[i][k], accumulate=k > 0, stream=stream.cuda_stream)
                launches[0] += 1

    def rays(rs):
        t = [r.collect() for r in rs]
        return sum(x.total_path_rays + x.total_shadow_rays for x in t)

    def timed(step, rs):
        for _ in range(warmup):
            step()
        stream.synchronize()
        r0, launches[0] = rays(rs), 0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        stream.synchronize()
        ms = e0.elapsed_time(e1)
        return ms, rays(rs) - r0, launches[0]

    # Autotuner on the batched launch (these steps also warm up): the path
    # budget of one launch (queue capacity) and the launch configuration
    # (traversal loop / node width, traversal CTA size, Shade form, CTAs per
    # SM) by coordinate descent, one full step per candidate.
    from renderingengine_b200.autotune import autotune_batched

    def step_ms(cand):
        budget[0] = cand
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batched_step()
        e1.record(stream)
        stream.synchronize()
        return e0.elapsed_time(e1)

    space = {"traversal": (1, 2, 3, 4, 5, 6, 7, 8), "block": (128, 256, 512), "shade_variant": (3, 4, 5, 6, 7),
             "blocks_per_sm": (0, 4)}
    best, budget[0], tune_results = autotune_batched(
        rb, step_ms, (4 << 20, 8 << 20, 16 << 20, 32 << 20), space,
        store=Path(save_tuning) / "batched.json" if save_tuning else None)
    sweep = {r["budget"]: r["ms_per_frame"] for r in tune_results if r.get("budget") is not None
             and all(r[k] == v for k, v in (("traversal", 3), ("block", 128), ("shade_variant", 4),
                                            ("blocks_per_sm", 0)))}
    for p_r in plain:  # the plain arm runs the same launch configuration
        p_r.set_tuning(fuse=best.fuse, graph=True, blocks_per_sm=best.blocks_per_sm, block=best.block,
                       shade_variant=best.shade_variant, refill=best.refill, traversal=best.traversal)
    b_ms, b_rays, b_launches = timed(batched_step, [rb])
    p_ms, _, p_launches = timed(plain_step, plain)
    # Per-view device times of one more plain step: each scene's best
    # samples/s over its views gives what a perfect schedule of single-view
    # launches could reach.
    ev = []
    for i, v in enumerate(views):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(v.spp):
            plain[v.scene].render(fcs[i][k], accumulate=k > 0, stream=stream.cuda_stream)
        e1.record(stream)
        ev.append((e0, e1))
    stream.synchronize()
    view_ms = [a.elapsed_time(b) for a, b in ev]
    best_rate = {}
    for v, ms in zip(views, view_ms):
        best_rate[v.scene] = max(best_rate.get(v.scene, 0.0), v.pixels * v.spp / ms)
    ideal_ms = sum(v.pixels * v.spp / best_rate[v.scene] for v in views)
    # Film identity on the non-ReSTIR views (ReSTIR views depend on each
    # view's own history, which the plain renderers share between views).
    checked = 0
    for s in (0, 1, 3):
        i = min((i for i, v in enumerate(views) if v.scene == s), key=lambda i: views[i].pixels)
        v = views[i]
        r = plain[v.scene]
        for k in range(v.spp):
            r.render(fcs[i][k], accumulate=k > 0)
        r.collect()
        a = r.read(FILM_MEAN, v.pixels)
        b = rb.read_view(FILM_MEAN, offs[i], v.pixels)
        if not np.array_equal(a.view(np.uint32), b.view(np.uint32)):
            raise RuntimeError(f"batched film of view {i} differs from the plain film")
        checked += 1
    out = {
        "workload": "64 views over 4 scenes (Cornell 36 tris, heightfield 2,424,832, heightfield + 10k emissive "
                    "2,434,832 with ReSTIR DI, soup 500,000); res U{256^2,512^2,720p,1080p}, spp U{1,4,16}, "
                    "max bounce 6; LBVH",
        "views": len(views), "paths_per_launch_max": total_paths, "pixel_samples_per_step": samples,
        "steps": steps, "warmup": warmup,
        "batched": {"samples_per_s": round(samples * steps / (b_ms / 1e3), 1),
                    "mrays_per_s": round(b_rays / (b_ms / 1e3) / 1e6, 2),
                    "ms_per_step": round(b_ms / steps, 3), "launches_per_step": b_launches // steps},
        # The plain launches trace the same paths (identical films), so the
        # same rays; their renderers reset the running totals per view.
        "plain": {"samples_per_s": round(samples * steps / (p_ms / 1e3), 1),
                  "mrays_per_s": round(b_rays / (p_ms / 1e3) / 1e6, 2),
                  "ms_per_step": round(p_ms / steps, 3), "launches_per_step": p_launches // steps},
        "speedup_samples_per_s": round(p_ms / b_ms, 3),
        "schedule_only_gain": {
            "value": round(p_ms / steps / ideal_ms, 3),
            "how": "plain step time over the step time if every view ran at its scene's best single-view "
                   "samples/s (per-view CUDA-event times of one plain step): what reordering single-view "
                   "launches could gain; batched launches beyond it make each sample cheaper than any single "
                   "view of its scene renders it",
            "scene_best_msamples_per_s": {str(k): round(r / 1e3, 1) for k, r in sorted(best_rate.items())},
        },
        "launch_paths": budget[0],
        "launch_paths_sweep_ms": {str(k >> 20) + "Mi": round(v, 1) for k, v in sweep.items()},
        "tuning": {k: v for k, v in best.__dict__.items() if k != "ms_per_frame"},
        "tuning_candidates_timed": len(tune_results),
        "films_identical_checked_views": checked,
        "timing": "CUDA events on the launch stream around all steps",
    }
    for r in plain + [rb]:
        r.close()
    return out


# ---------------------------------------------------------------------------
# Many-light ReSTIR DI + SVGF reconstruction over a camera path
# ---------------------------------------------------------------------------
def run_reconstruction(device: int, frames: int = 60, warmup: int = 3) -> dict:
    """The heightfield scene plus 10,000 emissive triangles at 1280x720:
    per frame one ReSTIR DI path-traced sample (32 RIS candidates, temporal
    M-cap 20, one spatial pass of 5 neighbours in a 30-px disk, winner
    visibility; max bounce 8), the G-buffer / signal export with motion to the
    previous camera, and SVGF (5 A-Trous iterations, sigma_z 1, sigma_n 128,
    sigma_l 4) on a seeded 60-frame camera path.  Device time by CUDA events
    around all frames and between the three stages."""
    import torch

    from renderingengine_b200 import _native as N
    from renderingengine_b200 import scenes
    from renderingengine_b200 import workloads as W
    from renderingengine_b200.svgf import SvgfConfig, SvgfReconstruction
    from renderingengine_b200.traversal import Scene
    from renderingengine_b200.wavefront import Renderer, frame_constants
    w, h, depth = 1280, 720, 8
    n = w * h
    sd = scenes.add_emissive_triangles(heightfield(), count=10000)
    scene = Scene(sd.triangles, sd.fingerprint, 1, device=device)
    r = Renderer(w, h, depth, device)
    r.set_scene(scene, sd, light_selection=1)
    r.set_restir(**W.RESTIR_MANY_LIGHTS)
    svgf = SvgfReconstruction(w, h, 2, SvgfConfig(atrous_iterations=5, phi_depth=1.0, phi_normal=128.0,
                                                  phi_luminance=4.0), device=device)
    gb = torch.empty(n * N.GBUFFER_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    sig = torch.empty(n * N.SIGNAL_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    path = W.camera_path(sd.camera, frames + warmup, seed=0xC2)
    fcs = [frame_constants(c, w, h, k, depth, estimator=N.ESTIMATOR_RESTIR_PRIMARY, light_selection=1)
           for k, c in enumerate(path)]
    stream = torch.cuda.Stream()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(frames)]

    def frame(k, marks=None):
        if marks:
            marks[0].record(stream)
        r.render(fcs[k], accumulate=False, stream=stream.cuda_stream)
        if marks:
            marks[1].record(stream)
        r.export_reconstruction(fcs[k], fcs[k - 1] if k else None, gbuffer_ptr=gb.data_ptr(),
                                signal_ptr=sig.data_ptr(), stream=stream.cuda_stream)
        if marks:
            marks[2].record(stream)
        svgf.process_device(gb.data_ptr(), sig.data_ptr(), w, h, k, 0, stream=stream.cuda_stream)
        if marks:
            marks[3].record(stream)

    for k in range(warmup):
        frame(k)
    stream.synchronize()
    for j in range(frames):
        frame(warmup + j, ev[j])
    stream.synchronize()
    total = ev[0][0].elapsed_time(ev[-1][3])
    render = sum(e[0].elapsed_time(e[1]) for e in ev)
    export = sum(e[1].elapsed_time(e[2]) for e in ev)
    recon = sum(e[2].elapsed_time(e[3]) for e in ev)
    stats = r.restir_statistics()
    out = {
        "workload": "heightfield 2,424,832 tris + 10,000 emissive tris, 1280x720, ReSTIR DI (32 candidates, M-cap 20, "
                    "5 neighbours / 30 px, winner visibility), max bounce 8, SVGF 5 A-Trous iterations, "
                    f"{frames}-frame seeded camera path",
        "frames": frames, "warmup": warmup,
        "ms_per_frame": round(total / frames, 3), "fps": round(frames / (total / 1e3), 1),
        "render_ms": round(render / frames, 3), "export_ms": round(export / frames, 4),
        "svgf_ms": round(recon / frames, 3),
        "samples_per_s": round(n * frames / (total / 1e3), 1),
        "restir_temporal_accepted": int(stats.get("temporal_accepted", 0)),
        "timing": "CUDA events on the launch stream: first frame start to last frame end; stage sums",
    }
    r.close()
    svgf.close()
    return out


# ---------------------------------------------------------------------------
# Served request stream vs serial plain launches
# ---------------------------------------------------------------------------
def run_served(device: int, n_requests: int, rank: int = 0, world: int = 1) -> dict | None:
    """The first `n_requests` of the seeded Poisson stream (200 requests/s)
    over 16 scenes of 10k-5M triangles, (a) served: submitted with their
    arrival times to the render server (continuous batching over one path
    pool, HBM budget, LRU eviction) and drained; latency = device-timed
    completion - arrival; (b) serial plain: every request rendered alone on a
    single-view renderer, one launch per sample, its device time measured,
    then the requests queued first-in-first-out on those times.  With
    several ranks the router (renderingengine_b200/routing.py) gives each
    rank its share of the stream (least work first); times are relative to
    the stream's start on every rank and rank 0 merges the ranks' figures
    (it alone returns them)."""
    import torch

    from renderingengine_b200 import _native as N
    from renderingengine_b200 import workloads as W
    from renderingengine_b200.routing import gather_to_rank0, merge_served, shard_requests
    from renderingengine_b200.serving import RenderServer
    from renderingengine_b200.traversal import Scene
    from renderingengine_b200.wavefront import Renderer, frame_constants
    pool = W.serving_pool()
    datas = [r.build() for r in pool]
    stream_all = W.request_stream(n_requests, len(pool))
    mine = shard_requests([q.samples for q in stream_all], world, rank)
    reqs = [stream_all[i] for i in mine]
    free, _ = torch.cuda.mem_get_info(device)
    budget = int(min(150e9, free - 24e9))
    capacity = 1 << 25

    def fc(q, k):
        sd = datas[q.scene]
        return frame_constants(sd.camera, q.width, q.height, k, W.SERVE_DEPTH, seed=q.seed,
                               estimator=N.ESTIMATOR_RESTIR_PRIMARY if q.restir else 2)

    srv = RenderServer(budget, capacity, max_depth=W.SERVE_DEPTH, device=device, max_batch_views=256,
                       **W.RESTIR_MANY_LIGHTS)
    for k, sd in enumerate(datas):
        srv.register_scene(k, sd)
    # Warm-up: one small request per scene (scenes built and resident, graphs
    # captured), then the stream.
    for k, sd in enumerate(datas):
        for est in (2, N.ESTIMATOR_RESTIR_PRIMARY):
            srv.submit(k, frame_constants(sd.camera, 256, 256, 0, W.SERVE_DEPTH, estimator=est), 2)
    srv.drain()
    samples = sum(q.samples for q in reqs)

    def serve(scale: float) -> dict:
        """The requests submitted with their arrival times stretched by
        `scale`, drained; the server's figures over that stream."""
        st0 = srv.stats()
        t0 = srv.clock() + 0.05
        ids = [srv.submit(q.scene, fc(q, 0), q.spp, arrival_time=t0 + q.arrival * scale) for q in reqs]
        srv.drain()
        st1 = srv.stats()
        stat = [srv.poll(i) for i in ids]
        if any(s.state != N.REQUEST_DONE for s in stat):
            raise RuntimeError("served request failed: " +
                               str([s.error for s in stat if s.state != N.REQUEST_DONE][:4]))
        out = {"samples": samples, "first_arrival": min(q.arrival for q in reqs) * scale,
               "last_completion": max(s.completion_time for s in stat) - t0,
               "latencies": [s.completion_time - s.arrival_time for s in stat],
               "rays": st1["path_rays"] + st1["shadow_rays"] - st0["path_rays"] - st0["shadow_rays"],
               "launches": st1["launches"] - st0["launches"], "scene_builds": st1["scene_builds"],
               "evictions": st1["evictions"], "resident_bytes": st1["resident_bytes"]}
        for i in ids:
            srv.release(i)
        return out

    part = serve(1.0)
    # The same requests offered at 80 % of the rate this server just
    # sustained (requests / s = its samples / s over the mean request), so
    # latency is service plus moderate queueing rather than the backlog of
    # an overloaded stream.
    rate = W.SERVE_RATE
    capacity_rps = samples / (part["last_completion"] - part["first_arrival"]) / (samples / len(reqs))
    sustained_rate = 0.8 * capacity_rps
    stretch = rate / sustained_rate
    part_sustained = serve(stretch)
    srv.close()
    del srv

    # Serial plain: per-request device time, grouped by scene to avoid
    # rebinding (binding is host work outside the timed region anyway).
    r = Renderer(1920, 1080, W.SERVE_DEPTH, device)
    r.set_restir(**W.RESTIR_MANY_LIGHTS)
    stream = torch.cuda.Stream()
    durations = np.zeros(len(reqs))
    order = sorted(range(len(reqs)), key=lambda i: reqs[i].scene)
    current, events = None, []
    for i in order:
        q = reqs[i]
        if q.scene != current:
            stream.synchronize()
            scene = Scene(datas[q.scene].triangles, datas[q.scene].fingerprint, 1, N.BUILD_LBVH, device=device)
            r.set_scene(scene, datas[q.scene])
            r.render(fc(q, 0), accumulate=False, stream=stream.cuda_stream)  # warm-up of this scene
            current = q.scene
        if q.restir:
            r.restir_reset()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(q.spp):
            r.render(fc(q, k), accumulate=k > 0, stream=stream.cuda_stream)
        e1.record(stream)
        events.append((i, e0, e1))
        if len(events) >= 64:
            stream.synchronize()
            for j, a, b in events:
                durations[j] = a.elapsed_time(b) / 1e3
            events = []
    stream.synchronize()
    for j, a, b in events:
        durations[j] = a.elapsed_time(b) / 1e3
    r.close()
    arrivals = np.array([q.arrival for q in reqs])

    def plain_fifo(scale: float) -> dict:
        a = arrivals * scale
        plat, _ = W.fifo_latencies(a, durations)
        return {"samples": samples, "first_arrival": float(a.min()), "last_completion": float((a + plat).max()),
                "latencies": list(plat), "busy_s": float(durations.sum()), "launches": int(sum(q.spp for q in reqs))}

    plain_part = plain_fifo(1.0)
    plain_sustained = plain_fifo(stretch)

    parts = gather_to_rank0({"served": part, "plain": plain_part, "served_s": part_sustained,
                             "plain_s": plain_sustained, "rate_s": sustained_rate})
    if parts is None:
        return None
    sv = merge_served([p["served"] for p in parts])
    pl = merge_served([p["plain"] for p in parts])
    sv_s = merge_served([p["served_s"] for p in parts])
    pl_s = merge_served([p["plain_s"] for p in parts])
    served = {"samples_per_s": round(sv["samples_per_s"], 1),
              "mrays_per_s": round(sum(p["served"]["rays"] for p in parts) / sv["makespan_s"] / 1e6, 2),
              "makespan_s": round(sv["makespan_s"], 3), "latency_p50_ms": round(sv["latency_p50_s"] * 1e3, 3),
              "latency_p99_ms": round(sv["latency_p99_s"] * 1e3, 3),
              "latency_mean_ms": round(sv["latency_mean_s"] * 1e3, 3),
              "launches": sum(p["served"]["launches"] for p in parts),
              "scene_builds": sum(p["served"]["scene_builds"] for p in parts),
              "evictions": sum(p["served"]["evictions"] for p in parts),
              "resident_bytes": max(p["served"]["resident_bytes"] for p in parts), "budget_bytes": budget,
              "path_capacity": capacity}
    plain = {"samples_per_s": round(pl["samples_per_s"], 1),
             "busy_samples_per_s": round(pl["samples"] / max(p["plain"]["busy_s"] for p in parts), 1),
             "makespan_s": round(pl["makespan_s"], 3), "latency_p50_ms": round(pl["latency_p50_s"] * 1e3, 3),
             "latency_p99_ms": round(pl["latency_p99_s"] * 1e3, 3),
             "latency_mean_ms": round(pl["latency_mean_s"] * 1e3, 3),
             "launches": sum(p["plain"]["launches"] for p in parts)}
    return {
        "workload": (f"first {n_requests} requests of a seeded Poisson stream (200 req/s) over 16 scenes of "
                     "10k-5M tris (heightfields + soups); res U{256^2,720p,1080p}, spp U{1,8,64}, ReSTIR p=0.5, "
                     "max bounce 6; LBVH"),
        "requests": n_requests, "pixel_samples": sv["samples"],
        "routing": {"ranks": world, "policy": "balanced (least assigned work first)"},
        "served": served, "serial_plain": plain,
        "speedup_samples_per_s": round(served["samples_per_s"] / plain["samples_per_s"], 3),
        "sustained": {
            "offered_req_per_s": round(sum(p["rate_s"] for p in parts), 3),
            "how": "the same requests with arrival times stretched to 80 % of the request rate the server "
                   "sustained on the stream above",
            "served": {"latency_p50_ms": round(sv_s["latency_p50_s"] * 1e3, 3),
                       "latency_p99_ms": round(sv_s["latency_p99_s"] * 1e3, 3),
                       "latency_mean_ms": round(sv_s["latency_mean_s"] * 1e3, 3),
                       "makespan_s": round(sv_s["makespan_s"], 3)},
            "serial_plain": {"latency_p50_ms": round(pl_s["latency_p50_s"] * 1e3, 3),
                             "latency_p99_ms": round(pl_s["latency_p99_s"] * 1e3, 3),
                             "latency_mean_ms": round(pl_s["latency_mean_s"] * 1e3, 3),
                             "makespan_s": round(pl_s["makespan_s"], 3)},
        },
        "timing": "served: CUDA-event completion times minus arrival; plain: CUDA-event device time per request, "
                  "queued FIFO on the arrival times; both relative to the stream start on every rank",
    }


def run_reference(args, rank: int, world: int) -> None:
    """CPU arm: the same workload on the host cores, one bounded sample per
    step.  The scene comes from the same seeded generator, its hierarchy from
    the reference's own CPU builders (oracle/_ref); neither the GPU nor the
    product library is touched."""
    if rank != 0:
        return
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "metric": METRIC,
                          "unavailable": "reference CPU oracle library (oracle/_ref) not built"}))
        return
    sd = heightfield()
    build = "sah" if args.workload == "trace" else args.build  # the trace workload traces the SAH
    nodes, order = reference_hierarchy(sd, build)
    from renderingengine_b200 import scenes
    if args.workload == "trace":
        kind, what = "reference", "SoftwareGpu::Trace (reference CPU mirror, oracle/_ref)"
        arm = CpuTraceArm(sd, nodes, order, scenes.pinhole_rays(sd.camera, 1920, 1080, seed=1))
        name, sample = TraceWorkload.name, 1920 * 1080
    else:
        # The reference has no CPU implementation of its PBR wavefront path
        # (its CPU integrator is the Lambert-only Cornell fixture), so the CPU
        # arm is the FP32 restatement of that path (oracle/oracle_pbr.cpp)
        # over the hierarchy the reference's own builder made.
        from renderingengine_b200.wavefront import frame_constants
        kind, what = "port", "FP32 CPU port of the wavefront PBR frame (oracle/oracle_pbr.cpp)"
        arm = CpuFrameArm(sd, nodes, order, frame_constants(sd.camera, 1920, 1080, 0, 8))
        name, sample = frame_workload_name(args.build), 1920 * 1080
    builder = ("SoftwareGpu::BuildKarrasLbvh" if build == "lbvh"
               else "Bvh<float> binned SAH + FlattenCanonicalL3BinnedSah")
    # Each step: the whole frame (or ray batch) on all host threads, ~1.6 s
    # of the 16-core host for the frame.
    for _ in range(args.warmup):
        arm.run(max(1024, sample // 8), threads)
    units, secs = 0, 0.0
    for _ in range(args.steps):
        n, s = arm.run(sample, threads)
        units += n
        secs += s
    value = units / secs / 1e6
    desc = f"{sample} pixels of the frame per step" if args.workload == "frame" else f"{sample} rays per step"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "Mrays/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(secs / args.steps * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators, benchmark shapes)",
        "config": {"workload": name, "sample": desc, "host_threads": threads,
                   "hierarchy": f"{builder} (reference CPU code, oracle/_ref)"},
        "cpu_baseline": {"value": round(value, 4), "unit": "Mrays/s", "cores": threads, "kind": kind,
                         "sample": f"{desc}; {what}"},
        "e2e": {"value": round(value, 4), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="frame", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--build", default="lbvh", choices=["lbvh", "sah"],
                    help="frame workload hierarchy: GPU LBVH (the traversal-bound configuration) or flattened SAH")
    ap.add_argument("--no-graph", action="store_true",
                    help="launch the frame's stages directly instead of replaying a CUDA graph "
                         "(for kernel-level profiling)")
    ap.add_argument("--fuse", type=int, default=None, help="1: fused Intersect+Shade, 0: split")
    ap.add_argument("--shade-variant", type=int, default=4,
                    help="Shade kernel form with --no-graph / --fuse (0 one kernel, 4 split in two)")
    ap.add_argument("--traversal", type=int, default=3,
                    help="traversal loop with --no-graph / --fuse (0 reference, 1 while-while, 2 four-wide, "
                         "3 per launch, 4 four-wide one step at a time, 5 eight-wide, 6 eight-wide compressed, "
                         "7 / 8 modes 4 / 2 with the conservative one-fma slab test)")
    ap.add_argument("--block", type=int, default=128, choices=[128, 256, 512],
                    help="traversal CTA size with --no-graph / --fuse")
    ap.add_argument("--no-tune", action="store_true", help="skip the launch-configuration autotuner")
    ap.add_argument("--tuning", default=None,
                    help="use a stored tuning (a JSON file written by --save-tuning, or the name of one of the "
                         "package's tuned configurations) instead of running the autotuner")
    ap.add_argument("--save-tuning", default=None, metavar="DIR",
                    help="write the tunings the run chose (frame_<build>.json, batched.json) into DIR")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-views comparison")
    ap.add_argument("--no-served", action="store_true", help="skip the served-stream comparison")
    ap.add_argument("--no-reconstruction", action="store_true",
                    help="skip the many-light ReSTIR + SVGF camera-path measurement")
    ap.add_argument("--batch-steps", type=int, default=2, help="timed steps of the batched comparison")
    ap.add_argument("--serve-requests", type=int, default=150, help="requests of the served-stream sample")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    from renderingengine_b200 import build as B
    if rank == 0:
        B.build()
    if world > 1:
        dist.barrier()
    wl = WORKLOADS[args.workload](local, build=args.build)
    tuning = None
    if hasattr(wl, "r"):
        if args.no_graph or args.fuse is not None:
            wl.r.set_tuning(fuse=bool(args.fuse), graph=not args.no_graph, traversal=args.traversal,
                            shade_variant=args.shade_variant, block=args.block)
        elif args.tuning:
            from renderingengine_b200 import autotune as AT
            best = AT.load(args.tuning)
            AT.apply(wl.r, best)
            tuning = {"loaded": args.tuning, **{k: v for k, v in best.__dict__.items() if k != "ms_per_frame"}}
        elif not args.no_tune:
            from renderingengine_b200.autotune import autotune
            best = autotune(wl.r, [wl._fc(1000 + k) for k in range(2)],
                            store=Path(args.save_tuning) / f"frame_{args.build}.json" if args.save_tuning else None)
            tuning = {"fuse_intersect_shade": best.fuse, "shade_variant": best.shade_variant,
                      "blocks_per_sm": best.blocks_per_sm, "refill": best.refill, "traversal": best.traversal,
                      "block": best.block, "graph": best.graph,
                      "tuned_ms_per_frame": round(best.ms_per_frame, 4)}
    if hasattr(wl, "run_profile") and (tuning is not None or args.no_graph or args.fuse is not None):
        wl.run_profile()  # the stage profile of the configuration the run times
    stream = torch.cuda.Stream()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        with torch.cuda.stream(stream):
            wl.step_device(stream)
    stream.synchronize()
    units0 = frames0 = 0
    if hasattr(wl, "reset_counts"):
        wl.reset_counts()
        units0, frames0 = wl.measured_units()

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    barrier()
    start.record(stream)
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            wl.step_device(stream)
    end.record(stream)
    stream.synchronize()
    barrier()
    time.sleep(0.2)
    clocks = sampler.stop()
    ms = start.elapsed_time(end)
    if hasattr(wl, "measured_units"):
        # Rays actually traced in the timed frames (device-side running totals).
        units1, frames1 = wl.measured_units()
        assert frames1 - frames0 == args.steps, (frames0, frames1, args.steps)
        units_rank = units1 - units0
    else:
        units_rank = wl.units_per_step() * args.steps
    from renderingengine_b200.routing import max_time_sum_work
    ms_max, units = max_time_sum_work(ms, float(units_rank))  # slowest rank's time, every rank's rays
    value = units / (ms_max / 1e3) / 1e6

    # End-to-end through the C ABI with pinned host buffers.
    for _ in range(2):
        wl.step_e2e()
    torch.cuda.synchronize()
    e2e_steps = max(3, args.steps // 2)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        wl.step_e2e()
    if hasattr(wl, "finish_e2e"):
        wl.finish_e2e()  # the last step's result has reached the host
    torch.cuda.synchronize()
    e2e_s, _ = max_time_sum_work(time.perf_counter() - t0, 0.0)
    per_step_units = units / world / args.steps
    e2e_value = per_step_units * e2e_steps * world / e2e_s / 1e6
    h2d, d2h = wl.bytes_per_step()

    peak, peak_kind = measured_peak_hbm()
    # L2-relative view: the traversal's algorithmic bytes are mostly served
    # from L1 / L2 (DRAM carries a few percent), so the same achieved rate
    # is also given against the L2 bandwidth measured here.
    try:
        l2_gbs = measure_l2_gbs()
    except Exception as exc:  # reported, never required
        l2_gbs = None
        l2_err = f"{type(exc).__name__}: {exc}"
    if hasattr(wl, "roofline_stage"):
        alg, secs, launches = wl.roofline_stage()
        achieved = alg / secs / 1e9
        kernel = "k_intersect (all bounces of one frame, split launch)"
    else:
        # One trace launch per step: its event time is the step's.
        alg = wl.algorithmic_bytes()
        achieved = alg / (ms_max / args.steps / 1e3) / 1e9
        kernel = "trace_batch_kernel (one launch per step)"
    l2_view = ({"peak": round(l2_gbs, 1), "unit": "GB/s", "frac": round(achieved / l2_gbs, 4),
                "how": "device copy of a 24 MiB L2-resident buffer, read + write bytes, best of 3 x 100, CUDA events"}
               if l2_gbs else {"unavailable": l2_err})
    extra = {}
    if args.workload == "frame":
        extra["samples_per_s"] = round(wl.n * args.steps * world / (ms_max / 1e3), 1)
        extra["stage_ms"] = {k: [round(x, 4) for x in v] if isinstance(v, list) else round(v, 4)
                             for k, v in wl.prof.items() if k.endswith("_ms")}
        extra["rays_per_bounce"] = wl.prof["rays"]
        extra["shadows_per_bounce"] = wl.prof["shadows"]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            sample = wl.n  # the whole frame / ray batch once
            n, s = wl.cpu_reference(sample, threads)
            kind = "port" if args.workload == "frame" else "reference"
            cpu = {"value": round(n / s / 1e6, 4), "unit": "Mrays/s", "cores": threads, "kind": kind,
                   "sample": (f"{sample} pixels of the frame, FP32 CPU port (oracle/oracle_pbr.cpp)"
                              if args.workload == "frame" else
                              f"{sample} camera rays, SoftwareGpu::Trace (oracle/_ref)")}
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "Mrays/s", "cores": 0, "kind": "port", "sample": f"unavailable: {exc}"}
    comparisons = {}
    if args.workload == "frame":
        # Every rank runs the comparisons (replicas); rank 0 reports its own.
        wl.r.close()
        for name, fn in (("batched", lambda: run_batched(local, 3, args.batch_steps, args.save_tuning)),
                         ("served", lambda: run_served(local, args.serve_requests, rank, world)),
                         ("reconstruction", lambda: run_reconstruction(local))):
            if getattr(args, "no_" + name):
                continue
            try:
                comparisons[name] = fn()
            except Exception as exc:  # reported, never silently dropped
                comparisons[name] = {"error": f"{type(exc).__name__}: {exc}"}
            import gc
            gc.collect()
            torch.cuda.empty_cache()
    if rank == 0:
        traffic = (None, "trace workload: no capture")
        if args.workload == "frame":
            layout = intersect_layout(wl.build, getattr(wl.r, "tuning", {}).get("traversal", 3))
            traffic = INTERSECT_DRAM_BYTES_PER_FRAME.get((wl.build, layout), (None, f"no capture for {layout} nodes"))
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generators, benchmark shapes)",
            "config": {"workload": wl.name, "tuning": tuning,
                       "l2": "no flush: inputs larger than the 126 MB L2 (hierarchy + triangles > 460 MB, "
                             "path state ~1 GB)",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": round(e2e_value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "achieved": None if achieved is None else round(achieved, 1),
                         "peak": peak, "unit": "GB/s",
                         "frac": None if achieved is None else round(achieved / peak, 4),
                         "traffic": traffic[0], "traffic_source": traffic[1],
                         "traffic_unit": "bytes per frame (8 launches), ncu dram__bytes_read + write",
                         "peak_kind": peak_kind, "kernel": kernel, "algorithmic_bytes_per_frame": alg,
                         "l2": l2_view},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": args.steps * frame_kernels(getattr(wl.r, "tuning", {}), wl.depth) if args.workload == "frame"
            else args.steps,
            **extra,
            **comparisons,
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
