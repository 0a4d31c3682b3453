"""Autotuner of the wavefront launch configuration.

Tunes the runtime axes of a renderer on a representative workload -- the
Intersect/Shade split point (separate kernels vs one fused kernel), the
Shade register/call-site variant, the number of persistent CTAs per SM, the
traversal kernels' CTA size (128, 256 or 512 threads), the traversal loop and
node width (reference and while-while loops over binary child-pair nodes,
four-wide nodes with or without postponed leaves, with the exact or the
conservative one-fma slab test, eight-wide nodes plain or compressed to 8-bit
child boxes, lane refill over child pairs or four-wide nodes)
and, for batched launches, the path budget of one launch (the queue
capacity) -- timing each candidate on the device with CUDA events.

The search is coordinate descent: starting from a default configuration,
each axis in turn is swept with the others held, keeping the fastest value,
until a full pass changes nothing (at most `passes` passes).  Results are
bit-identical across candidates (per-path RNG is counter based;
tests/test_wavefront_gpu.py checks every axis), so only time is compared.
"""
from __future__ import annotations

import json
from dataclasses import asdict, dataclass, replace
from pathlib import Path

import numpy as np


@dataclass
class Tuning:
    fuse: bool = False
    shade_variant: int = 4
    blocks_per_sm: int = 0
    refill: int = 0
    traversal: int = 3
    block: int = 128
    graph: bool = True
    ms_per_frame: float = float("nan")


DEFAULT_SPACE = {
    "traversal": (0, 1, 2, 3, 4, 5, 6, 7, 8),
    "block": (128, 256, 512),
    "shade_variant": (0, 3, 4, 5, 6, 7),
    "fuse": (False, True),
    "blocks_per_sm": (0, 4),
    "refill": (0, 8, 16),
}


def valid(t: Tuning) -> bool:
    if t.fuse and (t.refill or t.traversal != 0):
        return False  # the fused kernel traverses child pairs inside Shade (the reference loop, no refill)
    if t.refill and t.traversal not in (1, 4):
        return False  # lane refill steps one node or leaf at a time: child pairs (1) or four-wide (4)
    return True


def apply(renderer, t: Tuning) -> None:
    renderer.set_tuning(fuse=t.fuse, graph=t.graph, blocks_per_sm=t.blocks_per_sm, block=t.block,
                        shade_variant=t.shade_variant, refill=t.refill, traversal=t.traversal)


def _time_frames(renderer, frames, repeats: int) -> float:
    import torch
    stream = torch.cuda.Stream()
    for f in frames[:1]:
        renderer.render(f, accumulate=True, stream=stream.cuda_stream)
    stream.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(repeats):
        renderer.render(frames[k % len(frames)], accumulate=True, stream=stream.cuda_stream)
    e1.record(stream)
    stream.synchronize()
    return e0.elapsed_time(e1) / repeats


def coordinate_descent(measure, start: Tuning, space: dict, passes: int = 2):
    """Minimises measure(tuning) -> ms over the axes of `space` one at a time.
    Returns (best tuning, [(tuning dict, ms)] of every candidate timed)."""
    seen = {}

    def cost(t: Tuning) -> float:
        key = tuple(sorted((k, v) for k, v in asdict(t).items() if k != "ms_per_frame"))
        if key not in seen:
            seen[key] = (asdict(t), measure(t))
        return seen[key][1]

    best = start
    best_ms = cost(best)
    for _ in range(passes):
        changed = False
        for axis, values in space.items():
            for v in values:
                cand = replace(best, **{axis: v})
                if not valid(cand):
                    continue
                ms = cost(cand)
                if ms < best_ms:
                    best, best_ms, changed = cand, ms, True
        if not changed:
            break
    best = replace(best, ms_per_frame=best_ms)
    return best, [dict(d, ms_per_frame=ms) for d, ms in seen.values()]


def autotune(renderer, frames: list[np.ndarray], space: dict | None = None, repeats: int = 3,
             store: Path | None = None, passes: int = 2) -> Tuning:
    """The fastest tuning for `frames` (a list of frame-constant records) on
    one renderer; the renderer is left set to it, with its film reset."""
    space = dict(DEFAULT_SPACE if space is None else space)

    def measure(t: Tuning) -> float:
        apply(renderer, t)
        return _time_frames(renderer, frames, repeats)

    best, results = coordinate_descent(measure, Tuning(), space, passes)
    apply(renderer, best)
    renderer.render(frames[0], accumulate=False)
    renderer.collect()
    if store is not None:
        save(store, best, "frame", results)
    return best


TUNED_DIR = Path(__file__).resolve().parent / "tuned"


def save(path: Path, best: Tuning, workload: str, candidates: list | None = None, **extra) -> None:
    """Writes a tuning as JSON: the chosen configuration, the workload it was
    tuned on, the device and any further keys (e.g. the batched launch's path
    budget), with the candidates timed."""
    import torch
    dev = torch.cuda.get_device_name() if torch.cuda.is_available() else None
    Path(path).write_text(json.dumps({"workload": workload, "device": dev, "best": asdict(best), **extra,
                                      "candidates": candidates or []}, indent=1))


def load(path: Path | str) -> Tuning:
    """The tuning stored by save() (a bare name is looked up among the
    package's tuned configurations)."""
    p = Path(path)
    if not p.exists() and not p.suffix:
        p = TUNED_DIR / f"{path}.json"
    d = json.loads(p.read_text())["best"]
    fields = set(Tuning.__dataclass_fields__)
    t = Tuning(**{k: v for k, v in d.items() if k in fields})
    if not valid(t):
        raise ValueError(f"{p}: invalid tuning {d}")
    return t


def autotune_batched(renderer, step, budgets, space: dict | None = None, store: Path | None = None,
                     passes: int = 1):
    """Tunes a batched launch: `step(budget)` renders one full step (every
    view's samples in launches of at most `budget` paths) and returns its
    device milliseconds.  The path budget (queue capacity) is one more axis
    of the coordinate descent.  Returns (best tuning, best budget, results)."""
    space = dict(DEFAULT_SPACE if space is None else space)
    budgets = tuple(budgets)
    state = {"budget": budgets[0]}

    def measure(t: Tuning) -> float:
        apply(renderer, t)
        return step(state["budget"])

    best = Tuning()
    best_budget = budgets[0]
    results = []
    for _ in range(max(1, passes)):
        # Budget axis with the tuning held.
        apply(renderer, best)
        times = {b: step(b) for b in budgets}
        best_budget = min(times, key=times.get)
        results += [dict(asdict(best), budget=b, ms_per_frame=ms) for b, ms in times.items()]
        state["budget"] = best_budget
        best, res = coordinate_descent(measure, best, space, passes=1)
        results += [dict(r, budget=best_budget) for r in res]
    apply(renderer, best)
    if store is not None:
        save(store, best, "batched", results, budget=best_budget)
    return best, best_budget, results
