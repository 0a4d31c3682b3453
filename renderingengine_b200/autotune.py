"""Autotuner of the wavefront launch configuration.

Sweeps the runtime tuning axes of a renderer on a representative frame --
the Intersect/Shade split point (separate kernels vs one fused kernel), the
Shade register/call-site variant, the number of persistent CTAs per SM, the
traversal loop (reference, while-while with postponed leaves, four-wide
nodes, lane refill over child pairs or four-wide nodes) and
CUDA-graph replay -- timing each candidate on the device with CUDA events
over a few frames, and returns (and optionally stores) the fastest.  The film
is reset afterwards; results are bit-identical across candidates (per-path
RNG is counter based), which tests/test_wavefront_gpu.py checks.
"""
from __future__ import annotations

import itertools
import json
from dataclasses import asdict, dataclass
from pathlib import Path

import numpy as np


@dataclass
class Tuning:
    fuse: bool = False
    shade_variant: int = 0
    blocks_per_sm: int = 0
    refill: int = 0
    traversal: int = 0
    graph: bool = True
    ms_per_frame: float = float("nan")


DEFAULT_SPACE = {
    "fuse": (False, True),
    "shade_variant": (0, 3, 4, 5),
    "blocks_per_sm": (0, 4),
    "refill": (0, 8, 16),
    "traversal": (1, 2, 3, 4),
}


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


def autotune(renderer, frames: list[np.ndarray], space: dict | None = None, repeats: int = 3,
             store: Path | None = None) -> Tuning:
    """Returns the fastest tuning for `frames` (a list of frame-constant records)."""
    space = dict(DEFAULT_SPACE if space is None else space)
    best = None
    results = []
    for fuse, variant, bps, refill, trav in itertools.product(space["fuse"], space["shade_variant"],
                                                              space["blocks_per_sm"], space["refill"],
                                                              space.get("traversal", (0,))):
        if fuse and (refill or trav):
            continue  # the fused kernel traverses inside Shade (no refill or while-while form)
        if refill and trav not in (1, 4):
            continue  # lane refill steps one node or leaf at a time: child pairs (1) or four-wide nodes (2-4 alike)
        renderer.set_tuning(fuse=fuse, graph=True, blocks_per_sm=bps, shade_variant=variant, refill=refill,
                            traversal=trav)
        ms = _time_frames(renderer, frames, repeats)
        t = Tuning(fuse, variant, bps, refill, trav, True, ms)
        results.append(asdict(t))
        if best is None or ms < best.ms_per_frame:
            best = t
    renderer.set_tuning(fuse=best.fuse, graph=True, blocks_per_sm=best.blocks_per_sm,
                        shade_variant=best.shade_variant, refill=best.refill, traversal=best.traversal)
    renderer.render(frames[0], accumulate=False)
    renderer.collect()
    if store is not None:
        Path(store).write_text(json.dumps({"best": asdict(best), "candidates": results}, indent=2))
    return best
