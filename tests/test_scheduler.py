"""The render server's host bookkeeping (csrc/scheduler.h), compiled on the
CPU: first-fit path ranges with coalescing, and least-recently-used victim
choice that never picks a pinned scene."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def sched(tmp_path_factory):
    out = tmp_path_factory.mktemp("sched") / "libsched.so"
    subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I", str(ROOT / "renderingengine_b200" / "csrc"),
                    str(ROOT / "tests" / "native" / "scheduler_harness.cpp"), "-o", str(out)], check=True)
    lib = C.CDLL(str(out))
    P, U32, U64 = C.c_void_p, C.c_uint32, C.c_uint64
    for name, res, args in [
        ("alloc_create", P, [U32]), ("alloc_destroy", None, [P]), ("alloc_take", C.c_int, [P, U32, C.POINTER(U32)]),
        ("alloc_give", None, [P, U32, U32]), ("alloc_used", U32, [P]), ("alloc_largest", U32, [P]),
        ("alloc_fragments", U64, [P]), ("lru_create", P, []), ("lru_destroy", None, [P]),
        ("lru_insert", None, [P, U64, U64, U64]), ("lru_touch", None, [P, U64, U64]), ("lru_pin", None, [P, U64]),
        ("lru_unpin", None, [P, U64]), ("lru_erase", None, [P, U64]), ("lru_bytes", U64, [P]),
        ("lru_victims", U32, [P, U64, P, U32])]:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def test_allocator_random_sequences(sched):
    """Random allocate / release sequences against an interval model: ranges
    never overlap, stay in bounds, first fit is the lowest fitting offset,
    and releasing everything coalesces back to one free range."""
    rng = np.random.default_rng(1)
    cap = 100_000
    a = sched.alloc_create(cap)
    live = {}
    for step in range(4000):
        if live and rng.random() < 0.45:
            off = int(rng.choice(list(live)))
            sched.alloc_give(a, off, live.pop(off))
        else:
            size = int(rng.integers(1, 9000))
            occupied = np.zeros(cap, bool)
            for o, n in live.items():
                occupied[o:o + n] = True
            # lowest offset with `size` free positions in a row
            expect = None
            run = 0
            for i in range(cap):
                run = run + 1 if not occupied[i] else 0
                if run == size:
                    expect = i - size + 1
                    break
            off = C.c_uint32()
            ok = sched.alloc_take(a, size, C.byref(off))
            assert bool(ok) == (expect is not None)
            if ok:
                assert off.value == expect
                live[off.value] = size
        assert sched.alloc_used(a) == sum(live.values())
        if step % 500 == 0:
            spans = sorted(live.items())
            for (o1, n1), (o2, _) in zip(spans, spans[1:]):
                assert o1 + n1 <= o2
    for off, n in list(live.items()):
        sched.alloc_give(a, off, n)
    assert sched.alloc_used(a) == 0 and sched.alloc_largest(a) == cap and sched.alloc_fragments(a) == 1
    sched.alloc_destroy(a)


def test_lru_victims_skip_pinned(sched):
    l = sched.lru_create()
    for key, (size, stamp) in enumerate([(100, 5), (200, 1), (300, 3), (400, 2)]):
        sched.lru_insert(l, key, size, stamp)
    assert sched.lru_bytes(l) == 1000
    out = (C.c_uint64 * 8)()
    n = sched.lru_victims(l, 700, out, 8)
    assert list(out[:n]) == [1, 3]  # oldest first: stamps 1 (200 B), 2 (400 B) -> total 400 <= 700
    sched.lru_pin(l, 3)
    n = sched.lru_victims(l, 700, out, 8)
    assert list(out[:n]) == [1, 2]  # pinned 3 skipped: 200 B + 300 B -> 500 <= 700
    assert sched.lru_victims(l, 300, out, 8) == 0  # only 600 B unpinned: cannot reach 300
    sched.lru_touch(l, 1, 10)
    n = sched.lru_victims(l, 900, out, 8)
    assert list(out[:n]) == [2]
    sched.lru_unpin(l, 3)
    sched.lru_erase(l, 2)
    assert sched.lru_bytes(l) == 700
    sched.lru_destroy(l)


def test_launch_plan_groups_scenes_under_the_path_budget(native):
    """re_plan_launches against a model: each scene's views, in order, cut
    into chunks of at most the path budget (a larger view alone), chunks
    placed first-fit into launches of at most the budget; scenes in the
    order of their first view."""
    from renderingengine_b200.wavefront import plan_launches
    rng = np.random.default_rng(7)
    for trial in range(300):
        n = int(rng.integers(0, 60))
        slots = rng.integers(0, 6, n).astype(np.uint32)
        pixels = rng.choice([65536, 262144, 921600, 2073600, 10, 5_000_000], n).astype(np.uint32)
        budget = int(rng.choice([1, 1 << 20, 4 << 20, 16 << 20, 64 << 20]))
        plan, count = plan_launches(slots, pixels, budget)
        seen = []
        for s in slots.tolist():
            if s not in seen:
                seen.append(s)
        chunks = []
        for s in seen:
            cur, used = [], 0
            for i in np.flatnonzero(slots == s):
                if cur and used + int(pixels[i]) > budget:
                    chunks.append((cur, used))
                    cur, used = [], 0
                cur.append(i)
                used += int(pixels[i])
            chunks.append((cur, used))
        fill, want = [], np.zeros(n, np.uint32)
        for members, used in chunks:
            l = next((k for k, f in enumerate(fill) if f + used <= budget), len(fill))
            if l == len(fill):
                fill.append(0)
            fill[l] += used
            want[members] = l
        assert count == len(fill)
        np.testing.assert_array_equal(plan, want)
        for l in range(count):
            members = np.flatnonzero(plan == l)
            assert len(members) == 1 or int(pixels[members].astype(np.int64).sum()) <= budget
