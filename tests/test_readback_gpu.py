"""Asynchronous film reads (re_renderer_read_view_async / re_renderer_wait_reads):
the read of frame k lands in host memory while frame k + 1 renders, and every
read equals the synchronous read of the same frame."""
import numpy as np
import pytest
import torch

from renderingengine_b200 import _native as N
from renderingengine_b200 import scenes
from renderingengine_b200.traversal import Scene
from renderingengine_b200.wavefront import FILM_MEAN, FILM_SAMPLE, Renderer, frame_constants

pytestmark = pytest.mark.gpu


def _pinned(pixels):
    return torch.zeros((pixels, 4), dtype=torch.float32).pin_memory().numpy()


def test_async_reads_equal_synchronous_reads(native):
    sd = scenes.heightfield_scene(grid=64, spheres=64, seed=7)
    w, h, depth = 160, 96, 6
    n = w * h
    scene = Scene(sd.triangles, sd.fingerprint, 1, N.BUILD_LBVH)
    frames = [frame_constants(sd.camera, w, h, f, depth, seed=0x5151) for f in range(5)]
    # Synchronous reads after each frame.
    ref = Renderer(w, h, depth)
    ref.set_scene(scene, sd)
    want_sample, want_mean = [], []
    for f, fc in enumerate(frames):
        ref.render(fc, accumulate=f > 0)
        ref.collect()
        want_sample.append(ref.read(FILM_SAMPLE, n))
        want_mean.append(ref.read(FILM_MEAN, n))
    # Asynchronous: every frame queued back to back, its reads started
    # without waiting (more reads in flight than staging buffers).
    r = Renderer(w, h, depth)
    r.set_scene(scene, sd)
    got_sample = [_pinned(n) for _ in frames]
    got_mean = [_pinned(n) for _ in frames]
    for f, fc in enumerate(frames):
        r.render(fc, accumulate=f > 0)
        r.read_async(FILM_SAMPLE, got_sample[f])
        r.read_async(FILM_MEAN, got_mean[f])
    r.wait_reads()
    assert r.collect().fatal_mask == 0
    for f in range(len(frames)):
        np.testing.assert_array_equal(got_sample[f].view(np.uint32), want_sample[f].view(np.uint32), err_msg=str(f))
        np.testing.assert_array_equal(got_mean[f].view(np.uint32), want_mean[f].view(np.uint32), err_msg=str(f))
    # A view range, and the contract checks.
    part = _pinned(1000)
    r.read_async(FILM_SAMPLE, part, offset=n - 1000)
    r.wait_reads()
    np.testing.assert_array_equal(part.view(np.uint32), want_sample[-1][n - 1000:].view(np.uint32))
    with pytest.raises(N.NativeError) as e:
        r.read_async(FILM_SAMPLE, _pinned(10), offset=n - 5)
    assert e.value.code == N.INVALID_ARGUMENT
    with pytest.raises(N.NativeError) as e:
        r.read_async(FILM_SAMPLE, np.zeros((0, 4), np.float32))
    assert e.value.code == N.INVALID_ARGUMENT
