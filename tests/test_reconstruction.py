"""Camera matrices of the renderer -> reconstruction hand-off (host only):
through the reference's own ComputeMotionVector (reconstruction/src/
MotionVectors.cpp:37-74, compiled under oracle/_ref) a point on the camera ray
RayGen shoots through a pixel lands on that pixel's UV, at the view depth the
renderer exports, with zero motion for a still camera."""
import numpy as np

from renderingengine_b200 import scenes
from renderingengine_b200.wavefront import camera_matrices, frame_constants


def test_camera_matrices_reproject_raygen_pixels(native, oracle):
    if not oracle.ref_available():
        import pytest
        pytest.skip("reference library (oracle/_ref) not built")
    rng = np.random.default_rng(4)
    for eye, target, fov, w, h in [((0.5, 0.55, -0.35), (0.5, 0.05, 0.55), 45.0, 1920, 1080),
                                   ((0.0, 1.0, -2.0), (0.1, 0.2, 0.3), 70.0, 64, 48),
                                   ((3.0, -1.0, 2.0), (0.0, 0.0, 0.0), 20.0, 300, 700)]:
        cam = scenes.Camera.look_at(eye, target, fov)
        fc = frame_constants(cam, w, h, 0, 4)
        vp, w2v = camera_matrices(fc)
        for _ in range(40):
            x, y = rng.uniform(0, w), rng.uniform(0, h)
            sx = (x / w) * 2 - 1
            sy = -((y / h) * 2 - 1)
            d = cam.forward + cam.right * (sx * (w / h) * cam.tan_half_fov) + cam.up * (sy * cam.tan_half_fov)
            d = d / np.linalg.norm(d)
            t = rng.uniform(0.1, 5.0)
            p = (cam.position + d * t).astype(np.float32)
            out = oracle.ref_motion_vector(p, vp, vp, w2v)
            assert out[7] == 1.0
            np.testing.assert_allclose(out[0:2], (x / w, y / h), atol=2e-5)
            np.testing.assert_allclose(out[4:6], 0.0, atol=1e-7)
            depth = float(np.dot(p.astype(np.float64) - cam.position, cam.forward))
            np.testing.assert_allclose(out[6], depth, rtol=1e-5, atol=1e-6)
        # A point behind the camera does not reproject.
        behind = (cam.position - cam.forward * 0.5).astype(np.float32)
        assert oracle.ref_motion_vector(behind, vp, vp, w2v)[7] == 0.0
