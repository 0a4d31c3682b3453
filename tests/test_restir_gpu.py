"""ReSTIR DI on the GPU (csrc/restir.cu) against the CPU restatement of the
reference's production passes (oracle_pbr.cpp: oracle_restir_frame).

Per frame, the oracle gets the GPU's own inputs (this and the previous
frame's primary surfaces, the previous published reservoirs), so every frame
is compared independently: the integer words of every reservoir
(GpuRestirReservoirV3: selected light identity, M, age, flags, provenance,
history identity) must be identical and its float words within RTOL relative
(+ATOL) on at least MIN_FRACTION of pixels, and the ReSTIR direct term must
agree within the same tolerance on the same fraction.  CUDA's and glibc's
sinf / cosf (sphere-light solid-angle sampling) differ by an ulp now and
then: such a sample's position and direction differ in the last bit, and a
resampling decision near a tie may flip.  The film
of a RestirPrimary frame must match the oracle's (its path planes plus the
ReSTIR direct term) as in the wavefront film tests."""
import numpy as np
import pytest

from helpers import OracleScene
from renderingengine_b200 import _native as N
from renderingengine_b200 import scenes
from renderingengine_b200.scenes import Camera
from renderingengine_b200.traversal import Scene
from renderingengine_b200.wavefront import FILM_SAMPLE, Renderer, frame_constants

pytestmark = pytest.mark.gpu

RTOL, ATOL, MIN_FRACTION = 1e-4, 1e-6, 0.995


def _scene(kind):
    if kind == "many-lights":
        return scenes.add_emissive_triangles(scenes.heightfield_scene(grid=48, spheres=48, seed=2), count=400, seed=5)
    return scenes.cornell_box()


def _orbit(cam: Camera, k: int, step: float) -> Camera:
    """A small sideways camera move per frame (the reprojection has work)."""
    pos = (np.asarray(cam.position, np.float64) + np.asarray(cam.right, np.float64) * (step * k)).astype(np.float32)
    return Camera(pos, cam.forward, cam.right, cam.up, cam.tan_half_fov)


def _close(a, b):
    return np.all(np.abs(a - b) <= ATOL + RTOL * np.abs(b), axis=-1)


# GpuRestirReservoirV3 words: float lanes (sample position / direction /
# radiance / pdfs, weight state, selected terms) and integer lanes (sample
# identity / generation / metadata / source, state, provenance, history).
_FLOAT_WORDS = np.r_[0:16, 32:40]
_INT_WORDS = np.r_[16:32, 40:64]


def _reservoirs_match(got: np.ndarray, want: np.ndarray) -> np.ndarray:
    """Per pixel: integer words identical and float words within tolerance."""
    ints = np.all(got[:, _INT_WORDS] == want[:, _INT_WORDS], axis=1)
    gf = got[:, _FLOAT_WORDS].view(np.float32).astype(np.float64)
    wf = want[:, _FLOAT_WORDS].view(np.float32).astype(np.float64)
    floats = np.all((np.abs(gf - wf) <= ATOL + RTOL * np.abs(wf)) | (gf == wf), axis=1)
    return ints & floats


@pytest.mark.parametrize("kind,sel,cfg", [
    ("many-lights", 1, dict(candidates=32, max_m=20, spatial_neighbors=5)),
    ("many-lights", 0, dict(candidates=8, spatial_neighbors=5, neighbor_mode=1, disk_radius=30.0)),
    ("cornell", 0, dict(candidates=4, spatial_neighbors=0)),
    ("many-lights", 1, dict(candidates=16, temporal=0, spatial_neighbors=8)),
    # Reference correction (RestirReferenceVisibilityPrepareV3 / ResolveV3).
    ("many-lights", 1, dict(candidates=16, max_m=20, spatial_neighbors=5, estimator=1)),
    ("cornell", 0, dict(candidates=4, spatial_neighbors=3, estimator=1)),
    ("many-lights", 0, dict(candidates=8, spatial_neighbors=0, estimator=1)),
])
def test_restir_frames_match_oracle(native, oracle, kind, sel, cfg):
    sd = _scene(kind)
    w, h, depth = 96, 64, 4
    scene = Scene(sd.triangles, sd.fingerprint)
    r = Renderer(w, h, depth)
    r.set_scene(scene, sd, light_selection=sel)
    r.set_restir(**cfg)
    os_ = OracleScene(sd)
    inp = oracle.OracleRenderInputs(sd, os_.nodes, os_.order)
    ors = oracle.OracleRestir(inp, light_selection=sel, **cfg)
    prev_surf = prev_pub = None
    n = w * h
    accepted_any = False
    owned_any = False
    for k in range(5):
        cam = _orbit(sd.camera, k, 0.003)
        fc = frame_constants(cam, w, h, 10 + k, depth, estimator=N.ESTIMATOR_RESTIR_PRIMARY, light_selection=sel)
        r.render(fc, accumulate=False)
        tel = r.collect()
        assert tel.fatal_mask == 0
        surf = r.restir_read(N.RESTIR_SURFACES, n)
        temporal = r.restir_read(N.RESTIR_TEMPORAL, n)
        published = r.restir_read(N.RESTIR_PUBLISHED, n)
        direct = r.restir_read(N.RESTIR_DIRECT, n)
        reasons = r.restir_read(N.RESTIR_REASONS, n)
        stats = r.restir_statistics()
        # The primary surfaces equal the oracle path tracer's.
        planes, _, _ = oracle.render(inp, fc, light_selection=sel)
        same_surf = np.all(surf == planes["surface"].view(np.uint32), axis=1)
        assert same_surf.mean() >= 0.999, f"frame {k}: surfaces equal on {same_surf.mean():.4f}"
        out = ors.frame(fc, surf.view(np.float32), prev_surf, prev_pub)
        for name, got, want in (("temporal", temporal, out["temporal"]), ("published", published, out["published"])):
            same = _reservoirs_match(got, want)
            assert same.mean() >= MIN_FRACTION, f"frame {k} {name}: {same.mean():.4f} of reservoirs match"
        assert (reasons == out["reasons"]).mean() >= MIN_FRACTION
        ok = _close(direct, out["direct"]).all(axis=0)
        assert ok.mean() >= MIN_FRACTION, f"frame {k}: direct within tolerance on {ok.mean():.4f}"
        assert np.isfinite(direct).all() and (direct >= 0).all()
        # Statistics: counts of the same events (flips may move a few).
        st = out["stats"]
        assert stats["candidates_generated"] == st[0]
        assert abs(stats["visibility_evaluated"] - int(st[9])) <= max(3, n // 200)
        owned_any |= bool(np.any(surf[:, 23] & 1))
        if k > 0 and cfg.get("temporal", 1):
            accepted_any |= stats["temporal_accepted"] > 0
        # Film: the oracle's path planes (ReSTIR owns primary direct) plus the ReSTIR term.
        film = r.read(FILM_SAMPLE, n)[:, :3]
        want = planes["sample"][:, :3] + out["direct"][0][:, :3] + out["direct"][1][:, :3]
        fok = np.all(np.abs(film - want) <= ATOL + RTOL * np.abs(want), axis=-1)
        assert fok.mean() >= 0.99, f"frame {k}: film within tolerance on {fok.mean():.4f}"
        if cfg.get("estimator", 0) == 1:
            valid = (published[:, 42] & 1) != 0  # state.z: valid
            assert np.all(published[valid, 42] & 16), "reference-mode flag missing on a valid reservoir"
        prev_surf, prev_pub = surf.view(np.float32), published
    # ReSTIR owns only metallic-roughness primary surfaces
    # (BsdfSupportsRestirPrimaryDirectL6): the Lambertian Cornell box has none.
    assert owned_any == (kind != "cornell")
    if cfg.get("temporal", 1) and owned_any:
        assert accepted_any


def test_restir_camera_cut_and_scene_change_reject_history(native):
    sd = _scene("many-lights")
    w, h = 64, 48
    n = w * h
    scene = Scene(sd.triangles, sd.fingerprint)
    r = Renderer(w, h, 2)
    r.set_scene(scene, sd, light_selection=1)
    r.set_restir(candidates=8, spatial_neighbors=0)
    for k in range(2):
        r.render(frame_constants(sd.camera, w, h, 1 + k, 2, estimator=3, light_selection=1), accumulate=False)
        r.collect()
    assert r.restir_statistics()["temporal_accepted"] > 0
    r.restir_reset()
    r.render(frame_constants(sd.camera, w, h, 3, 2, estimator=3, light_selection=1), accumulate=False)
    r.collect()
    reasons = r.restir_read(N.RESTIR_REASONS, n)
    surf = r.restir_read(N.RESTIR_SURFACES, n)
    owned = (surf[:, 23] & 1) != 0
    assert r.restir_statistics()["temporal_accepted"] == 0
    assert np.all(np.isin(reasons[owned], [1, 4]))  # CameraCut (or an empty history)
    assert (reasons[owned] == 4).mean() > 0.5
    # A frame index gap also rejects (the history is not the previous frame's).
    r.render(frame_constants(sd.camera, w, h, 9, 2, estimator=3, light_selection=1), accumulate=False)
    r.collect()
    assert r.restir_statistics()["temporal_accepted"] == 0
    # Rebinding the scene bumps the scene generation.
    r.render(frame_constants(sd.camera, w, h, 10, 2, estimator=3, light_selection=1), accumulate=False)
    r.collect()
    assert r.restir_statistics()["temporal_accepted"] > 0
    r.set_scene(scene, sd, light_selection=1)
    r.render(frame_constants(sd.camera, w, h, 11, 2, estimator=3, light_selection=1), accumulate=False)
    r.collect()
    reasons = r.restir_read(N.RESTIR_REASONS, n)
    assert r.restir_statistics()["temporal_accepted"] == 0
    assert (reasons[owned] == 10).mean() > 0.5  # SceneGeneration


def test_restir_profile_keeps_history(native):
    """A profiling pass between frames commits nothing: the next frame still
    reuses the previous frame's reservoirs."""
    sd = _scene("many-lights")
    w, h = 64, 48
    scene = Scene(sd.triangles, sd.fingerprint)
    r = Renderer(w, h, 2)
    r.set_scene(scene, sd, light_selection=1)
    r.set_restir(candidates=8)
    r.render(frame_constants(sd.camera, w, h, 1, 2, estimator=3, light_selection=1), accumulate=False)
    r.collect()
    prof = r.profile(frame_constants(sd.camera, w, h, 2, 2, estimator=3, light_selection=1))
    assert prof["restir_ms"] > 0
    r.render(frame_constants(sd.camera, w, h, 2, 2, estimator=3, light_selection=1), accumulate=False)
    r.collect()
    assert r.restir_statistics()["temporal_accepted"] > 0


def test_restir_config_validation(native):
    sd = _scene("cornell")
    r = Renderer(32, 32, 2)
    r.set_scene(Scene(sd.triangles, sd.fingerprint), sd)
    for bad in (dict(spatial_neighbors=31), dict(max_m=0), dict(candidates=2000), dict(neighbor_mode=2),
                dict(disk_radius=0.5)):
        with pytest.raises(N.NativeError) as e:
            r.set_restir(**bad)
        assert e.value.code == N.INVALID_ARGUMENT


def test_restir_debug_views_match_oracle(native, oracle):
    """RestirDebugV3 on the GPU (re_renderer_restir_debug) equals its
    restatement over the same published reservoirs, bit for bit, in every
    debug mode; a frame that is not RestirPrimary yet is reported as not
    ready."""
    sd = _scene("many-lights")
    w, h = 96, 64
    n = w * h
    r = Renderer(w, h, 4)
    r.set_scene(Scene(sd.triangles, sd.fingerprint), sd, light_selection=1)
    with pytest.raises(N.NativeError):
        r.restir_debug(0, n)
    r.set_restir(candidates=8, spatial_neighbors=3, max_m=20, max_history_age=20)
    for f in range(3):
        cam = _orbit(sd.camera, f, 0.002)
        r.render(frame_constants(cam, w, h, f, 4, light_selection=1, estimator=N.ESTIMATOR_RESTIR_PRIMARY,
                                 seed=0x77), accumulate=f > 0)
        r.collect()
    words = r.restir_read(N.RESTIR_PUBLISHED, n)
    assert ((words[:, 42] & 1) != 0).mean() > 0.2  # the surface pixels hold valid reservoirs
    for mode in range(8):
        rec, img = r.restir_debug(mode, n)
        want_rec, want_img = oracle.restir_debug(words, mode, 20, 20)
        np.testing.assert_array_equal(rec, want_rec, err_msg=f"mode {mode}")
        np.testing.assert_array_equal(img.view(np.uint32), want_img.view(np.uint32), err_msg=f"mode {mode}")
