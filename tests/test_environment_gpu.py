"""Environment light on the device (row (f)2): the importance tables the
renderer builds equal the reference's BuildEnvironmentDistribution entry for
entry; frames with an environment (MIS, NEE and BSDF-only estimators) match
the oracle pixel for pixel; and the white furnace -- a plane under a constant
environment -- converges to the FP64 directional albedo of the reference's
own BSDF (ReferenceBsdf.hpp EvaluateBsdfL6, by quadrature) for Lambert, GGX
conductor, metallic-roughness and GGX dielectric reflection."""
import numpy as np
import pytest

import analytic_scenes as A
from helpers import OracleScene
from renderingengine_b200 import _native as N
from renderingengine_b200 import scenes
from renderingengine_b200.traversal import Scene
from renderingengine_b200.wavefront import FILM_MEAN, FILM_SAMPLE, Renderer, frame_constants
from test_environment import _z_gates

pytestmark = pytest.mark.gpu
RTOL, ATOL, MIN_FRACTION = 1e-4, 1e-6, 0.999


def _env_scene():
    sd = scenes.heightfield_scene(grid=64, spheres=96, seed=6)
    sd.lights = np.concatenate([sd.lights, scenes.environment_light(scale=0.8, light_id=1)])
    sd.extra = dict(sd.extra or {}, environment=scenes.sky_environment(48, 24, seed=3))
    return sd


def test_device_environment_tables_equal_reference(native, oracle):
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    sd = _env_scene()
    scene = Scene(sd.triangles, sd.fingerprint, 1, N.BUILD_LBVH)
    r = Renderer(64, 64, 4)
    r.set_scene(scene, sd, light_selection=1)
    rows, cols, integ = r.environment_tables(0)
    r_rows, r_cols, r_int, _ = oracle.ref_environment_tables(sd.extra["environment"])
    np.testing.assert_array_equal(rows.view(np.uint32), r_rows.view(np.uint32))
    np.testing.assert_array_equal(cols.view(np.uint32), r_cols.view(np.uint32))
    assert integ == r_int
    r.close()
    scene.close()


@pytest.mark.parametrize("estimator", [2, 1, 0], ids=["mis", "nee", "bsdf-only"])
@pytest.mark.parametrize("selection", [0, 1], ids=["uniform", "power"])
def test_film_with_environment_matches_oracle(native, oracle, estimator, selection):
    sd = _env_scene()
    w, h, depth = 128, 72, 6
    scene = Scene(sd.triangles, sd.fingerprint)
    r = Renderer(w, h, depth)
    r.set_scene(scene, sd, light_selection=selection)
    fc = frame_constants(sd.camera, w, h, 5, depth, light_selection=selection, estimator=estimator, seed=0xE17)
    r.render(fc, accumulate=False)
    tel = r.collect()
    os_ = OracleScene(sd)
    inp = oracle.OracleRenderInputs(sd, os_.nodes, os_.order)
    ref, rays, shadows = oracle.render(inp, fc, light_selection=selection)
    got = r.read(FILM_SAMPLE, w * h)[:, :3]
    ok = (np.abs(got - ref["sample"][:, :3]) <= ATOL + RTOL * np.abs(ref["sample"][:, :3])).all(axis=1)
    assert ok.mean() >= MIN_FRACTION, ok.mean()
    # Every pixel outside the tolerance evaluated a libm transcendental on its path.
    assert (ref["libm_calls"][~ok] > 0).all()
    assert abs(tel.path_rays - rays) <= max(2, rays // 2000)
    assert abs(tel.shadow_rays - shadows) <= max(2, shadows // 2000)
    assert tel.fatal_mask == 0 and tel.non_finite == 0
    # The sky is seen by the camera rays that miss: some pixels are pure environment.
    assert (ref["camera_emission"][:, :3].max(axis=1) > 0).any()
    r.close()
    scene.close()


def test_restir_over_an_environment_is_rejected(native):
    sd = _env_scene()
    scene = Scene(sd.triangles, sd.fingerprint)
    r = Renderer(64, 32, 4)
    r.set_scene(scene, sd)
    fc = frame_constants(sd.camera, 64, 32, 0, 4, estimator=3)
    with pytest.raises(RuntimeError, match="ReSTIR DI over a scene with an environment"):
        r.render(fc, accumulate=False)
    r.close()
    scene.close()


@pytest.mark.parametrize("name", list(A.FURNACE_MATERIALS))
def test_furnace_converges_to_reference_albedo(native, oracle, name):
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    sd = A.furnace_plane(A.FURNACE_MATERIALS[name]())
    w, h, depth, spp = 16, 12, 4, 2048
    scene = Scene(sd.triangles, sd.fingerprint, 1, N.BUILD_LBVH)
    r = Renderer(w, h, depth)
    r.set_scene(scene, sd)
    acc = np.zeros((w * h, 3))
    acc2 = np.zeros((w * h, 3))
    for s in range(spp):
        r.render(frame_constants(sd.camera, w, h, s, depth, rr=(1000.0, 0.05, 0.95, 1e-4)), accumulate=s > 0)
        x = r.read(FILM_SAMPLE, w * h)[:, :3].astype(np.float64)
        acc += x
        acc2 += x * x
    mean = acc / spp
    film = r.read(FILM_MEAN, w * h)[:, :3].astype(np.float64)
    np.testing.assert_allclose(film, mean, rtol=2e-5, atol=1e-7)  # the device's own progressive mean
    dirs = A.pixel_directions(sd.camera, w, h, sub=3)
    alb = sum(A.directional_albedo(oracle, sd.materials, -dirs[:, k]) for k in range(dirs.shape[1])) / dirs.shape[1]
    z = _z_gates(mean, acc2 / spp - mean * mean, spp, alb)
    print(f"furnace {name}: RMSE vs FP64 albedo {np.sqrt(((mean - alb) ** 2).mean()):.3e}, max |z| "
          f"{np.abs(z).max():.2f}")
    r.close()
    scene.close()
