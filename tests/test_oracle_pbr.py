"""CPU tests: the FP32 integrator oracle's building blocks pinned against the
reference's own CPU code (Philox, alias tables, light PMFs) and sanity of the
oracle integrator itself (energy, determinism).  No GPU needed."""
import numpy as np
import pytest

from helpers import OracleScene
from renderingengine_b200 import scenes
from renderingengine_b200.wavefront import frame_constants


def test_philox_matches_reference_counter_random(oracle):
    """Philox4x32-10 counter RNG equals MegakernelBridge::CounterRandomFloat
    (MegakernelBridge.cpp:552-589) on a sweep of counters and keys, and the
    reference's own dimension-map asserts hold (ForBounce(0, RR) == 13)."""
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    rng = np.random.default_rng(1)
    for _ in range(2000):
        px, s, d, st = (int(x) for x in rng.integers(0, 2**32, 4, dtype=np.uint64))
        seed = int(rng.integers(0, 2**63))
        a = oracle.counter_random(px, s, d, st, seed & 0xFFFFFFFF, seed >> 32)
        b = oracle.ref_lib().ref_counter_random(px, s, d, st, seed)
        assert np.float32(a) == np.float32(b)
        assert 0.0 <= a < 1.0
    assert 4 + 0 * 16 + 9 == 13 and 4 + 1 * 16 + 0 == 20


@pytest.mark.parametrize("selection", [0, 1])
def test_light_distribution_matches_reference(oracle, selection):
    """The oracle's Vose alias table and top-level light PMF equal
    BuildTopLevelLightDistribution (MegakernelBridge.cpp:403-455) entry for
    entry, for uniform and power-weighted selection over mixed lights."""
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    sd = scenes.add_emissive_triangles(scenes.heightfield_scene(grid=32, spheres=8, seed=4), count=300, seed=2)
    lights = sd.lights.copy()
    lights["identity"][5, 1] = 0  # a disabled light
    mine = oracle.light_distribution(lights, selection, 2.0)
    ref_alias, ref_pmf = oracle.ref_light_distribution(lights, selection, 2.0)
    np.testing.assert_array_equal(mine.view(np.uint32), ref_alias)
    pmf = np.zeros(len(lights), np.float32)
    pmf[mine[:, 3].view(np.uint32)] = mine[:, 1]
    np.testing.assert_array_equal(pmf, ref_pmf)


def _oracle_image(sd, w, h, depth, sample=0, estimator=2, selection=0):
    os_ = OracleScene(sd)
    from oracle import oracle as O
    inp = O.OracleRenderInputs(sd, os_.nodes, os_.order)
    fc = frame_constants(sd.camera, w, h, sample, depth, estimator=estimator, light_selection=selection)
    return O.render(inp, fc, light_selection=selection)


def test_oracle_render_deterministic_and_finite(oracle):
    sd = scenes.cornell_box()
    a, ra, sa = _oracle_image(sd, 64, 36, 4)
    b, rb, sb = _oracle_image(sd, 64, 36, 4)
    np.testing.assert_array_equal(a["sample"], b["sample"])
    assert ra == rb and sa == sb
    assert np.isfinite(a["sample"]).all() and (a["sample"][:, :3] >= 0).all()
    # The five signals add up to the sample value.
    parts = sum(a[k][:, :3] for k in ("camera_emission", "direct_diffuse", "direct_specular",
                                      "indirect_diffuse", "indirect_specular"))
    np.testing.assert_allclose(parts, a["sample"][:, :3], rtol=1e-6, atol=1e-7)
    assert ra >= 64 * 36 and sa > 0


def test_oracle_cornell_converges_to_reference_fp64(oracle):
    """The FP32 oracle integrator (triangle-light NEE + MIS, Philox) converges
    to the reference FP64 Cornell integrator (rectangle-light NEE, PCG) on the
    reference fixture: 32x32 pixels, 256 spp each, 8 bounces; mean radiance
    within 2% and per-pixel RMSE below 0.05."""
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    sd = scenes.cornell_reference()
    w = h = 32
    acc = np.zeros((w * h, 3))
    spp = 256
    os_ = OracleScene(sd)
    inp = oracle.OracleRenderInputs(sd, os_.nodes, os_.order)
    for s in range(spp):
        fc = frame_constants(sd.camera, w, h, s, 8)
        planes, _, _ = oracle.render(inp, fc)
        acc += planes["sample"][:, :3]
    mine = (acc / spp).reshape(h, w, 3)
    ref, _ = oracle.ref_cornell(w, h, spp, 8, 1, 0)
    assert abs(mine.mean() - ref.mean()) / ref.mean() < 0.02
    assert np.sqrt(((mine - ref) ** 2).mean()) < 0.05
