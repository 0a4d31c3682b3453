"""The SVGF restatement (oracle/oracle_svgf.cpp) is pinned bit for bit to the
reference's own SvgfReconstruction (reconstruction/src/Svgf.cpp, compiled from
its sources into oracle/_ref), and reproduces the reference's L8 unit-test
expectations (reconstruction/tests/ReconstructionTests.cpp)."""
import numpy as np
import pytest

import svgf_cases as S
from renderingengine_b200 import _native as N

PLANES = ("raw", "temporal", "atrous", "svgf", "history_length", "moments", "variance", "accepted", "reject")


def _need_ref(oracle):
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")


@pytest.mark.parametrize("w,h,frames,seed,flights,cfg", [
    (24, 16, 6, 1, 2, {}),
    (33, 21, 5, 2, 1, {"atrous_iterations": 5, "phi_normal": 128.0}),
    (17, 29, 5, 3, 3, {"demodulate_specular": 0, "require_material_id": 0, "spatial_radius": 1}),
    (20, 12, 4, 4, 2, {"atrous_iterations": 0, "max_history_length": 3, "minimum_color_alpha": 0.0}),
    (40, 8, 4, 5, 2, {"atrous_iterations": 16, "short_history_length": 1, "require_object_id": 0}),
    (12, 10, 40, 7, 2, {"max_history_length": 8}),
])
def test_oracle_equals_reference_sequence(oracle, w, h, frames, seed, flights, cfg):
    _need_ref(oracle)
    c = S.config(**cfg)
    ours = oracle.OracleSvgf(w, h, flights, c)
    ref = oracle.RefSvgf(w, h, flights, c)
    for gb, sig, fi, trig in S.sequence(w, h, frames, seed, hostile=frames < 20):
        a = ours.process(gb, sig, fi, trig)
        b = ref.process(gb, sig, fi, trig)
        for p in PLANES:
            np.testing.assert_array_equal(S.bits(a[p]), S.bits(b[p]), err_msg=f"frame {fi} plane {p}")


def test_oracle_equals_reference_resize_and_config_change(oracle):
    _need_ref(oracle)
    c = S.config()
    ours = oracle.OracleSvgf(16, 12, 2, c)
    ref = oracle.RefSvgf(16, 12, 2, c)
    seq_a = S.sequence(16, 12, 3, 11)
    seq_b = S.sequence(21, 9, 3, 12)
    steps = [seq_a[0], seq_a[1], seq_b[0], seq_b[1], "config", seq_b[2]]
    for i, step in enumerate(steps):
        if step == "config":
            c2 = S.config(phi_depth=2.0, atrous_iterations=2)
            ours.set_config(c2)
            ref.set_config(c2)
            continue
        gb, sig, _, trig = step
        a = ours.process(gb, sig, i, trig)
        b = ref.process(gb, sig, i, trig)
        for p in PLANES:
            np.testing.assert_array_equal(S.bits(a[p]), S.bits(b[p]), err_msg=f"step {i} plane {p}")
        if i == 2:  # resolution change: everything reset
            assert np.all(a["reject"] & 2)
        if i == 5:  # ReconstructionParameters reset after SetConfig
            assert np.all(a["reject"] & 2)


def test_invalid_configs_rejected(oracle):
    for bad in ({"minimum_albedo": 0.0}, {"max_history_length": 0}, {"spatial_radius": 65},
                {"atrous_iterations": 17}, {"normal_cosine_threshold": 1.5}, {"phi_luminance": 0.0}):
        with pytest.raises(ValueError):
            oracle.OracleSvgf(4, 4, 1, S.config(**bad))


def test_temporal_moments_motion_and_reset(oracle):
    """TestTemporalMomentsMotionAndReset (ReconstructionTests.cpp:234-287)."""
    c = S.config(minimum_color_alpha=0.0, minimum_moments_alpha=0.0, atrous_iterations=0)
    r = oracle.OracleSvgf(2, 1, 2, c)
    g0 = S.valid_gbuffer(1, 2)
    s0 = S.uniform_signal(1, 2, 1.0)
    s0["diffuse"][0, 1] = 2.0
    f0 = r.process(g0, s0, 0)
    assert f0["history_length"][0, 0] == 1 and f0["reject"][0, 0] & 1
    g1 = S.valid_gbuffer(1, 2)
    g1["motion"][0, 1] = (-0.5, 0.0)
    s1 = S.uniform_signal(1, 2, 3.0)
    f1 = r.process(g1, s1, 1)
    assert f1["accepted"][0, 1] == 1 and f1["history_length"][0, 1] == 2
    assert abs(f1["temporal"][0, 1, 0] - 2.0) <= 1e-5
    assert abs(f1["moments"][0, 1, 0] - 2.0) <= 1e-5 and abs(f1["moments"][0, 1, 1] - 5.0) <= 1e-5
    cut = r.process(g1, s1, 2, 1)
    assert cut["history_length"][0, 1] == 1 and cut["reject"][0, 1] & 2
    g1["motion"][0, 0] = (2.0, 0.0)
    off = r.process(g1, s1, 3)
    assert off["reject"][0, 0] == 4  # ScreenBounds only


def test_depth_time_domain_and_invalid_motion(oracle):
    """TestTemporalDepthTimeDomainAndInvalidMotion (ReconstructionTests.cpp:289-329)."""
    c = S.config(minimum_color_alpha=0.0, minimum_moments_alpha=0.0, atrous_iterations=0)
    r = oracle.OracleSvgf(1, 1, 2, c)
    g = S.valid_gbuffer(1, 1)
    g["linear_depth"] = 6.0
    g["expected_previous_linear_depth"] = 6.0
    s = S.uniform_signal(1, 1, 1.0)
    r.process(g, s, 0)
    g1 = S.valid_gbuffer(1, 1)
    g1["linear_depth"], g1["expected_previous_linear_depth"] = 5.0, 6.0
    s["diffuse"] = 3.0
    moved = r.process(g1, s, 1)
    assert moved["accepted"][0, 0] == 1 and moved["reject"][0, 0] == 0
    g2 = S.valid_gbuffer(1, 1)
    g2["linear_depth"], g2["expected_previous_linear_depth"] = 4.0, 5.0
    g2["flags"] = N.GBUFFER_VALID
    inv = r.process(g2, s, 2)
    assert inv["accepted"][0, 0] == 0 and inv["reject"][0, 0] == 1 << 10
    g3 = S.valid_gbuffer(1, 1)
    g3["linear_depth"], g3["expected_previous_linear_depth"] = 3.0, 4.0
    rec = r.process(g3, s, 3)
    assert rec["accepted"][0, 0] == 1 and rec["history_length"][0, 0] == 2


def test_disocclusion_and_edge_stopping(oracle):
    """TestDisocclusionAndEdgeStopping (ReconstructionTests.cpp:353-384)."""
    c = S.config(atrous_iterations=1, phi_luminance=100000.0)
    r = oracle.OracleSvgf(10, 1, 2, c)
    g = S.valid_gbuffer(1, 10)
    s = np.zeros((1, 10), N.SIGNAL_DTYPE)
    for x in range(10):
        right = x >= 5
        g["object_id"][0, x] = 2 if right else 1
        s["diffuse"][0, x] = 4.0 if right else 0.25
    g["object_id"][0, 3] = 3
    f0 = r.process(g, s, 0)
    assert abs(f0["atrous"][0, 4, 0] - 0.25) <= 1e-4 and abs(f0["atrous"][0, 5, 0] - 4.0) <= 1e-4
    fb = g.copy()
    fb["motion"][0, 5] = (-0.08, 0.0)
    fb["object_id"][0, 5] = 3
    f1 = r.process(fb, s, 1)
    assert f1["accepted"][0, 5] == 1
    dis = fb.copy()
    dis["object_id"][0, 5] = 99
    f2 = r.process(dis, s, 2)
    assert f2["accepted"][0, 5] == 0 and f2["reject"][0, 5] & (1 << 9)


def test_checkerboard_denoising_metric(oracle):
    """TestVarianceBootstrapAndDenoisingMetric (ReconstructionTests.cpp:386-407):
    raw RMSE 0.5 and the A-Trous RMSE the reference prints (0.00183614)."""
    _need_ref(oracle)
    c = S.config(atrous_iterations=2, phi_luminance=100000.0)
    g, s = S.checkerboard()
    f = oracle.OracleSvgf(16, 16, 2, c).process(g, s, 0)
    raw = f["raw"][..., :3] + f["raw"][..., 3:]
    atr = f["atrous"][..., :3] + f["atrous"][..., 3:]
    one = np.ones_like(raw)
    raw_rmse, atr_rmse = oracle.image_rmse(raw, one), oracle.image_rmse(atr, one)
    assert raw_rmse > 0.49 and atr_rmse < raw_rmse
    assert abs(atr_rmse - 0.00183614) < 5e-8
    assert raw_rmse == oracle.ref_image_rmse(raw, one) and atr_rmse == oracle.ref_image_rmse(atr, one)
    assert f["variance"][8, 8] > 1e-6


def test_motion_vectors_equal_reference(oracle):
    """ComputeMotionVector (MotionVectors.cpp:37-67) on seeded cameras plus the
    reference test's edge cases (ReconstructionTests.cpp:80-132)."""
    _need_ref(oracle)
    rng = np.random.default_rng(3)
    eye = np.eye(4, dtype=np.float32).ravel()
    cases = [(np.zeros(3), eye, eye, eye, (0.01, -0.02), (-0.02, 0.03))]
    bad = eye.copy()
    bad[15] = 0.0
    cases.append((np.zeros(3), bad, eye, eye, (0, 0), (0, 0)))
    neg = eye.copy()
    neg[15] = -1.0
    cases.append((np.zeros(3), neg, eye, eye, (0, 0), (0, 0)))
    tiny = eye.copy()
    tiny[15] = 2e-8
    cases.append((np.array([3.4e38, 0, 0]), tiny, tiny, eye, (0, 0), (0, 0)))
    for _ in range(200):
        m = [rng.normal(size=16).astype(np.float32) for _ in range(3)]
        cases.append((rng.normal(size=3), m[0], m[1], m[2], rng.normal(scale=0.01, size=2),
                      rng.normal(scale=0.01, size=2)))
    for case in cases:
        a = oracle.motion_vector(*case)
        b = oracle.ref_motion_vector(*case)
        np.testing.assert_array_equal(S.bits(a), S.bits(b))
