"""Environment light (row (f)2): the importance tables against the
reference's own BuildEnvironmentDistribution (integrators/megakernel/
MegakernelBridge.cpp:191-273, compiled in oracle/_ref) entry for entry, the
top-level distribution with the environment's power weight against
BuildTopLevelLightDistribution (:403-455), and the oracle's environment
sampling consistent with its PDF."""
import numpy as np
import pytest

from renderingengine_b200 import scenes


def _maps():
    rng = np.random.default_rng(4)
    sky = scenes.sky_environment(64, 32, seed=1)
    black = np.zeros((8, 16, 4), np.float32)
    rows = rng.random((16, 24, 4)).astype(np.float32)
    rows[3] = 0.0          # a black row
    rows[:, 5] = 0.0       # a black column
    tall = rng.random((40, 7, 4)).astype(np.float32) ** 4
    return {"sky": sky, "black": black, "zero-rows-cols": rows, "tall": tall}


@pytest.mark.parametrize("name", list(_maps()))
def test_environment_tables_equal_reference(oracle, name):
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    env = _maps()[name]
    r_rows, r_cols, r_int, r_fb = oracle.ref_environment_tables(env)
    o_rows, o_cols, o_int = oracle.environment_tables(env)
    np.testing.assert_array_equal(o_rows.view(np.uint32), r_rows.view(np.uint32))
    np.testing.assert_array_equal(o_cols.view(np.uint32), r_cols.view(np.uint32))
    assert o_int == r_int
    assert r_fb == (name == "black")


def test_top_level_distribution_with_environment_equals_reference(oracle):
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    import ctypes as C
    env = scenes.sky_environment(64, 32, seed=2)
    _, _, integ = oracle.environment_tables(env)
    lights = np.concatenate([scenes.environment_light(scale=0.7), scenes.sphere_light((0, 2, 0), 0.3, (5, 4, 3)),
                             scenes.sphere_light((1, 2, 0), 0.1, (50, 40, 30))])
    n = len(lights)
    for sel in (0, 1):
        alias = np.zeros((n, 4), np.uint32)
        pmf = np.zeros(n, np.float32)
        cnt = oracle.ref_lib().ref_light_distribution_env(lights.ctypes.data, n, sel, 2.5, integ, alias.ctypes.data,
                                                          pmf.ctypes.data)
        assert cnt == n
        # The renderer's weights: pi R^2 scale x integrated luminance for the map.
        w = 3.141592653589793 * 2.5 * 2.5 * 0.7 * integ
        assert sel == 0 or pmf[0] > 0
        if sel == 1:
            lum = lambda l: (0.2126 * l[0] + 0.7152 * l[1] + 0.0722 * l[2]) * l[3]
            p = [w] + [4 * np.pi ** 2 * float(l["shape_params"][0]) ** 2 * lum(l["radiance_scale"].astype(float))
                       for l in lights[1:]]
            np.testing.assert_allclose(pmf, np.asarray(p) / sum(p), rtol=1e-6)


def _z_gates(mean, var, spp, expected):
    """Per pixel and channel z = (mean - E) / sqrt(var / spp), the variance
    estimated from the same samples.  The channels of a pixel share its
    paths, so the pixels are the independent units: max |z| <= 5.5,
    |mean z| <= 5.5 / sqrt(pixels), mean z^2 within 1 +- 5 sqrt(2 / pixels)."""
    z = (mean - expected) / np.sqrt(np.maximum(var, 1e-30) / spp)
    n = len(z)
    assert np.abs(z).max() <= 5.5, np.abs(z).max()
    assert abs(z.mean()) <= 5.5 / np.sqrt(n), z.mean()
    assert abs((z * z).mean() - 1.0) <= 5.0 * np.sqrt(2.0 / n), (z * z).mean()
    return z


@pytest.mark.parametrize("name", ["lambert", "ggx-conductor"])
def test_oracle_furnace_converges_to_reference_albedo(oracle, name):
    """White furnace on the oracle: a plane under a constant environment
    converges to the FP64 directional albedo of the reference's BSDF
    (tests/analytic_scenes.py), 512 spp."""
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    import analytic_scenes as A
    from helpers import host_sah_oracle_inputs
    from renderingengine_b200.wavefront import frame_constants
    sd = A.furnace_plane(A.FURNACE_MATERIALS[name]())
    w, h, depth, spp = 8, 6, 4, 512
    inp = host_sah_oracle_inputs(oracle, sd)
    acc = np.zeros((w * h, 3))
    acc2 = np.zeros((w * h, 3))
    for s in range(spp):
        planes, _, _ = oracle.render(inp, frame_constants(sd.camera, w, h, s, depth, rr=(1000.0, 0.05, 0.95, 1e-4)))
        x = planes["sample"][:, :3].astype(np.float64)
        acc += x
        acc2 += x * x
    mean = acc / spp
    dirs = A.pixel_directions(sd.camera, w, h, sub=3)
    alb = sum(A.directional_albedo(oracle, sd.materials, -dirs[:, k]) for k in range(dirs.shape[1])) / dirs.shape[1]
    _z_gates(mean, acc2 / spp - mean * mean, spp, alb)
