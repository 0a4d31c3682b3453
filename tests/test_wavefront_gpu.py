"""GPU parity of the wavefront PBR integrator (RayGen, Intersect, Shade with
NEE+MIS, TraceShadow, Resolve, progressive film) against the FP32 CPU oracle
with the same counter-based RNG, plus the FP64 convergence check against the
reference's own Cornell integrator."""
import numpy as np
import pytest

from helpers import OracleScene
from renderingengine_b200 import scenes
from renderingengine_b200.traversal import Scene
from renderingengine_b200.wavefront import (FILM_CAMERA_EMISSION, FILM_DIRECT_DIFFUSE, FILM_DIRECT_SPECULAR,
                                            FILM_INDIRECT_DIFFUSE, FILM_INDIRECT_SPECULAR, FILM_MEAN,
                                            FILM_PRIMARY_NORMAL, FILM_PRIMARY_POSITION, FILM_SAMPLE, Renderer,
                                            frame_constants)

pytestmark = pytest.mark.gpu

# Per-pixel film tolerance: FP32 with the same operation order up to libm
# ulp differences (sin/cos/pow/acos/atan2); 1e-4 relative (plus 1e-6
# absolute for near-black pixels).  A pixel outside it must be one whose
# oracle path evaluated such a transcendental (the oracle counts them per
# pixel): there CUDA's and glibc's last bits may differ and a discrete
# decision (RR, lobe, hit/miss) can flip.  The measured fraction of such
# pixels is printed; at least 99.9% must match.
RTOL, ATOL, MIN_FRACTION = 1e-4, 1e-6, 0.999


def _explained_fraction(got, want, libm_calls, name, near_tie=None):
    """Fraction of pixels within tolerance; every pixel outside it must have
    evaluated a libm transcendental on its oracle path, or be a primary-hit
    near-tie (`near_tie`: pixels whose primary triangle differs between two
    candidates at the same depth)."""
    ok = (np.abs(got - want) <= ATOL + RTOL * np.abs(want)).all(axis=-1)
    bad = np.flatnonzero(~ok)
    explained = libm_calls[bad] > 0
    if near_tie is not None:
        explained |= np.isin(bad, near_tie)
    assert explained.all(), f"{name}: {int((~explained).sum())} mismatching pixels neither used libm nor tie"
    print(f"{name}: {len(bad)} of {len(ok)} pixels outside tolerance, all on libm paths or primary near-ties")
    return ok.mean()


def _setup(sd, w, h, depth, selection=0):
    scene = Scene(sd.triangles, sd.fingerprint)
    r = Renderer(w, h, depth)
    r.set_scene(scene, sd, light_selection=selection)
    return scene, r


def _oracle(oracle, sd, fc, selection=0):
    os_ = OracleScene(sd)
    inp = oracle.OracleRenderInputs(sd, os_.nodes, os_.order)
    return oracle.render(inp, fc, light_selection=selection)


def _close_fraction(a, b):
    ok = np.abs(a - b) <= ATOL + RTOL * np.abs(b)
    return ok.all(axis=-1).mean()


def _tiny():
    """Three triangles: one leaf, so the hierarchy is a single leaf under a
    synthetic root (an empty sibling box that no ray may enter)."""
    pos = np.array([[[-1, 0, -1], [1, 0, -1], [1, 0, 1]], [[-1, 0, -1], [1, 0, 1], [-1, 0, 1]],
                    [[-0.2, 0.3, 0], [0.2, 0.3, 0], [0, 0.6, 0.1]]], np.float32)
    tri = scenes.canonical_triangles(pos, None, np.zeros(3, np.uint32), np.arange(3, dtype=np.uint32),
                                     np.array([0, 0, 1], np.uint32))
    mats = np.concatenate([scenes.material(scenes.LAMBERT, base=(0.7, 0.7, 0.7)),
                           scenes.material(scenes.METALLIC_ROUGHNESS, base=(0.9, 0.5, 0.2), roughness=0.3)])
    lights = scenes.sphere_light((0.0, 1.5, 0.0), 0.2, (10.0, 10.0, 10.0))
    cam = scenes.Camera.look_at((0.0, 1.0, -2.0), (0.0, 0.2, 0.0), 50.0)
    return scenes.SceneData("tiny", tri, mats, lights, np.zeros(0, scenes.FIXTURE_TRIANGLE_DTYPE), cam,
                            fingerprint=0x7171)


CASES = [
    ("tiny", _tiny, 64, 48, 4, 0),
    ("cornell", scenes.cornell_box, 160, 90, 4, 0),
    ("cornell-reference", scenes.cornell_reference, 96, 96, 8, 0),
    ("heightfield", lambda: scenes.heightfield_scene(grid=96, spheres=256, seed=3), 192, 108, 8, 0),
    ("many-lights", lambda: scenes.add_emissive_triangles(scenes.heightfield_scene(grid=64, spheres=64, seed=2),
                                                           count=1000, seed=5), 128, 72, 6, 1),
]


@pytest.mark.parametrize("name,make,w,h,depth,sel", CASES)
@pytest.mark.parametrize("tuning", [dict(fuse=False), dict(fuse=True), dict(traversal=2), dict(traversal=5),
                                    dict(traversal=6), dict(traversal=7), dict(traversal=8)],
                         ids=["split", "fused", "wide", "eight", "eight-compressed", "fma-slab", "fma-slab-ww"])
def test_film_matches_oracle(native, oracle, name, make, w, h, depth, sel, tuning):
    sd = make()
    scene, r = _setup(sd, w, h, depth, sel)
    r.set_tuning(**tuning)
    fc = frame_constants(sd.camera, w, h, 3, depth, light_selection=sel, seed=0x1234_5678_9ABC)
    r.render(fc, accumulate=False)
    tel = r.collect()
    ref, rays, shadows = _oracle(oracle, sd, fc, sel)
    n = w * h
    planes = {"sample": FILM_SAMPLE, "camera_emission": FILM_CAMERA_EMISSION,
              "direct_diffuse": FILM_DIRECT_DIFFUSE, "direct_specular": FILM_DIRECT_SPECULAR,
              "indirect_diffuse": FILM_INDIRECT_DIFFUSE, "indirect_specular": FILM_INDIRECT_SPECULAR}
    # Primary-surface export.
    pos = r.read(FILM_PRIMARY_POSITION, n)
    assert _close_fraction(pos, ref["primary_position"]) >= MIN_FRACTION
    nrm = r.read(FILM_PRIMARY_NORMAL, n)
    # Primary material: equal, except near-ties -- two triangles at the same
    # distance (the many-light scene's coplanar emitters overlap), where the
    # lower (instance, primitive) wins unless a 1-ulp slab rounding prunes
    # one of them, which depends on the visiting order (the while-while and
    # four-wide loops visit in another order than the reference loop).
    mat_g, mat_r = nrm[:, 3].view(np.uint32), ref["primary_normal"][:, 3].view(np.uint32)
    diff = np.flatnonzero(mat_g != mat_r)
    assert len(diff) <= n // 1000, f"{len(diff)} primary materials differ"
    dg, dr = pos[diff, 3].astype(np.float64), ref["primary_position"][diff, 3].astype(np.float64)
    assert np.all(np.abs(dg - dr) <= 1e-6 * np.abs(dr) + 1e-7), "a differing primary hit is not a near-tie"
    for key, plane in planes.items():
        got = r.read(plane, n)[:, :3]
        frac = _explained_fraction(got, ref[key][:, :3], ref["libm_calls"], f"{name} {key}", near_tie=diff)
        assert frac >= MIN_FRACTION, f"{key}: only {frac:.5f} of pixels within tolerance"
    # Ray counts: identical paths trace identical rays (allow flips).
    assert abs(tel.path_rays - rays) <= max(2, rays // 2000)
    assert abs(tel.shadow_rays - shadows) <= max(2, shadows // 2000)
    assert tel.fatal_mask == 0 and tel.non_finite == 0
    assert np.isfinite(r.read(FILM_SAMPLE, n)).all()


def test_split_points_and_graph_are_bit_identical(native):
    """Fused vs split Intersect/Shade, graph replay vs direct launches, lane
    refill, while-while traversal: the same film bit for bit (per-path RNG is
    counter based, the closest hit and visibility do not depend on the
    visiting order)."""
    sd = scenes.heightfield_scene(grid=64, spheres=128, seed=9)
    w, h, depth = 128, 96, 8
    scene, r = _setup(sd, w, h, depth)
    fc = frame_constants(sd.camera, w, h, 1, depth)
    outs = []
    configs = [dict(fuse=False, graph=True), dict(fuse=True, graph=True), dict(fuse=False, graph=False),
               dict(fuse=True, graph=False), dict(refill=8), dict(refill=32, graph=False),
               dict(shade_variant=1), dict(shade_variant=2, fuse=True), dict(blocks_per_sm=2, refill=16),
               dict(traversal=1), dict(traversal=1, graph=False, shade_variant=1), dict(traversal=2),
               dict(traversal=2, graph=False, blocks_per_sm=2), dict(shade_variant=3),
               dict(shade_variant=4, graph=False), dict(shade_variant=3, fuse=True), dict(shade_variant=4, fuse=True),
               dict(shade_variant=5), dict(shade_variant=5, fuse=True, graph=False), dict(shade_variant=6),
               dict(shade_variant=7, graph=False), dict(traversal=3),
               dict(traversal=4), dict(traversal=4, refill=8), dict(traversal=2, refill=16, graph=False),
               dict(traversal=3, refill=32), dict(block=256), dict(block=512, traversal=4),
               dict(block=256, traversal=1, graph=False), dict(block=512, traversal=2, blocks_per_sm=4),
               dict(traversal=5), dict(traversal=6), dict(traversal=6, graph=False, block=256),
               dict(traversal=5, block=512), dict(traversal=7), dict(traversal=8),
               dict(traversal=7, block=512, graph=False), dict(traversal=8, block=256)]
    for cfg in configs:
        r.set_tuning(**cfg)
        r.render(fc, accumulate=False)
        r.collect()
        outs.append(r.read(FILM_SAMPLE, w * h))
    for o in outs[1:]:
        np.testing.assert_array_equal(o.view(np.uint32), outs[0].view(np.uint32))


@pytest.mark.parametrize("make", [lambda: scenes.triangle_soup(60000, seed=8),
                                  lambda: scenes.heightfield_scene(grid=128, spheres=256, seed=4)],
                         ids=["soup", "heightfield"])
def test_traversal_modes_agree_on_lbvh(native, make):
    """The traversal loops (reference loop, while-while, four-wide, eight-wide
    plain and compressed) on GPU-built LBVH hierarchies, whose depth exceeds
    the SAH trees': the same film bit for bit; the profile reports the node
    bytes each loop fetched (64 B child pairs, 128 B four-wide, 224 B
    eight-wide, 96 B compressed eight-wide nodes)."""
    from renderingengine_b200 import _native as N
    sd = make()
    w, h, depth = 160, 120, 6
    scene = Scene(sd.triangles, sd.fingerprint, 1, N.BUILD_LBVH)
    r = Renderer(w, h, depth)
    r.set_scene(scene, sd)
    fc = frame_constants(sd.camera, w, h, 2, depth)
    outs, profs = [], []
    for mode in (0, 1, 2, 3, 4, 5, 6, 7, 8):
        r.set_tuning(traversal=mode)
        r.render(fc, accumulate=False)
        tel = r.collect()
        assert tel.fatal_mask == 0 and tel.non_finite == 0
        outs.append(r.read(FILM_SAMPLE, w * h))
        profs.append(r.profile(fc))
    for o in outs[1:]:
        np.testing.assert_array_equal(o.view(np.uint32), outs[0].view(np.uint32))
    # Lane refill over the four-wide nodes and over the child pairs.
    for cfg in (dict(traversal=4, refill=8), dict(traversal=1, refill=16)):
        r.set_tuning(**cfg)
        r.render(fc, accumulate=False)
        assert r.collect().fatal_mask == 0
        np.testing.assert_array_equal(r.read(FILM_SAMPLE, w * h).view(np.uint32), outs[0].view(np.uint32),
                                      err_msg=str(cfg))
    for p in profs:
        assert sum(p["intersect_node_bytes"]) > 0 and sum(p["intersect_triangle_tests"]) > 0
    # Mode 1 counts with the reference loop; mode 2 counts wide fetches.
    assert profs[0]["intersect_node_bytes"] == profs[1]["intersect_node_bytes"]
    wide_fetches = sum(profs[2]["intersect_node_bytes"]) / 128
    pair_fetches = sum(profs[0]["intersect_node_bytes"]) / 64
    assert wide_fetches < pair_fetches
    assert profs[3]["intersect_node_bytes"] == profs[2]["intersect_node_bytes"]  # LBVH: mode 3 is four-wide
    # Eight-wide: 224 B plain (the entries included), 96 B compressed; fewer
    # fetches than four-wide.  Compressed boxes only ever add visits.
    eight_fetches = sum(profs[5]["intersect_node_bytes"]) / 224
    q_fetches = sum(profs[6]["intersect_node_bytes"]) / 96
    assert eight_fetches == int(eight_fetches) and q_fetches == int(q_fetches)
    assert eight_fetches < wide_fetches and q_fetches >= eight_fetches
    assert sum(profs[6]["intersect_triangle_tests"]) >= sum(profs[5]["intersect_triangle_tests"])
    # Conservative one-fma slab test over the four-wide nodes: every box the
    # exact test enters, and a few more (a zero direction component, boxes
    # within a few ulps), so at least the exact loop's fetches.
    for m in (7, 8):
        assert sum(profs[m]["intersect_node_bytes"]) % 128 == 0
        assert sum(profs[m]["intersect_node_bytes"]) >= sum(profs[4]["intersect_node_bytes"])
        assert sum(profs[m]["intersect_node_bytes"]) <= 1.01 * sum(profs[4]["intersect_node_bytes"])
        assert sum(profs[m]["intersect_triangle_tests"]) >= sum(profs[4]["intersect_triangle_tests"])


def test_progressive_film_mean(native):
    """Film progressive mean over frames equals the mean of the per-frame
    samples (the reference's frame-signal check, threshold 2e-5 max scaled
    error: RE/docs/handoffs/L0/p0-2-through-p0-4.md:101-113)."""
    sd = scenes.cornell_box()
    w, h, depth = 640, 360, 4
    scene, r = _setup(sd, w, h, depth)
    samples = []
    for f in range(3):
        r.render(frame_constants(sd.camera, w, h, f, depth, seed=47), accumulate=f > 0)
        r.collect()
        samples.append(r.read(FILM_SAMPLE, w * h)[:, :3].astype(np.float64))
    mean = r.read(FILM_MEAN, w * h)
    assert np.all(mean[:, 3] == 3.0)
    expect = np.mean(samples, axis=0)
    scale = max(1.0, float(np.abs(expect).max()))
    err = np.abs(mean[:, :3] - expect) / scale
    assert err.max() <= 2e-5
    tel = r.collect()
    assert tel.frames_accumulated == 3


def test_converged_cornell_matches_reference_fp64(native, oracle):
    """4096 spp of the GPU path on the reference Cornell fixture agree with the
    reference's FP64 CPU integrator (RenderCornellReference) at 4096 spp:
    64x64 pixels, 8 bounces.  Both are unbiased estimators of the same image
    (triangle-light NEE + MIS with Philox vs rectangle-light NEE with PCG), so
    the difference is Monte Carlo noise: mean within 1%, RMSE below 0.01."""
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    sd = scenes.cornell_reference()
    w = h = 64
    scene, r = _setup(sd, w, h, 8)
    for f in range(4096):
        r.render(frame_constants(sd.camera, w, h, f, 8), accumulate=f > 0)
    r.collect()
    gpu = r.read(FILM_MEAN, w * h)[:, :3].reshape(h, w, 3)
    ref, _ = oracle.ref_cornell(w, h, 4096, 8, 1, 0)
    assert abs(gpu.mean() - ref.mean()) / ref.mean() < 0.01
    assert np.sqrt(((gpu - ref) ** 2).mean()) < 0.01


def test_frame_contract_rejections(native):
    sd = scenes.cornell_box()
    scene, r = _setup(sd, 64, 64, 4)
    bad = frame_constants(sd.camera, 64, 64, 0, 4)
    bad["russian_roulette"] = [3.5, 0.05, 0.95, 1e-4]  # non-integral start
    from renderingengine_b200 import _native as N
    with pytest.raises(N.NativeError) as e:
        r.render(bad)
    assert e.value.code == N.INVALID_ARGUMENT
    big = frame_constants(sd.camera, 128, 64, 0, 4)
    with pytest.raises(N.NativeError):
        r.render(big)
    deep = frame_constants(sd.camera, 64, 64, 0, 5)
    with pytest.raises(N.NativeError):
        r.render(deep)
    pcf = frame_constants(sd.camera, 64, 64, 0, 4)
    pcf["output"][0, 3] = 0
    with pytest.raises(N.NativeError) as e:
        r.render(pcf)
    assert e.value.code == N.UNSUPPORTED
