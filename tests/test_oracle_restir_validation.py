"""The reuse gates of the ReSTIR restatement (oracle_pbr.cpp: validate_pair,
the spatial neighbour gate, temporal_gate -- the production passes'
RestirValidateSurfacePairV3 and RestirTemporalV3 / RestirSpatialV3 checks)
against the reference's CPU validation (src/restir/RestirDi.cpp:181-293,
ValidateTemporalHistory / ValidateSpatialNeighbor, compiled into
oracle/_ref), on the inputs where the two reference implementations agree.

The production passes report the first failing check as one
RestirRejectionReason code (contracts/RestirAbiV3.hpp:82-98); the CPU code
ORs every failing check into a RejectionReason mask
(include/restir/RestirTypes.hpp:84-103).  Shared inputs: surface identity
(material, instance), relative depth, normal cosine and position distance
against the thresholds, the neighbour reservoir's validity, the history's
scene / light / camera / resolution generations, age and the reprojection.
Not shared, so held fixed: the CPU's thin-geometry test (the production ABI
has no thin flag; its code 9 labels a position mismatch), and the
production's stale-frame and surface-validity checks (the CPU takes the
history as handed to it; here a stale history is handed over as invalid).
"""
import numpy as np
import pytest

# RejectionReason bits of the CPU code.
EMPTY, OUTSIDE, MOTION, CUT, RESIZE = 1 << 0, 1 << 1, 1 << 2, 1 << 3, 1 << 4
DEPTH, NORMAL, INSTANCE, THIN, SCENE = 1 << 5, 1 << 6, 1 << 7, 1 << 8, 1 << 9
LIGHT_GEN, LIGHT_DELETED, AGE, INVALID, MATERIAL, POSITION = 1 << 10, 1 << 11, 1 << 12, 1 << 13, 1 << 14, 1 << 15

# Production code -> the CPU bits that name the same failure.
CODE_BITS = {1: EMPTY, 2: OUTSIDE, 3: MOTION, 4: CUT, 5: RESIZE, 6: DEPTH, 7: NORMAL, 8: INSTANCE, 9: POSITION,
             10: SCENE, 11: LIGHT_GEN | LIGHT_DELETED, 12: AGE, 13: MATERIAL}
# The spatial gate's order of checks (validate_pair, then the reservoir).
SPATIAL_ORDER = (13, 8, 6, 7, 9, 1)

THRESHOLDS = [(0.9063078, 0.05, 0.10), (0.8, 0.05, 0.02)]  # ReuseConfig defaults; the renderer's defaults


def _need_ref(oracle):
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")


def _unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def _surfaces(rng, n):
    """Valid GpuPrimarySurfaceV2 records: position, depth, normals,
    albedos in [0, 1], roughness 0.5, identity (material, instance,
    primitive, valid flag)."""
    s = np.zeros((n, 24), np.float32)
    s[:, 0:3] = rng.uniform(-2, 2, (n, 3))
    s[:, 3] = rng.uniform(0.5, 20.0, n)
    nrm = _unit(rng.normal(size=(n, 3))).astype(np.float32)
    s[:, 4:7] = nrm
    s[:, 7] = 0.5
    s[:, 8:11] = nrm
    s[:, 12:15] = 0.5
    s[:, 16:19] = 0.04
    ids = s.view(np.uint32)
    ids[:, 20] = rng.integers(0, 4, n)
    ids[:, 21] = rng.integers(0, 4, n)
    ids[:, 22] = rng.integers(0, 1000, n)
    ids[:, 23] = 1
    return s


def _perturbed(rng, s, thr):
    """Neighbours / histories straddling every threshold: the position moved
    by up to twice the distance threshold, the normal turned by up to twice
    the threshold angle, the depth scaled by up to twice the relative
    threshold either way, identity kept with probability 0.85 each."""
    cos_t, rel, dist = thr
    n = len(s)
    b = s.copy()
    off = _unit(rng.normal(size=(n, 3))) * rng.uniform(0, 2 * dist, (n, 1))
    b[:, 0:3] += off.astype(np.float32)
    ang = rng.uniform(0, 2 * np.arccos(cos_t), n)
    axis = _unit(np.cross(s[:, 8:11], rng.normal(size=(n, 3))))
    nrm = s[:, 8:11] * np.cos(ang)[:, None] + axis * np.sin(ang)[:, None]
    b[:, 8:11] = nrm.astype(np.float32)
    b[:, 3] = (s[:, 3] * (1 + rng.uniform(-2 * rel, 2 * rel, n))).astype(np.float32)
    ids = b.view(np.uint32)
    flip = rng.random(n) > 0.85
    ids[flip, 20] = (ids[flip, 20] + 1) % 4
    flip = rng.random(n) > 0.85
    ids[flip, 21] = (ids[flip, 21] + 1) % 4
    return b


def _ref_geo_ids(a, b):
    """Reference SurfaceRecord packing: 7 floats (position, shading normal,
    linear depth) and 5 words (instance, primitive, material, scene
    generation, thin) per surface."""
    n = len(a)
    geo = np.zeros((n, 14), np.float32)
    ids = np.zeros((n, 14), np.uint32)
    for k, s in enumerate((a, b)):
        w = s.view(np.uint32)
        geo[:, 7 * k:7 * k + 3] = s[:, 0:3]
        geo[:, 7 * k + 3:7 * k + 6] = s[:, 8:11]
        geo[:, 7 * k + 6] = s[:, 3]
        ids[:, 5 * k + 0] = w[:, 21]
        ids[:, 5 * k + 1] = w[:, 22]
        ids[:, 5 * k + 2] = w[:, 20]
        ids[:, 5 * k + 3] = 1
    return geo, ids


def _rparams(oracle, thr, n_lights=8, max_age=20):
    rp = np.zeros(1, oracle.RESTIR_PARAMS_DTYPE)
    rp["normal_cos"], rp["rel_depth"], rp["position_dist"] = thr
    rp["max_age"] = max_age
    rp["scene_gen"], rp["light_gen"], rp["camera_gen"], rp["resolution_gen"] = 3, 5, 7, 2
    rp["history_gen"] = 1
    rp["frame_lo"], rp["frame_hi"] = 100, 0
    rp["light_count"] = rp["prev_light_count"] = n_lights
    return rp


@pytest.mark.parametrize("thr", THRESHOLDS)
def test_spatial_gate_matches_reference(oracle, thr):
    """The spatial neighbour gate accepts exactly the pairs
    ValidateSpatialNeighbor accepts, and its reason is the first of the
    CPU's reasons in the production order."""
    _need_ref(oracle)
    rng = np.random.default_rng(11)
    n = 40000
    a = _surfaces(rng, n)
    b = _perturbed(rng, a, thr)
    valid = (rng.random(n) < 0.85).astype(np.uint32)
    got = oracle.restir_spatial_gate(a, b, valid, _rparams(oracle, thr))
    geo, ids = _ref_geo_ids(a, b)
    ids[:, 10] = valid
    ids[:, 11] = 0        # age
    ids[:, 12] = 5        # selected light generation = current
    ids[:, 13] = 1        # light exists
    mask = oracle.ref_restir_validate("spatial", geo, ids, np.full(n, 5), thr, 20)
    assert ((got == 0) == (mask == 0)).all()
    first = np.zeros(n, np.uint32)
    for code in reversed(SPATIAL_ORDER):
        first = np.where(mask & CODE_BITS[code], code, first)
    assert (got == first).all()
    # Every check is exercised on both sides of its threshold.
    for code in SPATIAL_ORDER:
        assert (got == code).sum() > 100, code
    assert (got == 0).sum() > 1000


def test_spatial_gate_zero_normal(oracle):
    """A zero shading normal: the production gate rejects the surface as
    invalid (1), the CPU code as a normal mismatch (Normalize returns zero);
    both reject."""
    _need_ref(oracle)
    rng = np.random.default_rng(3)
    a = _surfaces(rng, 64)
    b = a.copy()
    b[:, 8:11] = 0.0
    got = oracle.restir_spatial_gate(a, b, np.ones(64, np.uint32), _rparams(oracle, THRESHOLDS[0]))
    geo, ids = _ref_geo_ids(a, b)
    ids[:, 10], ids[:, 12], ids[:, 13] = 1, 5, 1
    mask = oracle.ref_restir_validate("spatial", geo, ids, np.full(64, 5), THRESHOLDS[0], 20)
    assert (got == 1).all() and (mask & NORMAL).all()


@pytest.mark.parametrize("thr", THRESHOLDS)
def test_temporal_gate_matches_reference(oracle, thr):
    """The temporal history gate accepts exactly the histories
    ValidateTemporalHistory accepts (camera static between the frames, so the
    reprojected depth is the current depth), and the reason it reports is one
    of the CPU's reasons."""
    _need_ref(oracle)
    rng = np.random.default_rng(23)
    n = 40000
    rp = _rparams(oracle, thr)
    cur = _surfaces(rng, n)
    hist = _perturbed(rng, cur, thr)
    # Reprojection: 0 inside, 2 outside, 3 no valid reprojection; prior pixel outside the frame.
    reproj = rng.choice([0, 2, 3], n, p=[0.9, 0.05, 0.05]).astype(np.uint32)
    prior_out = rng.random(n) < 0.02
    hist.view(np.uint32)[prior_out, 23] |= np.uint32(1 << 31)
    h = np.zeros((n, 64), np.uint32)
    hf = h.view(np.float32)
    h[:, 40] = rng.integers(1, 40, n)                                 # M
    h[:, 41] = rng.integers(0, 26, n)                                 # age
    valid = rng.random(n) < 0.95
    h[:, 42] = valid.astype(np.uint32)                                # flags: valid
    stale = rng.random(n) < 0.03
    h[:, 56] = np.where(stale, 98, 99)                                # written in the previous frame
    h[:, 57], h[:, 58], h[:, 59] = 0, 1, 1
    gens = np.array([3, 5, 7, 2], np.uint32)
    hs = np.tile(gens, (n, 1))
    for k in range(4):
        d = rng.random(n) < 0.04
        hs[d, k] += 1
    h[:, 52:56] = hs
    h[:, 20] = hs[:, 1]                                               # selected light's generation
    light = np.where(rng.random(n) < 0.03, 9, rng.integers(0, 8, n))  # index 9 >= 8 lights: deleted
    h[:, 27] = light
    hf[:, 0:3] = 1.0
    got = oracle.restir_temporal_gate(cur, hist, h, reproj, cur[:, 3], rp)

    geo, ids = _ref_geo_ids(cur, hist)
    ids[:, 3] = 3                     # current scene generation
    ids[:, 8] = hs[:, 0]              # history's scene generation
    ids[:, 10] = (valid & ~stale).astype(np.uint32)
    ids[:, 11] = h[:, 41]
    ids[:, 12] = hs[:, 1]
    ids[:, 13] = (light < 8).astype(np.uint32)
    flags = (((reproj != 2) & ~prior_out).astype(np.uint32) | ((reproj != 3).astype(np.uint32) << 1)
             | ((hs[:, 2] != 7).astype(np.uint32) << 2) | ((hs[:, 3] != 2).astype(np.uint32) << 3))
    mask = oracle.ref_restir_validate("temporal", geo, ids, np.full(n, 5), thr, 20, flags=flags)
    assert ((got == 0) == (mask == 0)).all()
    rejected = got != 0
    bits = np.array([CODE_BITS.get(int(c), 0) for c in got], np.uint32)
    assert (mask[rejected] & bits[rejected] != 0).all()
    for code in (1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13):
        assert (got == code).sum() > 20, code
    assert (got == 0).sum() > 1000
