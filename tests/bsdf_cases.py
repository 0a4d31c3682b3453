"""Seeded BSDF probe queries (the 160-byte re_bsdf_query layout) over every
material model and both transport modes, and helpers that run them through
the oracle restatement (FP32), the reference's FP64 BSDF and the device."""
from __future__ import annotations

import ctypes as C

import numpy as np

QUERY_DTYPE = np.dtype([
    ("geometric_normal", "<f4", 3), ("eta_incident", "<f4"),
    ("shading_normal", "<f4", 3), ("eta_transmitted", "<f4"),
    ("tangent", "<f4", 3), ("transport_mode", "<u4"),
    ("base_color", "<f4", 3), ("metallic", "<f4"),
    ("f0", "<f4", 3), ("perceptual_roughness", "<f4"),
    ("conductor_eta", "<f4", 3), ("transmission", "<f4"),
    ("conductor_k", "<f4", 3), ("model", "<u4"),
    ("wo", "<f4", 3), ("allowed_lobes", "<u4"),
    ("wi", "<f4", 3), ("use_complex_conductor_fresnel", "<u4"),
    ("random", "<f4", 3), ("reserved", "<u4")])
assert QUERY_DTYPE.itemsize == 160

RESULT_DTYPE = np.dtype([
    ("eval_value", "<f4", 3), ("eval_pdf", "<f4"),
    ("eval_diffuse", "<f4", 3), ("eval_measure", "<u4"),
    ("eval_specular", "<f4", 3), ("eval_lobe", "<u4"),
    ("sample_direction", "<f4", 3), ("sample_pdf", "<f4"),
    ("sample_value", "<f4", 3), ("sample_eta", "<f4"),
    ("sample_diffuse", "<f4", 3), ("sample_measure", "<u4"),
    ("sample_specular", "<f4", 3), ("sample_lobe", "<u4"),
    ("eval_valid", "<u4"), ("sample_delta", "<u4"), ("sample_valid", "<u4"), ("pdf_at_sample", "<f4")])
assert RESULT_DTYPE.itemsize == 128

# The reference's FP64 results: the same fields as doubles (integers as
# exact double values).
RESULT64_DTYPE = np.dtype([(name, "<f8", sub[1]) if len(sub) > 1 and sub[1] else (name, "<f8")
                           for name, sub in [(n, RESULT_DTYPE.fields[n][0].subdtype or (None, ()))
                                             for n in RESULT_DTYPE.names]])
assert RESULT64_DTYPE.itemsize == 256

MODELS = {"lambert": 0, "ggx_conductor": 1, "ggx_dielectric_reflection": 2, "smooth_glass": 3,
          "rough_dielectric": 4, "metallic_roughness": 5}
LOBES_ALL = 31


def _unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def random_queries(model: int, count: int, seed: int, transport: int | None = None,
                   tilted_shading: bool = True) -> np.ndarray:
    """`count` queries of one model: random frames (shading normal tilted up to
    ~0.35 rad from the geometric one), outgoing directions in the geometric
    hemisphere, incident directions over the sphere, material parameters over
    their valid ranges, random triples in [0, 1)."""
    rng = np.random.default_rng(seed)
    q = np.zeros(count, QUERY_DTYPE)
    ng = _unit(rng.normal(size=(count, 3)))
    tilt = _unit(rng.normal(size=(count, 3))) * (rng.uniform(0, 0.35, (count, 1)) if tilted_shading else 0.0)
    ns = _unit(ng + tilt)
    q["geometric_normal"] = ng
    q["shading_normal"] = ns
    q["tangent"] = _unit(rng.normal(size=(count, 3)))
    inside = rng.random(count) < 0.3
    eta = rng.uniform(1.2, 1.8, count)
    q["eta_incident"] = np.where(inside, eta, 1.0)
    q["eta_transmitted"] = np.where(inside, 1.0, eta)
    q["transport_mode"] = rng.integers(0, 2, count) if transport is None else transport
    q["base_color"] = rng.uniform(0.02, 1.0, (count, 3))
    q["metallic"] = rng.uniform(0, 1, count)
    q["f0"] = np.where(rng.random((count, 1)) < 0.5, 0.04, rng.uniform(0.02, 1.0, (count, 3)))
    q["perceptual_roughness"] = rng.uniform(0.05, 1.0, count)
    q["conductor_eta"] = rng.uniform(0.2, 3.0, (count, 3))
    q["conductor_k"] = rng.uniform(0.0, 5.0, (count, 3))
    q["transmission"] = rng.uniform(0, 1, count)
    q["model"] = model
    q["allowed_lobes"] = LOBES_ALL
    q["use_complex_conductor_fresnel"] = rng.integers(0, 2, count) if model == 1 else 0
    # Outgoing directions mostly well inside the geometric hemisphere.
    d = _unit(rng.normal(size=(count, 3)))
    d = np.where((d * ng).sum(-1, keepdims=True) < 0, -d, d)
    q["wo"] = _unit(d + ng * 0.15)
    q["wi"] = _unit(rng.normal(size=(count, 3)))
    q["random"] = rng.random((count, 3), dtype=np.float32) * np.float32(1 - 2 ** -24)
    return q


def oracle_probe(oracle, queries: np.ndarray) -> np.ndarray:
    q = np.ascontiguousarray(queries, QUERY_DTYPE)
    out = np.zeros(len(q), RESULT_DTYPE)
    oracle.oracle_lib().oracle_bsdf_probe(q.ctypes.data, len(q), out.ctypes.data)
    return out


def reference_probe(oracle, queries: np.ndarray) -> np.ndarray:
    q = np.ascontiguousarray(queries, QUERY_DTYPE)
    out = np.zeros(len(q), RESULT64_DTYPE)
    oracle.ref_lib().ref_bsdf_probe(q.ctypes.data, len(q), out.ctypes.data)
    return out


def device_probe(native_module, queries: np.ndarray) -> np.ndarray:
    """re_bsdf_probe on host buffers (the library stages them through device
    memory)."""
    N = native_module
    q = np.ascontiguousarray(queries, QUERY_DTYPE)
    out = np.zeros(len(q), RESULT_DTYPE)
    N.check(N.load().re_bsdf_probe(q.ctypes.data, len(q), out.ctypes.data, N.MEMORY_HOST, None))
    return out


def vec(r, name) -> np.ndarray:
    """Field `name` as an (n, k) float64 array."""
    a = np.asarray(r[name], np.float64)
    return a.reshape(len(r), -1)


def philox_uniform(pixel, sample, dim, stream, seed: int) -> np.ndarray:
    """Vectorised Philox4x32-10 counter random float (the reference's
    CounterRandomFloat, integrators/megakernel/MegakernelBridge.cpp:552-600):
    counter (pixel, sample, dim, stream), key = the 64-bit seed, result
    (x >> 8) * 2^-24."""
    shape = np.broadcast(np.asarray(pixel), np.asarray(sample), np.asarray(dim), np.asarray(stream)).shape
    c0, c1, c2, c3 = (np.broadcast_to(np.asarray(v, np.uint64), shape).copy() for v in (pixel, sample, dim, stream))
    k0 = np.uint64(seed & 0xFFFFFFFF)
    k1 = np.uint64((seed >> 32) & 0xFFFFFFFF)
    m32 = np.uint64(0xFFFFFFFF)
    for _ in range(10):
        p0 = np.uint64(0xD2511F53) * c0
        p1 = np.uint64(0xCD9E8D57) * c2
        n0 = (p1 >> np.uint64(32)) ^ c1 ^ k0
        n1 = p1 & m32
        n2 = (p0 >> np.uint64(32)) ^ c3 ^ k1
        n3 = p0 & m32
        c0, c1, c2, c3 = n0, n1, n2, n3
        k0 = (k0 + np.uint64(0x9E3779B9)) & m32
        k1 = (k1 + np.uint64(0xBB67AE85)) & m32
    return ((c0 >> np.uint64(8)).astype(np.float64) * 2.0 ** -24).astype(np.float32)


def bounce_dim(bounce: int, local: int) -> int:
    """BounceSampleDimension (MegakernelBridge.hpp:426): 4 + 16 b + local."""
    return 4 + 16 * bounce + local


DIM_LOBE, DIM_BSDF_U, DIM_BSDF_V = 5, 6, 7


# ---------------------------------------------------------------------------
# FP32-vs-FP64 comparison with the conditioning of each query made explicit.
# ---------------------------------------------------------------------------
RTOL, ATOL = 4e-4, 1e-5      # per component, on top of the conditioning terms
D_ULPS = 32                  # FP32 ulps of the half vector's z fed through GGX D
SPREAD_FACTOR = 4.0          # multiple of the FP64 spread under 1-ulp input perturbations
DECISIONS = ("eval_valid", "eval_measure", "eval_lobe", "sample_valid", "sample_delta", "sample_lobe",
             "sample_measure")


def ggx_d_condition(q: np.ndarray, wi: np.ndarray, transmission: np.ndarray) -> np.ndarray:
    """|d ln D / d ln z| of the GGX distribution at the half vector of (wo,
    wi) -- the reflection half vector, or -(eta_i wo + eta_t wi) for a
    transmission -- against the shading normal: 4 / (z^2 (a^2 + t^2)) - 4
    with t^2 = (1 - z^2) / z^2.  Near a narrow lobe's peak this grows like
    2 / a^2, and an FP32 result carries that many ulps of z's rounding."""
    with np.errstate(invalid="ignore", divide="ignore"):
        wo = _unit(np.asarray(q["wo"], np.float64))
        w = np.asarray(wi, np.float64)
        w = w / (np.linalg.norm(w, axis=1, keepdims=True) + 1e-300)
        ns = _unit(np.asarray(q["shading_normal"], np.float64))
        ei = np.asarray(q["eta_incident"], np.float64)[:, None]
        et = np.asarray(q["eta_transmitted"], np.float64)[:, None]
        h = np.where(np.asarray(transmission)[:, None], -(ei * wo + et * w), wo + w)
        h = h / (np.linalg.norm(h, axis=1, keepdims=True) + 1e-300)
        z = np.clip(np.abs((h * ns).sum(1)), 1e-12, 1.0)
        a = np.asarray(q["perceptual_roughness"], np.float64) ** 2
        k = np.abs(4.0 / (z * z * (a * a + (1 - z * z) / (z * z))) - 4.0)
    k[~np.isfinite(k)] = 0.0
    lam = np.asarray(q["model"]) == MODELS["lambert"]
    k[lam] = 0.0
    return k


def perturbed(q: np.ndarray, rng, eps: float = 2.0 ** -23) -> np.ndarray:
    """The queries with every direction component and random number scaled
    by 1 + U(-eps, eps): the FP32 rounding of the inputs and of the first
    quantities derived from them."""
    p = q.copy()
    for f in ("wo", "wi", "geometric_normal", "shading_normal", "tangent", "random"):
        p[f] = (np.asarray(p[f], np.float64) * (1 + rng.uniform(-eps, eps, p[f].shape))).astype(np.float32)
    return p


def _excess(got, want, kappa, scale_spread=None):
    """Per query: max over components of |got - want| / tolerance."""
    g = np.asarray(got, np.float64).reshape(len(got), -1)
    w = np.asarray(want, np.float64).reshape(len(want), -1)
    tol = RTOL * np.abs(w) + ATOL + D_ULPS * kappa[:, None] * 2.0 ** -24 * np.abs(w)
    if scale_spread is not None:
        tol = tol + SPREAD_FACTOR * scale_spread.reshape(len(w), -1)
    with np.errstate(invalid="ignore"):
        return np.max(np.abs(g - w) / tol, axis=1)


def compare_with_reference(oracle, q: np.ndarray, got: np.ndarray, perturbations: int = 16) -> dict:
    """Compares FP32 probe results `got` (oracle restatement or device) with
    the reference's FP64 BSDF on the same queries.

    - Decisions (validity, measure, lobe, delta) must agree, or the query must
      be ill-conditioned at the FP32 input level: some FP64 evaluation of the
      query with its inputs perturbed by one FP32 rounding reproduces the FP32
      decision.
    - Evaluated value / diffuse / specular / pdf, where both are valid: within
      RTOL |r| + ATOL + D_ULPS kappa_D eps |r|; beyond that only if within the
      FP64 spread under 1-ulp input perturbations (x SPREAD_FACTOR).
    - A finite sample: its value and pdf against the FP64 evaluation at the
      FP32 sampled direction (the sampled direction's own rounding is then
      not amplified through a narrow lobe), its direction against the FP64
      sample's within 2e-5 or the perturbation spread; pdf_at_sample against
      the FP64 PdfBsdfL6 at that direction.
    - A delta sample: direction and value against the FP64 sample.
    Returns counts and the indices left unexplained."""
    n = len(q)
    r = reference_probe(oracle, q)
    rng = np.random.default_rng(12345)
    rep = {"queries": n, "unexplained": []}

    def perturbed_runs(idx, wi_override=None):
        runs = []
        for _ in range(perturbations):
            qq = q[idx].copy()
            if wi_override is not None:
                qq["wi"] = wi_override
            runs.append(reference_probe(oracle, perturbed(qq, rng)))
        return runs

    # Decisions.
    dec_bad = np.zeros(n, bool)
    for f in DECISIONS:
        dec_bad |= np.asarray(got[f], np.float64) != np.asarray(r[f], np.float64)
    idx = np.nonzero(dec_bad)[0]
    rep["decision_mismatches"] = int(len(idx))
    if len(idx):
        runs = perturbed_runs(idx)
        for j, i in enumerate(idx):
            ok = True
            for f in DECISIONS:
                if float(got[f][i]) != float(r[f][i]):
                    ok &= any(float(run[f][j]) == float(got[f][i]) for run in runs)
            if not ok:
                rep["unexplained"].append(("decision", int(i)))
    agree = ~dec_bad

    # Evaluation.
    ev = agree & (np.asarray(got["eval_valid"]) == 1)
    kap = ggx_d_condition(q, q["wi"], (np.asarray(got["eval_lobe"]) & 16) != 0)
    worst = np.zeros(n)
    for f in ("eval_value", "eval_diffuse", "eval_specular", "eval_pdf"):
        worst = np.maximum(worst, np.where(ev, _excess(got[f], r[f], kap), 0.0))
    idx = np.nonzero(worst > 1)[0]
    rep["eval_compared"] = int(ev.sum())
    rep["eval_beyond_base_tolerance"] = int(len(idx))
    if len(idx):
        runs = perturbed_runs(idx)
        for j, i in enumerate(idx):
            for f in ("eval_value", "eval_diffuse", "eval_specular", "eval_pdf"):
                spread = np.max([np.abs(np.asarray(run[f][j], np.float64) - np.asarray(r[f][i], np.float64))
                                 for run in runs], axis=0)
                if _excess(got[f][i:i + 1], r[f][i:i + 1], kap[i:i + 1], np.atleast_1d(spread))[0] > 1:
                    rep["unexplained"].append((f, int(i)))
                    break

    # Finite samples: against the FP64 evaluation at the FP32 direction.
    fs = agree & (np.asarray(got["sample_valid"]) == 1) & (np.asarray(got["sample_delta"]) == 0)
    q2 = q.copy()
    q2["wi"] = got["sample_direction"]
    r2 = reference_probe(oracle, q2)
    fs_eval = fs & (np.asarray(r2["eval_valid"]) == 1)
    rep["sample_compared"] = int(fs.sum())
    rep["sample_direction_not_evaluable"] = int((fs & ~fs_eval).sum())
    kap2 = ggx_d_condition(q, got["sample_direction"], (np.asarray(got["sample_lobe"]) & 16) != 0)
    worst = np.zeros(n)
    for f, g in (("sample_value", "eval_value"), ("sample_diffuse", "eval_diffuse"),
                 ("sample_specular", "eval_specular"), ("sample_pdf", "eval_pdf"), ("pdf_at_sample", "eval_pdf")):
        worst = np.maximum(worst, np.where(fs_eval, _excess(got[f], r2[g], kap2), 0.0))
    ddir = np.abs(vec(got, "sample_direction") - vec(r, "sample_direction")).max(axis=1)
    rep["sample_direction_max_abs"] = float(ddir[fs].max()) if fs.any() else 0.0
    idx = np.nonzero((worst > 1) | (fs & (ddir > 2e-5)) | (fs & ~fs_eval))[0]
    rep["sample_beyond_base_tolerance"] = int(len(idx))
    if len(idx):
        runs = perturbed_runs(idx)
        runs2 = perturbed_runs(idx, wi_override=got["sample_direction"][idx])
        for j, i in enumerate(idx):
            sd = np.max([np.abs(vec(run[j:j + 1], "sample_direction")[0] - vec(r[i:i + 1], "sample_direction")[0])
                         for run in runs], axis=0)
            if ddir[i] > 2e-5 + SPREAD_FACTOR * sd.max():
                rep["unexplained"].append(("sample_direction", int(i)))
                continue
            if not fs_eval[i]:
                # FP64 rejects the FP32 direction: it must sit at a validity edge.
                if not any(run["eval_valid"][j] == 1 for run in runs2):
                    rep["unexplained"].append(("sample_direction_rejected", int(i)))
                continue
            for f, g in (("sample_value", "eval_value"), ("sample_pdf", "eval_pdf")):
                spread = np.max([np.abs(np.asarray(run[g][j], np.float64) - np.asarray(r2[g][i], np.float64))
                                 for run in runs2], axis=0)
                if _excess(got[f][i:i + 1], r2[g][i:i + 1], kap2[i:i + 1], np.atleast_1d(spread))[0] > 1:
                    rep["unexplained"].append((f, int(i)))
                    break

    # Delta samples.
    ds = agree & (np.asarray(got["sample_valid"]) == 1) & (np.asarray(got["sample_delta"]) == 1)
    rep["delta_compared"] = int(ds.sum())
    worst = np.zeros(n)
    for f in ("sample_value", "sample_specular", "sample_pdf", "sample_eta"):
        worst = np.maximum(worst, np.where(ds, _excess(got[f], r[f], np.zeros(n)), 0.0))
    idx = np.nonzero((worst > 1) | (ds & (ddir > 2e-5)))[0]
    rep["delta_beyond_base_tolerance"] = int(len(idx))
    if len(idx):
        runs = perturbed_runs(idx)
        for j, i in enumerate(idx):
            for f in ("sample_direction", "sample_value", "sample_specular", "sample_pdf", "sample_eta"):
                spread = np.max([np.abs(np.asarray(run[f][j], np.float64) - np.asarray(r[f][i], np.float64))
                                 for run in runs], axis=0)
                if _excess(got[f][i:i + 1], r[f][i:i + 1], np.zeros(1), np.atleast_1d(spread))[0] > 1:
                    rep["unexplained"].append((f, int(i)))
                    break
    return rep


def oracle_probe64(oracle, queries: np.ndarray) -> np.ndarray:
    """The oracle's BSDF instantiated in double (oracle/oracle_bsdf64.cpp)."""
    q = np.ascontiguousarray(queries, QUERY_DTYPE)
    out = np.zeros(len(q), RESULT64_DTYPE)
    oracle.oracle_lib().oracle_bsdf_probe64(q.ctypes.data, len(q), out.ctypes.data)
    return out


def as_words(r: np.ndarray) -> np.ndarray:
    """Results as an (n, 32) array of float64 (integers as exact values)."""
    if r.dtype == RESULT64_DTYPE:
        return r.view(np.float64).reshape(len(r), 32)
    out = np.zeros((len(r), 32))
    col = 0
    for name in RESULT_DTYPE.names:
        a = np.asarray(r[name], np.float64).reshape(len(r), -1)
        out[:, col:col + a.shape[1]] = a
        col += a.shape[1]
    return out
