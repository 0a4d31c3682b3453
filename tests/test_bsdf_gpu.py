"""The device BSDF (csrc/bsdf.cuh, the functions the Shade kernels call)
through re_bsdf_probe:

- against the FP32 restatement: evaluation bit for bit; sampling decisions
  identical (sampled directions may differ by the last bits of CUDA's vs
  glibc's sinf / cosf);
- against the reference's FP64 BSDF (ReferenceBsdf.hpp) with the
  conditioning-aware bound of tests/bsdf_cases.py;
- statistically, restating the sampling-statistics and energy gates of
  TestSamplingStatisticsAndEnergy (integrators/megakernel/tests/
  MegakernelCpuTests.cpp:545-858) on device samples: the Lambert cosine
  chi-square, PDF normalisation and white furnace, the PDF mass / acceptance
  and first two moments of four finite BSDFs, the smooth-glass Fresnel branch
  frequency, and the metallic-roughness furnace bound with Sample/PDF
  consistency."""
import numpy as np
import pytest

import bsdf_cases as B
from renderingengine_b200 import _native as N

pytestmark = pytest.mark.gpu

SEED = 0x2468ACE013579BDF  # the statistics tests' Philox key


def _probe(q):
    return B.device_probe(N, q)


@pytest.mark.parametrize("model", list(B.MODELS))
def test_device_bsdf_equals_restatement_and_reference(native, oracle, model):
    m = B.MODELS[model]
    q = B.random_queries(m, 40000, seed=7000 + m)
    d = _probe(q)
    o = B.oracle_probe(oracle, q)
    dw, ow = B.as_words(d), B.as_words(o)
    ev = list(range(0, 12)) + [28]
    np.testing.assert_array_equal(d[["eval_valid", "eval_measure", "eval_lobe"]], o[["eval_valid", "eval_measure",
                                                                                       "eval_lobe"]])
    np.testing.assert_array_equal(dw[:, ev].view(np.uint64), ow[:, ev].view(np.uint64),
                                  err_msg="evaluation differs from the FP32 restatement")
    for f in ("sample_valid", "sample_delta", "sample_lobe", "sample_measure"):
        np.testing.assert_array_equal(d[f], o[f], err_msg=f)
    if oracle.ref_available():
        # Against FP64: the device's decisions are the FP32 restatement's
        # (asserted above), whose double instantiation equals the reference
        # (tests/test_oracle_bsdf.py), so a decision flip is FP32 rounding
        # crossing a validity threshold inside the chain: at most 2 in 40,000.
        rep = B.compare_with_reference(oracle, q, d)
        assert rep["decision_mismatches"] <= 2, rep
        assert len(rep["unexplained"]) <= 4, rep


def _frame_queries(n):
    q = np.zeros(n, B.QUERY_DTYPE)
    q["geometric_normal"] = (0, 0, 1)
    q["shading_normal"] = (0, 0, 1)
    q["tangent"] = (1, 0, 0)
    q["eta_incident"], q["eta_transmitted"] = 1.0, 1.5
    q["wo"] = (0, 0, 1)
    q["allowed_lobes"] = B.LOBES_ALL
    # BsdfParamsL6 defaults (ReferenceBsdf.hpp:158-172).
    q["f0"] = (0.04, 0.04, 0.04)
    q["perceptual_roughness"] = 0.5
    q["conductor_eta"] = (1, 1, 1)
    return q


def _randoms(pixel, n, stream, lobe=None):
    i = np.arange(n)
    u = np.zeros((n, 3), np.float32)
    u[:, 0] = B.philox_uniform(pixel, i, B.bounce_dim(0, B.DIM_LOBE), stream, SEED) if lobe is None else lobe
    u[:, 1] = B.philox_uniform(pixel, i, B.bounce_dim(0, B.DIM_BSDF_U), stream, SEED)
    u[:, 2] = B.philox_uniform(pixel, i, B.bounce_dim(0, B.DIM_BSDF_V), stream, SEED)
    return u


def _hemisphere_grid(z_steps=192, phi_steps=384):
    """SampleUniformHemisphere (ReferenceBsdf.hpp:993) on the midpoint grid
    of the reference's quadrature; dOmega = 2 pi / (z_steps phi_steps)."""
    z = (np.arange(z_steps) + 0.5) / z_steps
    ph = (np.arange(phi_steps) + 0.5) / phi_steps
    zz, pp = np.meshgrid(z, ph, indexing="ij")
    s = np.sqrt(np.maximum(0.0, 1 - zz * zz))
    d = np.stack([s * np.cos(2 * np.pi * pp), s * np.sin(2 * np.pi * pp), zz], -1).reshape(-1, 3)
    return d, 2 * np.pi / (z_steps * phi_steps)


def test_lambert_cosine_chi_square_and_furnace(native):
    n, bins = 131072, 16
    q = _frame_queries(n)
    q["model"] = 0
    q["base_color"] = (0.8, 0.35, 0.1)
    q["random"] = _randoms(0, n, 0x57A20002, lobe=0.5)
    r = _probe(q)
    assert (r["sample_valid"] == 1).all()
    np.testing.assert_allclose(r["sample_pdf"], r["pdf_at_sample"], rtol=1e-6)
    z = r["sample_direction"][:, 2].astype(np.float64)
    hist = np.bincount(np.minimum((z * bins).astype(int), bins - 1), minlength=bins)
    lo, hi = np.arange(bins) / bins, (np.arange(bins) + 1) / bins
    expected = n * (hi * hi - lo * lo)
    chi2 = float(((hist - expected) ** 2 / expected).sum())
    assert chi2 <= 45.0, chi2
    d, dw = _hemisphere_grid()
    g = _frame_queries(len(d))
    g["model"] = 0
    g["base_color"] = (0.8, 0.35, 0.1)
    g["wi"] = d
    e = _probe(g)
    assert (e["eval_valid"] == 1).all()
    assert abs(float((e["eval_pdf"].astype(np.float64) * dw).sum()) - 1.0) <= 5e-4
    furnace = (e["eval_value"].astype(np.float64) * (d[:, 2:3] * dw)).sum(0)
    np.testing.assert_allclose(furnace, [0.8, 0.35, 0.1], atol=5e-4)


STATISTICAL = [
    ("ggx_conductor", dict(model=1, f0=(0.9, 0.7, 0.5), perceptual_roughness=0.45)),
    ("ggx_dielectric_reflection", dict(model=2, perceptual_roughness=0.45)),
    ("rough_dielectric", dict(model=4, base_color=(1, 1, 1), transmission=0.85, perceptual_roughness=0.45)),
    ("metallic_roughness", dict(model=5, base_color=(0.8, 0.6, 0.3), f0=(0.04, 0.04, 0.04), metallic=0.35,
                                perceptual_roughness=0.45)),
]


@pytest.mark.parametrize("index,name,params", [(i, n, p) for i, (n, p) in enumerate(STATISTICAL)],
                         ids=[n for n, _ in STATISTICAL])
def test_finite_bsdf_pdf_mass_and_moments(native, index, name, params):
    """Sphere quadrature of PdfBsdfL6 (65,536 z x 4 azimuth midpoints) vs the
    acceptance rate and the mean z, z^2 of 131,072 device samples: the
    reference's gates |mass - pdfMass| <= 0.005 pdfMass + 6 sigma and
    |moment - expected| <= 0.002 + 6 sigma."""
    zs, ps = 65536, 4
    z = -1 + 2 * (np.arange(zs) + 0.5) / zs
    phi = 2 * np.pi * (np.arange(ps) + 0.5) / ps
    zz, pp = np.meshgrid(z, phi, indexing="ij")
    rad = np.sqrt(np.maximum(0.0, 1 - zz * zz))
    d = np.stack([rad * np.cos(pp), rad * np.sin(pp), zz], -1).reshape(-1, 3)
    dw = 4 * np.pi / (zs * ps)
    g = _frame_queries(len(d))
    for k, v in params.items():
        g[k] = v
    g["wi"] = d
    e = _probe(g)
    pdf = np.where((e["eval_valid"] == 1) & (e["eval_measure"] == 1), e["eval_pdf"].astype(np.float64), 0.0)
    assert np.isfinite(pdf).all() and (pdf >= 0).all()
    dz = d[:, 2].astype(np.float32).astype(np.float64)
    mass, ez, ez2 = (pdf * dw).sum(), (dz * pdf * dw).sum(), (dz * dz * pdf * dw).sum()
    assert 0.05 < mass <= 1.005, mass
    n = 131072
    q = _frame_queries(n)
    for k, v in params.items():
        q[k] = v
    q["random"] = _randoms(index + 3, n, 0x57A20001)
    r = _probe(q)
    ok = r["sample_valid"] == 1
    assert (r["sample_delta"][ok] == 0).all() and (r["sample_measure"][ok] == 1).all()
    np.testing.assert_allclose(r["sample_pdf"][ok], r["pdf_at_sample"][ok], rtol=2e-5)
    zv = np.where(ok, r["sample_direction"][:, 2].astype(np.float64), 0.0)
    om, oz, oz2 = ok.mean(), zv.mean(), (zv * zv).mean()
    s_m = np.sqrt(max(0.0, om * (1 - om)) / n)
    s_z = np.sqrt(max(0.0, (zv * zv).mean() - oz * oz) / n)
    s_z2 = np.sqrt(max(0.0, (zv ** 4).mean() - oz2 * oz2) / n)
    assert abs(om - mass) <= 0.005 * mass + 6 * s_m, (om, mass)
    assert abs(oz - ez) <= 0.002 + 6 * s_z, (oz, ez)
    assert abs(oz2 - ez2) <= 0.002 + 6 * s_z2, (oz2, ez2)


def test_smooth_glass_fresnel_branch_frequency(native):
    n = 131072
    q = _frame_queries(n)
    q["model"] = 3
    q["base_color"] = (1, 1, 1)
    q["transmission"] = 1.0
    u = np.full((n, 3), 0.5, np.float32)
    u[:, 0] = B.philox_uniform(9, np.arange(n), B.bounce_dim(0, B.DIM_LOBE), 0x57A20005, SEED)
    q["random"] = u
    r = _probe(q)
    assert (r["sample_valid"] == 1).all() and (r["sample_delta"] == 1).all() and (r["sample_measure"] == 2).all()
    freq = float(((r["sample_lobe"] & 8) != 0).mean())
    f0 = 0.04
    assert abs(freq - f0) <= 6 * np.sqrt(f0 * (1 - f0) / n), freq


@pytest.mark.parametrize("roughness", [0.15, 0.35, 0.70, 1.0])
@pytest.mark.parametrize("metallic", [0.0, 0.5, 1.0])
def test_metallic_roughness_furnace_and_consistency(native, roughness, metallic):
    d, dw = _hemisphere_grid()
    g = _frame_queries(len(d))
    g["model"] = 5
    g["base_color"] = (1, 1, 1)
    g["metallic"] = metallic
    g["perceptual_roughness"] = roughness
    g["wi"] = d
    e = _probe(g)
    assert (e["eval_valid"] == 1).all()
    furnace = (e["eval_value"].astype(np.float64) * (d[:, 2:3] * dw)).sum(0)
    assert np.isfinite(furnace).all() and (furnace >= 0).all() and (furnace <= 1.005).all(), furnace
    n = 16384
    q = _frame_queries(n)
    q["model"] = 5
    q["base_color"] = (1, 1, 1)
    q["metallic"] = metallic
    q["perceptual_roughness"] = roughness
    q["random"] = _randoms(1, n, 0x57A20003)
    r = _probe(q)
    ok = r["sample_valid"] == 1
    assert ok.sum() * 4 >= n
    assert (r["sample_measure"][ok] == 1).all() and (r["sample_delta"][ok] == 0).all()
    assert (r["sample_pdf"][ok] > 0).all() and np.isfinite(r["sample_value"][ok]).all()
    np.testing.assert_allclose(r["sample_pdf"][ok], r["pdf_at_sample"][ok], rtol=2e-5)
