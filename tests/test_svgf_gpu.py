"""GPU SVGF / A-Trous (csrc/svgf.cu) against the CPU restatement, which is
pinned bit for bit to the reference's SvgfReconstruction
(tests/test_oracle_svgf.py).

Planes without transcendental functions (raw, temporal, moments, history
length, acceptance, reject reasons) must be bit-identical.  Variance and the
two filtered outputs go through expf / powf, whose CUDA results may differ
from glibc's by a few ulp; they must agree within RTOL relative (plus ATOL
absolute) on at least MIN_FRACTION of the values and within LOOSE_RTOL
everywhere."""
import numpy as np
import pytest

import svgf_cases as S
from renderingengine_b200 import _native as N
from renderingengine_b200.svgf import (ReconstructionOutput, SvgfConfig, SvgfReconstruction, compute_psnr,
                                       compute_rmse)

pytestmark = pytest.mark.gpu

RTOL, ATOL, MIN_FRACTION, LOOSE_RTOL = 1e-4, 1e-6, 0.999, 1e-2
EXACT = {"raw": "raw", "temporal": "temporal", "moments": "moments", "history_length": "history_length",
         "accepted_history": "accepted", "reject_reasons": "reject"}
CLOSE = {"variance": "variance", "atrous": "atrous", "svgf": "svgf"}


def _flat(a: np.ndarray) -> np.ndarray:
    if a.dtype.names:
        return np.concatenate([a[n].reshape(a.shape + (-1,)) for n in a.dtype.names], axis=-1)
    return a


def _cfg_pair(**kw):
    native = S.config(**kw)
    return native, SvgfConfig.from_native(native)


def _compare(gpu_frame, ref: dict, where: str):
    for attr, key in EXACT.items():
        g = np.ascontiguousarray(_flat(getattr(gpu_frame, attr)))
        np.testing.assert_array_equal(S.bits(g), S.bits(ref[key].reshape(g.shape)), err_msg=f"{where} {attr}")
    for attr, key in CLOSE.items():
        g = _flat(getattr(gpu_frame, attr)).astype(np.float64)
        r = ref[key].reshape(g.shape).astype(np.float64)
        assert np.isfinite(g).all() == np.isfinite(r).all(), f"{where} {attr}: finiteness differs"
        err = np.abs(g - r)
        ok = err <= ATOL + RTOL * np.abs(r)
        assert ok.mean() >= MIN_FRACTION, f"{where} {attr}: {ok.mean():.5f} within tolerance"
        assert np.all(err <= ATOL + LOOSE_RTOL * np.abs(r)), f"{where} {attr}: max error {err.max():.3g}"


@pytest.mark.parametrize("w,h,frames,seed,flights,cfg", [
    (24, 16, 6, 1, 2, {}),
    (33, 21, 5, 2, 1, {"atrous_iterations": 5, "phi_normal": 128.0}),
    (17, 29, 5, 3, 3, {"demodulate_specular": 0, "require_material_id": 0, "spatial_radius": 1}),
    (20, 12, 4, 4, 2, {"atrous_iterations": 0, "max_history_length": 3, "minimum_color_alpha": 0.0}),
    (40, 8, 4, 5, 2, {"atrous_iterations": 16, "short_history_length": 1, "require_object_id": 0}),
    (12, 10, 40, 7, 2, {"max_history_length": 8}),
    (160, 90, 6, 8, 2, {"atrous_iterations": 5, "phi_normal": 128.0}),
])
def test_gpu_matches_oracle_sequence(native, oracle, w, h, frames, seed, flights, cfg):
    native_cfg, py_cfg = _cfg_pair(**cfg)
    gpu = SvgfReconstruction(w, h, flights, py_cfg)
    ora = oracle.OracleSvgf(w, h, flights, native_cfg)
    for gb, sig, fi, trig in S.sequence(w, h, frames, seed, hostile=frames < 20):
        got = gpu.process(gb, sig, fi, trig)
        ref = ora.process(gb, sig, fi, trig)
        _compare(got, ref, f"frame {fi}")


def test_gpu_resize_config_change_and_device_inputs(native, oracle):
    import torch

    native_cfg, py_cfg = _cfg_pair()
    gpu = SvgfReconstruction(16, 12, 2, py_cfg)
    ora = oracle.OracleSvgf(16, 12, 2, native_cfg)
    seq_a = S.sequence(16, 12, 3, 11)
    seq_b = S.sequence(21, 9, 3, 12)
    steps = [seq_a[0], seq_a[1], seq_b[0], seq_b[1], "config", seq_b[2]]
    for i, step in enumerate(steps):
        if step == "config":
            n2, p2 = _cfg_pair(phi_depth=2.0, atrous_iterations=2)
            gpu.set_config(p2)
            ora.set_config(n2)
            assert gpu.config.phi_depth == 2.0
            continue
        gb, sig, _, trig = step
        if i % 2:  # device-resident inputs through the same entry point
            dg = torch.from_numpy(gb.view(np.uint8).copy()).cuda()
            ds = torch.from_numpy(sig.view(np.uint8).copy()).cuda()
            gpu.process_device(dg.data_ptr(), ds.data_ptr(), gb.shape[1], gb.shape[0], i, trig)
            torch.cuda.synchronize()
            got = gpu.frame()
        else:
            got = gpu.process(gb, sig, i, trig)
        _compare(got, ora.process(gb, sig, i, trig), f"step {i}")


def test_reference_unit_scenarios_on_gpu(native):
    """The reference's L8 expectations (ReconstructionTests.cpp:234-407), run
    on the GPU path."""
    _, cfg = _cfg_pair(minimum_color_alpha=0.0, minimum_moments_alpha=0.0, atrous_iterations=0)
    r = SvgfReconstruction(2, 1, 2, cfg)
    s0 = S.uniform_signal(1, 2, 1.0)
    s0["diffuse"][0, 1] = 2.0
    f0 = r.process(S.valid_gbuffer(1, 2), s0, 0)
    assert f0.history_length[0, 0] == 1 and f0.reject_reasons[0, 0] & 1
    g1 = S.valid_gbuffer(1, 2)
    g1["motion"][0, 1] = (-0.5, 0.0)
    s1 = S.uniform_signal(1, 2, 3.0)
    f1 = r.process(g1, s1, 1)
    assert f1.accepted_history[0, 1] == 1 and f1.history_length[0, 1] == 2
    assert abs(f1.temporal["diffuse"][0, 1, 0] - 2.0) <= 1e-5
    assert abs(f1.moments[0, 1, 0] - 2.0) <= 1e-5 and abs(f1.moments[0, 1, 1] - 5.0) <= 1e-5
    cut = r.process(g1, s1, 2, 1)
    assert cut.history_length[0, 1] == 1 and cut.reject_reasons[0, 1] & 2
    g1["motion"][0, 0] = (2.0, 0.0)
    assert r.process(g1, s1, 3).reject_reasons[0, 0] == 4

    _, cfg = _cfg_pair(atrous_iterations=1, phi_luminance=100000.0)
    r = SvgfReconstruction(10, 1, 2, cfg)
    g = S.valid_gbuffer(1, 10)
    s = np.zeros((1, 10), N.SIGNAL_DTYPE)
    for x in range(10):
        g["object_id"][0, x] = 2 if x >= 5 else 1
        s["diffuse"][0, x] = 4.0 if x >= 5 else 0.25
    g["object_id"][0, 3] = 3
    f = r.process(g, s, 0)
    assert abs(f.atrous["diffuse"][0, 4, 0] - 0.25) <= 1e-4 and abs(f.atrous["diffuse"][0, 5, 0] - 4.0) <= 1e-4


def test_checkerboard_metric_and_outputs(native, oracle):
    """Checkerboard: raw RMSE 0.5 -> A-Trous RMSE 0.00183614 (the reference's
    printed metric), PSNR improves; every SelectOutput surface equals the
    reference's SelectOutput of the same frame."""
    _, cfg = _cfg_pair(atrous_iterations=2, phi_luminance=100000.0)
    g, s = S.checkerboard()
    r = SvgfReconstruction(16, 16, 2, cfg)
    f = r.process(g, s, 0)
    raw = r.select_output(ReconstructionOutput.RAW)
    atr = r.select_output(ReconstructionOutput.ATROUS)
    one = np.ones_like(raw)
    raw_rmse, atr_rmse = compute_rmse(raw, one), compute_rmse(atr, one)
    assert raw_rmse > 0.49 and atr_rmse < raw_rmse
    assert abs(atr_rmse - 0.00183614) < 1e-6
    assert compute_psnr(atr, one) > compute_psnr(raw, one)
    assert f.variance[8, 8] > 1e-6
    if not oracle.ref_available():
        return
    native_cfg = S.config(atrous_iterations=2, phi_luminance=100000.0)
    ref = oracle.RefSvgf(16, 16, 2, native_cfg)
    ref.process(g, s, 0)
    g2 = g.copy()
    g2["motion"] = np.random.default_rng(1).normal(scale=0.01, size=(16, 16, 2))
    for out in ReconstructionOutput:
        got = r.select_output(out, g2)
        want = ref.select_output(g2, int(out))
        np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-7, err_msg=str(out))


def test_full_size_720p_sequence(native, oracle):
    """1280x720 with the many-light workload's settings (5 iterations,
    phi_normal 128): three frames, every plane against the restatement."""
    native_cfg, py_cfg = _cfg_pair(atrous_iterations=5, phi_normal=128.0)
    gpu = SvgfReconstruction(1280, 720, 2, py_cfg)
    ora = oracle.OracleSvgf(1280, 720, 2, native_cfg)
    for gb, sig, fi, trig in S.sequence(1280, 720, 3, 21):
        _compare(gpu.process(gb, sig, fi, trig), ora.process(gb, sig, fi, trig), f"720p frame {fi}")


def test_contract_errors(native):
    with pytest.raises(N.NativeError) as e:
        SvgfReconstruction(4, 4, 1, SvgfConfig(minimum_albedo=0.0))
    assert e.value.code == N.INVALID_ARGUMENT
    with pytest.raises(N.NativeError):
        SvgfReconstruction(0, 4, 1)
    r = SvgfReconstruction(4, 4, 1)
    with pytest.raises(N.NativeError) as e:
        r.read(0)
    assert e.value.code == N.NOT_READY
    with pytest.raises(ValueError):
        r.process(S.valid_gbuffer(4, 4), S.uniform_signal(4, 5, 1.0), 0)
