"""The ReSTIR reservoir core of the restatement (oracle_pbr.cpp, the float
arithmetic of resources/shaders/restir/RestirProductionV3.hlsli) against the
reference's own CPU reservoir code (src/restir/Reservoir.cpp, compiled into
oracle/_ref), and the reference's L9 reservoir statistics
(tests/unit/L9/RestirTestsMain.cpp:109-230)."""
import numpy as np
import pytest


def _need_ref(oracle):
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")


def _terms(rng, n, zero_fraction=0.2):
    target = rng.lognormal(0.0, 2.0, n).astype(np.float32)
    target[rng.random(n) < zero_fraction] = 0.0
    pdf = rng.lognormal(0.0, 1.5, n).astype(np.float32)
    t = np.zeros((n, 4), np.float32)
    t[:, 0] = target
    t[:, 1] = pdf
    t[:, 2] = (target > 0).astype(np.float32)  # support is binary in the production ABI
    t[:, 3] = 1.0
    return t


def test_float_ris_selects_what_the_reference_selects(oracle):
    """Same candidates and random numbers: the same winner (up to decisions
    within float rounding of a tie), the same M, and W equal to the
    reference's double-precision W within float rounding."""
    _need_ref(oracle)
    rng = np.random.default_rng(7)
    trials, same = 4000, 0
    for _ in range(trials):
        n = int(rng.integers(1, 48))
        t = _terms(rng, n)
        u = rng.random(n).astype(np.float32)
        max_m = int(rng.integers(1, 64))
        s0, ws0, w0, m0 = oracle.restir_ris(t, u, max_m)
        s1, ws1, w1, m1 = oracle.ref_restir_ris(t, u, max_m)
        assert m0 == m1
        if s0 == s1:
            same += 1
            if s0 >= 0:
                assert abs(w0 - w1) <= 2e-5 * abs(w1)
                assert abs(ws0 - ws1) <= 2e-5 * abs(ws1)
    assert same / trials >= 0.999


def test_equal_and_weighted_selection_frequencies(oracle):
    """TestEqualReservoirStatistics / TestWeightedReservoirStatistics: winner
    frequencies within 0.012 of the normalised weights, M == 4."""
    rng = np.random.default_rng(0x12345678)
    for weights, trials in (([1.0, 1.0, 1.0, 1.0], 50000), ([1.0, 2.0, 3.0, 4.0], 75000)):
        t = np.zeros((4, 4), np.float32)
        t[:, 0] = weights
        t[:, 1] = 1.0
        t[:, 2] = 1.0
        t[:, 3] = 1.0
        counts = np.zeros(4)
        for _ in range(trials // 10):
            for _ in range(10):
                sel, _, _, m = oracle.restir_ris(t, rng.random(4).astype(np.float32), 4)
                assert m == 4
                counts[sel] += 1
        freq = counts / counts.sum()
        expect = np.asarray(weights) / np.sum(weights)
        assert np.all(np.abs(freq - expect) <= 0.012)


def test_candidate_contract_and_m_clamp(oracle):
    """TestCandidateContractAndInitialRis (RestirTestsMain.cpp:159-230) under
    the production ABI's binary support: zero-target candidates count toward
    M without winning; a zero proposal pdf is rejected; clamping M to 2 of 4
    candidates of weights 1, 10, 100, 1000 leaves a weight sum of 555.5 in
    either order."""
    t = np.array([[1.0, 0.5, 1, 1], [2.0, 0.25, 1, 1], [0.0, 0.25, 0, 1]], np.float32)
    sel, ws, w, m = oracle.restir_ris(t, np.array([0.3, 0.7, 0.1], np.float32), 2)
    assert m == 2 and w > 0 and sel in (0, 1)
    bad = np.array([[1.0, 0.0, 1, 1]], np.float32)
    assert oracle.restir_ris(bad, np.array([0.5], np.float32), 8)[3] == 0
    cap = np.array([[1, 1, 1, 1], [10, 1, 1, 1], [100, 1, 1, 1], [1000, 1, 1, 1]], np.float32)
    u = np.array([0.1, 0.2, 0.3, 0.4], np.float32)
    fwd = oracle.restir_ris(cap, u, 2)
    rev = oracle.restir_ris(cap[::-1], u, 2)
    assert fwd[3] == rev[3] == 2
    assert fwd[1] == rev[1] == 555.5
