"""Alpha-masked geometry (row (f)2) in the oracle's traversal: the
checkerboard quad against its closed form (a ray through a texel centre hits
the masked quad exactly where the checker keeps it, else the backstop behind
it), factor-only masks, and invalid mappings ending the traversal as
invalid -- the acceptance rule of pbr_software_traversal.hlsli:207-240,
430-470."""
import numpy as np

import alpha_scenes as S
from helpers import host_sah_oracle_inputs


def _rays(x, y):
    r = np.zeros((len(x), 8), np.float32)
    r[:, 0], r[:, 1], r[:, 2], r[:, 3] = x, y, 1.0, 1e-4
    r[:, 6], r[:, 7] = -1.0, 1e30
    return r


def _grid():
    c = (np.arange(S.CHECKER * 4) + 0.5) / (S.CHECKER * 4)
    x, y = np.meshgrid(c, c)
    return x.ravel(), y.ravel()


def test_checkerboard_closed_form(oracle):
    sd = S.checker_quads()
    inp = host_sah_oracle_inputs(oracle, sd)
    x, y = _grid()
    for any_hit in (False, True):
        res = oracle.trace(inp.nodes, inp.tri_v, inp.tri_key, _rays(x, y), any_hit=any_hit, alpha=inp.alpha)
        assert (res["status"] == 0).all()
        keep = S.checker_expected(x, y)
        np.testing.assert_array_equal(res["t"] == np.float32(1.0), keep)
        np.testing.assert_array_equal(res["t"] == np.float32(2.0), ~keep)


def test_factor_only_and_invalid_mappings(oracle):
    sd = S.checker_quads()
    x, y = _grid()
    cases = [(S.v0_material(0.4, 0.5), "transparent"), (S.v0_material(0.6, 0.5), "opaque"),
             (S.v0_material(1.0, 0.5, 5, S.SAMPLER), "invalid"),        # layer beyond the atlas
             (S.v0_material(1.0, 0.5, 0, S.SAMPLER + 1), "invalid"),    # another sampler
             (S.v0_material(1.0, 0.5, S.INVALID, S.SAMPLER), "invalid")]  # sampler without a layer
    for mat, want in cases:
        sd.extra["alpha"]["materials"] = np.concatenate([mat, S.v0_material()])
        inp = host_sah_oracle_inputs(oracle, sd)
        res = oracle.trace(inp.nodes, inp.tri_v, inp.tri_key, _rays(x, y), alpha=inp.alpha)
        if want == "invalid":
            assert (res["status"] == 3).all() and (res["tri"] == 0xFFFFFFFF).all()
        else:
            assert (res["status"] == 0).all()
            assert (res["t"] == np.float32(2.0 if want == "transparent" else 1.0)).all()
    # No coverage data at all: a masked candidate is invalid.
    sd.extra.pop("alpha")
    inp = host_sah_oracle_inputs(oracle, sd)
    res = oracle.trace(inp.nodes, inp.tri_v, inp.tri_key, _rays(x, y), alpha=inp.alpha)
    assert (res["status"] == 3).all()
