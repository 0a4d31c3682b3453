"""Converged images against closed forms computed in double precision
(tests/analytic_scenes.py): the glass slab pins the smooth-glass Fresnel
branch probabilities, Snell refraction (through the in-medium path length),
the 1 / eta^2 radiance scaling of refraction, Beer-Lambert attenuation
beta *= c^(s / D) (pbr_material_bsdf.hlsli:78-129) and the full MIS weight
of an emitter reached through delta bounces -- against physics, not against
the restatement.  Russian roulette is disabled (rr_start beyond the depth)
so the per-sample distribution is the closed form's.

Per pixel and channel, z = (mean - E) / sqrt((M2 - E^2) / spp); the gates
are max |z| <= 5.5, |mean z| <= 5.5 / sqrt(pixels x 3 / 3) and mean z^2 in
[0.85, 1.15] (the variance of the estimator is the closed form's)."""
import numpy as np
import pytest

import analytic_scenes as A
from renderingengine_b200.wavefront import frame_constants

NO_RR = (1000.0, 0.05, 0.95, 1.0e-4)


def _gates(mean, spp, sd, w, h, depth):
    E, M2 = A.glass_slab_expectation(sd.camera, w, h, depth)
    z = (mean - E) / np.sqrt(np.maximum(M2 - E * E, 1e-30) / spp)
    assert np.abs(z).max() <= 5.5, np.abs(z).max()
    assert np.abs(z.mean()) <= 5.5 / np.sqrt(w * h), z.mean()
    assert 0.85 <= (z * z).mean() <= 1.15, (z * z).mean()
    return float(np.sqrt(((mean - E) ** 2).mean())), float(np.abs(z).max())


def test_oracle_glass_slab_converges_to_the_closed_form(oracle):
    from helpers import host_sah_oracle_inputs
    sd = A.glass_slab()
    w, h, depth, spp = 32, 24, 8, 512
    inp = host_sah_oracle_inputs(oracle, sd)
    acc = np.zeros((w * h, 3))
    for s in range(spp):
        planes, _, _ = oracle.render(inp, frame_constants(sd.camera, w, h, s, depth, rr=NO_RR))
        acc += planes["sample"][:, :3]
    _gates(acc / spp, spp, sd, w, h, depth)


@pytest.mark.gpu
def test_device_glass_slab_converges_to_the_closed_form(native):
    """4096 spp, 64 x 48, on the device's progressive film mean."""
    from renderingengine_b200 import _native as N
    from renderingengine_b200.traversal import Scene
    from renderingengine_b200.wavefront import FILM_MEAN, Renderer
    sd = A.glass_slab()
    w, h, depth, spp = 64, 48, 8, 4096
    scene = Scene(sd.triangles, sd.fingerprint, 1, N.BUILD_LBVH)
    r = Renderer(w, h, depth)
    r.set_scene(scene, sd)
    for s in range(spp):
        r.render(frame_constants(sd.camera, w, h, s, depth, rr=NO_RR), accumulate=s > 0)
    tel = r.collect()
    assert tel.frames_accumulated == spp
    mean = r.read(FILM_MEAN, w * h)[:, :3].astype(np.float64)
    rmse, zmax = _gates(mean, spp, sd, w, h, depth)
    print(f"glass slab 4096 spp: RMSE vs closed form {rmse:.3e}, max |z| {zmax:.2f}")
    r.close()
    scene.close()
