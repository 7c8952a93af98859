"""The fixed-grid ensemble of randomly oriented spheroids on the GPU
(scatrs_ensemble_fixed_spheroid) against the oracle's restatement of the engine's direct path
over per-node oracle solutions at the same (N, n_theta) per node: the scalars (C_ext, C_sca,
C_abs, C_back, ssa, g, lidar ratio, depolarization ratio, r_eff, mean area and volume), the
Greek coefficients and the phase matrix from the averaged Greek expansion, within 1e-10 (the
oracle's double-precision EBCM at these moderate shapes and sizes carries about 1e-12); and the
sphere limit: aspect ratio 1 equals the sphere ensemble of the same grid."""

import numpy as np
import pytest

from oracle import oracle as O
from scatrs_b200 import _native

pytestmark = pytest.mark.gpu


def _dists():
    d = np.zeros(2, dtype=_native.DIST_DTYPE)
    d["kind"] = 1
    d["param"][0, :2] = [0.12, 1.5]
    d["param"][1, :2] = [0.08, 1.7]
    for i in range(2):
        rg, sg = d["param"][i, 0], d["param"][i, 1]
        d["r_lo"][i], d["r_hi"][i] = rg * sg ** -2.5, rg * sg ** 2.5
    return d


def test_matches_the_oracle(gpu):
    d = _dists()
    wl = np.array([0.55, 0.9])
    eps = np.array([1.6, 0.6])
    m = np.array([[1.5 + 0.01j, 1.52 + 0.003j], [1.33 + 0.0j, 1.45 + 0.05j]])
    mu = np.array([-0.9, -0.4, 0.0, 0.3, 0.7, 0.95])
    values, phase, greek, terms = _native.ensemble_fixed_spheroid(
        d, wl, eps, m, mu, n_nodes=5, greek_order=9, tmatrix_rtol=1e-10)
    want = O.ensemble_fixed_spheroid(d.view(O.DIST_DTYPE), wl, eps, m, 5, terms, mu=mu,
                                     greek_order=9)
    for k in range(11):
        # C_abs is a difference of C_ext and C_sca: measured against C_ext (0 when lossless).
        scale = want["values"][0] if k == 2 else np.abs(want["values"][k])
        assert np.all(np.abs(values[k] - want["values"][k]) <= 1e-10 * scale), k
    assert np.abs(greek - want["greek"]).max() <= 1e-10
    scale = np.abs(want["phase"][0]).max(axis=1, keepdims=True)
    assert np.all(np.abs(phase - want["phase"]) <= 1e-10 * scale)
    # Spheroids depolarize; ratios are in range.
    assert np.all(values[7] > 0) and np.all(values[4] <= 1.0)
    # Normalized: alpha1_0 = 1 and half the integral of F11 is 1 (the Greek expansion's l = 0).
    assert np.all(greek[0, :, 0] == 1.0)


def test_aspect_ratio_one_is_the_sphere_ensemble(gpu):
    d = _dists()
    wl = np.array([0.6])
    m = np.array([[1.45 + 0.002j], [1.55 + 0.02j]])
    mu = np.array([-0.8, 0.1, 0.9])
    v, ph, g, _ = _native.ensemble_fixed_spheroid(d, wl, 1.0, m, mu, n_nodes=6, greek_order=6,
                                                  tmatrix_rtol=1e-11)
    vs, phs, gs = _native.ensemble_fixed(d, wl, m, mu, 6, greek_order=6)
    # Scalars except the depolarization ratio (0 for spheres) to the truncations' difference.
    for k in [0, 1, 2, 3, 4, 5, 6, 8, 9, 10]:
        assert np.allclose(v[k], vs[k], rtol=1e-9), k
    assert np.all(np.abs(v[7]) < 1e-9)
    assert np.abs(g - gs).max() < 1e-9
    assert np.all(np.abs(ph - phs) <= 1e-9 * np.abs(phs[0]).max())
