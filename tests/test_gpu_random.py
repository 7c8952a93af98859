"""Randomly oriented spheroids on the GPU (scatrs_spheroid_compute: the double-double T-matrix
and the orientation average by the rank decomposition, random.cu) against the oracle's
restatement of random.rs and the reference's own checks: the brute-force average at one angle
(random.rs:343-355), a sphere giving Mie's efficiencies and Greek coefficients, the phase
function integrating to the scattering cross section (alpha1_0), and the converged records.

Tolerances: Greek coefficients within 1e-12 of alpha1_0 of the oracle's (the same T-matrix to
1e-26; Clebsch-Gordan coefficients by a recursion here and Racah's formula there), 2e-6 at the
brute-force angle (the published digits), Mie identities within 1e-12."""

import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from scatrs_b200 import _native

pytestmark = pytest.mark.gpu

RECORDS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "spheroid.json")))


def _phase_from_greek(g, mu):
    """F11, F12, F22, F33, F34, F44 from Greek coefficients (tmatrix/mod.rs:494-516)."""
    L = g.shape[1] - 1
    out = np.zeros((6, len(mu)))
    for j, u in enumerate(mu):
        d00, d22, d2m2, d02 = (O.wigner_d(a, b, u, L) for a, b in ((0, 0), (2, 2), (2, -2), (0, 2)))
        s = np.dot(g[1] + g[2], d22)
        d = np.dot(g[1] - g[2], d2m2)
        out[:, j] = [np.dot(g[0], d00), np.dot(g[4], d02), 0.5 * (s + d), 0.5 * (s - d),
                     np.dot(g[5], d02), np.dot(g[3], d00)]
    return out


@pytest.mark.parametrize("x,eps,s,n,nt", [(2.0, 1.8, 1.5 + 0.02j, 6, 15),
                                          (3.0, 0.5, 1.5 + 0.02j, 10, 30),
                                          (4.0, 3.0, 1.53 + 0.008j, 16, 40),
                                          (1.2, 0.6, 1.33 + 0.0j, 8, 20)])
def test_greek_matches_the_oracle(gpu, x, eps, s, n, nt):
    r = _native.spheroid_compute([x], [eps], [s], n_terms=n, n_theta=nt, greek_order=2 * n + 3,
                                 normalized=False)
    g = r["greek"][0] * x * x / 4.0  # raw, 1/k^2
    modes = O.tmatrix_modes(x, eps, s, n, nt, quad=True)
    want = O.random_greek(modes, 2 * n)
    assert np.abs(g[:, : 2 * n + 1] - want).max() <= 1e-12 * want[0, 0]
    assert np.all(g[:, 2 * n + 1:] == 0.0)
    # alpha1_0 = C_sca / (4 pi) and the efficiencies from T.
    qe, qs = O.spheroid_q(x, eps, s, n, nt, quad=True)
    eff = r["efficiencies"][0]
    assert abs(eff[0] - qe) <= 1e-13 * qe and abs(eff[1] - qs) <= 1e-13 * qs
    assert abs(g[0, 0] - qs * x * x / 4.0) <= 1e-12 * g[0, 0]
    assert abs(eff[4] - want[0, 1] / (3 * want[0, 0])) <= 1e-12


def test_matches_the_brute_force_average(gpu):
    r = _native.spheroid_compute([2.0], [1.8], [1.5 + 0.02j], n_terms=6, n_theta=15,
                                 greek_order=12, normalized=False)
    g = r["greek"][0] * 4.0 / 4.0  # x = 2: raw = unnormalized x^2/4
    f = _phase_from_greek(g, [np.cos(0.4)])[:, 0]
    want = [6.980506, -0.33857, 6.912394, 6.902738, 0.118319, 6.84077]
    assert np.abs(f - want).max() < 2e-6


def test_a_sphere_gives_mie(gpu):
    x, m, n = 3.0, 1.5 + 0.01j, 14
    r = _native.spheroid_compute([x], [1.0], [m], n_terms=n, n_theta=30, greek_order=2 * n)
    mie = O.mie(x, m, n_max=n)
    eff = r["efficiencies"][0]
    for k, key in enumerate(["q_ext", "q_sca", "q_abs", "q_back", "g"]):
        assert abs(eff[k] - mie[key]) <= 1e-12 * max(abs(mie[key]), 1e-3), key
    want = O.mie_greek(x, m, 2 * n)
    got = r["greek"][0]
    assert np.abs(got - want).max() <= 1e-12


def test_converged_records_with_greek(gpu):
    recs = [r for r in RECORDS if r["case"].endswith(",converged")][:6]
    x = np.array([r["x"] for r in recs])
    eps = np.array([r["eps"] for r in recs])
    m = np.array([complex(*r["m"]) for r in recs])
    out = _native.spheroid_compute(x, eps, m, rtol=1e-10, greek_order=8)
    for i, r in enumerate(recs):
        qe = r["q_ext"][0][0] + r["q_ext"][0][1]
        assert abs(out["efficiencies"][i, 0] - qe) <= 1e-9 * qe
        assert out["greek"][i, 0, 0] == 1.0
        assert 0.0 < out["efficiencies"][i, 4] < 1.0
        assert out["error_estimate"][i] <= 2.0 ** -53
    # One member alone gives the same bits.
    one = _native.spheroid_compute(x[2:3], eps[2:3], m[2:3], rtol=1e-10, greek_order=8)
    assert np.array_equal(one["greek"][0], out["greek"][2])
    assert np.array_equal(one["efficiencies"][0], out["efficiencies"][2])
