"""Mixtures of different particles in the oracle's adaptive engine (one flat layout per
wavelength: the spheres' cosine and band tables, the spheroids' direct Greek segment; mixed with
the number fractions, then projected and assembled, engine.rs:1964-2250, 2396-2497) against the
reference's checks: spheres with coated spheres average with the number weights
(scatrs/tests/ensemble_layered.rs:276-301), spheres with spheroids average their scalars,
unnormalized Greek coefficients and phase matrix, and the mixture depolarizes less than the
spheroids alone (ensemble_spheroid.rs:351-397, here at aspect ratio 1.5, where the oracle's
double-precision T-matrix converges over the whole size range); and a spheroid mixed with a
sphere of weight 0 is the spheroid alone."""

import numpy as np

from oracle import oracle as O

NONE = np.zeros(0, O.PARAM_DTYPE)


def test_spheres_and_layered_spheres_average_with_the_number_weights():
    wl = [0.55]
    d0, d1 = O.dist(1, 0.1, 1.5), O.dist(1, 0.3, 1.4)
    core, shell = 1.95 + 0.79j, 1.43 + 0.01j
    mixed = O.ensemble_mixture_d([(d0, None, 2.0, np.array([1.45 + 0j])),
                                  (d1, None, 0.5, ("layered", [0.5], [[core], [shell]]))],
                                 wl, NONE, greek_order=4)
    a = O.ensemble_adaptive(d0, wl, 1.45 + 0j, greek_order=4)
    b = O.ensemble_adaptive_layered(d1, wl, np.array([[0.5]]), np.array([[[core], [shell]]]),
                                    greek_order=4)
    fa, fb = 2.0 / 2.5, 0.5 / 2.5
    close = lambda x, y: abs(x - y) <= 1e-14 * abs(y)  # noqa: E731
    va, vb, vm = a["values"][:, 0], b["values"][:, 0], mixed["values"][:, 0]
    assert close(vm[0], fa * va[0] + fb * vb[0]) and close(vm[2], fa * va[2] + fb * vb[2])
    sca = fa * va[1] + fb * vb[1]
    g = (fa * va[1] * va[5] + fb * vb[1] * vb[5]) / sca
    assert abs(vm[5] - g) <= 1e-13


def test_spheres_and_spheroids_average_with_the_weights():
    mu = np.array([0.5, -1.0])
    wl = [1.0]
    d0, d1 = O.dist(1, 0.05, 1.5), O.dist(1, 0.08, 1.4)
    dust = 1.53 + 0.008j
    kw = dict(mu=mu, greek_order=4, normalized=False)
    mixed = O.ensemble_mixture_d([(d0, None, 2.0, np.array([1.45 + 0j])),
                                  (d1, None, 0.5, ("spheroid", 1.5, [dust]))], wl, NONE, **kw)
    a = O.ensemble_adaptive(d0, wl, 1.45 + 0j, **kw)
    b = O.ensemble_adaptive_spheroid(d1, wl, 1.5, np.array([dust]), **kw)
    fa, fb = 2.0 / 2.5, 0.5 / 2.5
    vm, va, vb = mixed["values"][:, 0], a["values"][:, 0], b["values"][:, 0]
    assert abs(vm[0] - (fa * va[0] + fb * vb[0])) <= 1e-14 * abs(vm[0])
    want = fa * a["greek"][:, 0] + fb * b["greek"][:, 0]
    assert np.all(np.abs(mixed["greek"][:, 0] - want) <= 1e-14 * a["greek"][0, 0, 0])
    pw = fa * a["phase"][:, 0] + fb * b["phase"][:, 0]
    assert np.all(np.abs(mixed["phase"][:, 0] - pw) <= 1e-13 * a["phase"][0, 0][None])
    assert np.array_equal(a["phase"][2, 0], a["phase"][0, 0])
    assert 0.0 < vm[7] < vb[7]


def test_a_spheroid_with_a_weightless_sphere_is_the_spheroid():
    mu = np.array([1.0, 0.2, -1.0])
    wl = [0.8]
    d = O.dist(1, 0.05, 1.5)
    kw = dict(mu=mu, greek_order=6)
    mixed = O.ensemble_mixture_d([(O.dist(1, 0.2, 1.3), None, 0.0, np.array([1.4 + 0j])),
                                  (d, None, 1.0, ("spheroid", 1.5, [1.5 + 0.01j]))], wl, NONE,
                                 **kw)
    alone = O.ensemble_adaptive_spheroid(d, wl, 1.5, np.array([1.5 + 0.01j]), **kw)
    for key in ("values", "errors", "greek", "greek_err", "phase", "phase_err"):
        assert np.allclose(mixed[key], alone[key], rtol=1e-14, atol=0), key
