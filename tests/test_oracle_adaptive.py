"""The oracle's restatement of the reference's adaptive engine (oracle/oracle_adaptive.cpp)
against the identities the reference's own ensemble tests check (scatrs/tests/ensemble.rs):
a monodisperse ensemble is the single sphere (62-112), moments and normalizations match the
closed forms (115-156), the Rayleigh limit is the sixth moment (159-174), the normalized phase
function averages to one (177-202), error estimates bound the true errors (469-647, against a
tighter rtol), and a batch matches each distribution within its error estimates (951-1060)."""

import math

import numpy as np
import pytest

from oracle import oracle as O


def _moment(kind, p, k):
    if kind == 1:
        return p[0] ** k * math.exp(k * k * math.log(p[1]) ** 2 / 2)
    if kind == 2:
        a, b = p[0], p[1]
        al = (1 - 3 * b) / b
        return (a * b) ** k * math.exp(math.lgamma(al + 1 + k) - math.lgamma(al + 1))
    if kind == 3:
        al, b, g = p
        return b ** (-k / g) * math.exp(math.lgamma((al + 1 + k) / g) - math.lgamma((al + 1) / g))
    if kind == 4:
        e, lo, hi = p

        def integral(q):
            return (hi ** (q + 1) - lo ** (q + 1)) / (q + 1) if q != -1 else math.log(hi / lo)
        return integral(k - e) / integral(-e)
    raise ValueError(kind)


def test_monodisperse_is_the_single_sphere():
    r, lam, m = 0.7, 0.55, 1.5 + 0.01j
    mu = np.array([1.0, 0.3, -1.0])
    x = 2 * math.pi * r / lam
    L = 2 * O.default_n_max(x)  # GreekOrder::All
    e = O.ensemble_adaptive(O.dist(O.MONODISPERSE, r), [lam], m, mu=mu, greek_order=L)
    s = O.mie(x, m)
    area = math.pi * r * r
    v = e["values"][:, 0]
    assert v[0] == area * s["q_ext"] and v[1] == area * s["q_sca"] and v[2] == area * s["q_abs"]
    assert abs(v[5] - s["g"]) < 1e-15 and abs(v[8] - r) < 1e-15
    assert e["converged"][0] and e["panels"][0] == 0 and np.all(e["errors"] == 0.0)
    g = O.mie_greek(x, m, L)
    assert np.abs(e["greek"][:, 0, :] - g).max() <= 1e-13 * max(abs(g[0, 1]), 1.0)
    s1, s2 = O.amplitudes(x, m, mu)
    c = 4.0 / (x * x) / s["q_sca"]
    f11 = c * 0.5 * (np.abs(s1) ** 2 + np.abs(s2) ** 2)
    assert np.abs(e["phase"][0, 0] - f11).max() <= 1e-13 * f11[0]


@pytest.mark.parametrize("kind,p", [(1, (0.08, 1.6, 0)), (2, (0.5, 0.15, 0)),
                                    (3, (2.0, 15.0, 0.5)), (4, (3.0, 0.02, 1.0))])
def test_moments_and_normalizations_match_the_closed_forms(kind, p):
    e = O.ensemble_adaptive(O.dist(kind, *p), [0.5], 1.45 + 0.001j, greek_order=8, rtol=1e-8)
    v = e["values"][:, 0]
    m2, m3 = _moment(kind, p, 2), _moment(kind, p, 3)
    assert abs(v[9] - math.pi * m2) <= 1e-7 * math.pi * m2
    assert abs(v[10] - 4 * math.pi / 3 * m3) <= 1e-7 * 4 * math.pi / 3 * m3
    assert abs(v[8] - m3 / m2) <= 1e-7 * m3 / m2
    g = e["greek"][:, 0, :]
    assert g[0, 0] == 1.0 and abs(g[0, 1] - 3 * v[5]) < 1e-12
    assert abs(v[0] - v[1] - v[2]) < 1e-12 * v[0] and v[7] == 0.0
    assert abs(v[6] - 4 * math.pi * v[0] / v[3]) < 1e-12 * v[6]
    assert e["converged"][0]


def test_the_rayleigh_limit_is_the_sixth_moment():
    lam, m = 1.0, 1.5 + 0j
    e = O.ensemble_adaptive(O.dist(1, 2e-4, 1.4), [lam], m, rtol=1e-9)
    k = (m * m - 1) / (m * m + 2)
    want = 8 / 3 * (2 * math.pi / lam) ** 4 * abs(k) ** 2 * math.pi * _moment(1, (2e-4, 1.4), 6)
    v = e["values"][:, 0]
    assert abs(v[1] / want - 1) < 1e-5 and v[2] == 0.0 and v[4] == 1.0 and abs(v[5]) < 1e-5


def test_the_normalized_phase_function_averages_to_one():
    x, w = O.gauss_legendre(400)
    e = O.ensemble_adaptive(O.dist(1, 0.3, 1.5), [0.5], 1.33 + 1e-6j, mu=x)
    assert abs((e["phase"][0, 0] * w).sum() / 2 - 1) < 1e-5
    u = O.ensemble_adaptive(O.dist(1, 0.3, 1.5), [0.5], 1.33 + 1e-6j, mu=x, greek_order=4,
                            normalized=False)
    v = u["values"][:, 0]
    assert abs((u["phase"][0, 0] * w).sum() / 2 / v[1] - 1) < 1e-5
    assert abs(u["greek"][0, 0, 0] / v[1] - 1) < 1e-12


def test_error_estimates_bound_the_true_errors():
    mu = np.array([1.0, 0.5, -0.2, -1.0])
    d = np.concatenate([O.dist(1, 0.2, 1.7), O.dist(2, 0.8, 0.1), O.dist(4, 3.5, 0.05, 1.5)])
    wl = [0.45, 0.9]
    m = [1.5 + 0.005j, 1.45 + 1e-6j]
    for rtol in (1e-3, 1e-5):
        a = O.ensemble_adaptive(d, wl, m, mu=mu, greek_order=12, rtol=rtol)
        b = O.ensemble_adaptive(d, wl, m, mu=mu, greek_order=12, rtol=1e-10)
        true = np.abs(a["values"] - b["values"])
        assert np.all(true <= a["errors"] + 1e-15 * np.abs(b["values"])), np.argwhere(
            true > a["errors"])
        for key in ("phase", "greek"):
            t = np.abs(a[key] - b[key])
            assert np.all(t <= a[key + "_err"] + 1e-13 * np.abs(b[key]).max())
        assert np.all(a["converged"])


def test_a_batch_matches_each_distribution():
    d = np.concatenate([O.dist(1, 0.1, 1.5), O.dist(1, 0.4, 1.3), O.dist(2, 0.3, 0.1),
                        O.dist(O.MONODISPERSE, 0.25)])
    wl = [0.4, 0.7]
    m = [1.4 + 1e-3j, 1.35 + 1e-4j]
    mu = np.array([0.9, -0.4])
    single = O.ensemble_adaptive(d, wl, m, mu=mu, greek_order=10)
    batch = O.ensemble_adaptive(d, wl, m, mu=mu, greek_order=10, batch=True)
    err = single["errors"] + batch["errors"]
    assert np.all(np.abs(single["values"] - batch["values"]) <= err + 1e-15)
    # Shared panels: every member of the batch reports the same count per wavelength.
    p = batch["panels"].reshape(4, 2)
    assert np.all(p[:3] == p[0]) and np.all(p[3] == 0)
    assert np.array_equal(single["values"][:, 6:8], batch["values"][:, 6:8])


def test_bad_inputs_are_rejected():
    with pytest.raises(O.OracleError):
        O.ensemble_adaptive(O.dist(1, 0.1, 1.5), [0.5], 1.5, rtol=0.5)
    with pytest.raises(O.OracleError, match="outside|validated"):
        O.ensemble_adaptive(O.dist(1, 0.1, 1.5), [0.5], 1.5 + 20j)


def test_mixtures_average_with_the_number_weights():
    """scatrs/tests/ensemble.rs:205-262."""
    lam, mu = 0.6, np.array([0.5])
    d1, m1, w1 = O.dist(1, 0.1, 1.5), 1.45 + 0j, 2.0
    d2, m2, w2 = O.dist(1, 1.0, 1.3), 1.53 + 0.01j, 0.5
    mix = O.ensemble_mixture([(d1, None, w1, m1), (d2, None, w2, m2)], [lam], mu=mu,
                             greek_order=10)
    a = O.ensemble_adaptive(d1, [lam], m1, mu=mu, greek_order=10)
    b = O.ensemble_adaptive(d2, [lam], m2, mu=mu, greek_order=10)
    fa, fb = w1 / (w1 + w2), w2 / (w1 + w2)
    va, vb, vm = a["values"][:, 0], b["values"][:, 0], mix["values"][:, 0]
    assert abs(vm[0] - (fa * va[0] + fb * vb[0])) <= 1e-12 * vm[0]
    assert abs(vm[10] - (fa * va[10] + fb * vb[10])) <= 1e-12 * vm[10]
    sca = fa * va[1] + fb * vb[1]
    want = (fa * va[1] * a["phase"][0, 0, 0] + fb * vb[1] * b["phase"][0, 0, 0]) / sca
    assert abs(mix["phase"][0, 0, 0] - want) < 1e-10 * want
    want = (fa * va[1] * a["greek"][4, 0, 4] + fb * vb[1] * b["greek"][4, 0, 4]) / sca
    assert abs(mix["greek"][4, 0, 4] - want) < 1e-10 * max(abs(want), 1e-6)
    # A bimodal distribution is a mixture of its modes with one refractive index.
    bi = O.ensemble_mixture([(np.concatenate([d1, d2]), [w1, w2], 1.0, m1)], [lam], mu=mu,
                            greek_order=10)
    both = O.ensemble_mixture([(d1, None, w1, m1), (d2, None, w2, m1)], [lam], mu=mu,
                              greek_order=10)
    assert np.array_equal(bi["values"], both["values"])
    assert bi["panels"][0] == both["panels"][0]


def test_all_orders_are_each_wavelengths_2n_max():
    """GreekOrder::All (engine.rs:2016-2020): each wavelength projects to 2 N_max, its largest
    number of terms, the arrays padded with zeros to the longest (scatrs-py ensemble.rs:419-429):
    the same as that explicit order at that wavelength."""
    d = O.dist(1, 0.3, 1.4)
    wl = [0.4, 1.6]
    mu = np.array([0.5, -0.5])
    a = O.ensemble_adaptive(d, wl, 1.45 + 0.01j, mu=mu, greek_order="all")
    w = a["greek"].shape[-1]
    for i, lam in enumerate(wl):
        g = a["greek"][0, i]
        order = int(np.flatnonzero(g)[-1])  # the last nonzero alpha1: 2 N_max
        assert order % 2 == 0 and np.all(a["greek"][:, i, order + 1:] == 0.0)
        b = O.ensemble_adaptive(d, [lam], 1.45 + 0.01j, mu=mu, greek_order=order)
        assert np.array_equal(a["greek"][:, i, :order + 1], b["greek"][:, 0])
        assert np.array_equal(a["greek_err"][:, i, :order + 1], b["greek_err"][:, 0])
        assert np.array_equal(a["values"][:, i], b["values"][:, 0])
    assert w == order + 1 or w > order + 1
