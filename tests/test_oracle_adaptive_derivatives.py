"""The oracle's adaptive engine with derivatives (oracle/oracle_adaptive.cpp,
orc_ensemble_mixture_d) against the reference's own checks (scatrs/tests/ensemble.rs):
every kind of parameter's Jacobian against central differences of the values at rtol 1e-11
(263-466: the scalars to 1e-5 of max(|fd|, |v|/|p|), beta1 to 1e-5 of max(|fd|, 1e-3), F12 to
1e-5 of max(|fd|, F11/|p|)); the error estimates of the derivatives bound their true errors
against a tighter run (469-647, a factor 2 for the unrefined outputs); derivatives that cannot
be resolved within the panel budget are flagged (666-680). A single radius's radius
derivative (engine.rs:1158-1170) is checked the same way (ensemble.rs's "radius" case)."""

import numpy as np
import pytest

from oracle import oracle as O

LAMBDA = 0.55
M = 1.45 + 0.02j
MU = np.array([0.8, -0.6])
PD, RE, IM, W = O.PK_DIST, O.PK_REFR_REAL, O.PK_REFR_IMAG, O.PK_WEIGHT


def _tight(comps, derivs=()):
    return O.ensemble_mixture_d(comps, [LAMBDA], O.params(*derivs) if derivs else
                                np.zeros(0, O.PARAM_DTYPE), mu=MU, greek_order=6, rtol=1e-11,
                                max_panels=50_000)


def _check(make, param, value, what, step=1e-4):
    """check_derivative (ensemble.rs:263-320); `step` relative to the value."""
    r = _tight(make(value), [param])
    h = step * max(abs(value), 1e-3)
    plus, minus = _tight(make(value + h)), _tight(make(value - h))
    d, v = r["d"][0, :, 0], r["values"][:, 0]
    fd = (plus["values"][:, 0] - minus["values"][:, 0]) / (2 * h)
    scale = np.maximum(np.maximum(np.abs(fd), np.abs(v) / max(abs(value), 1e-3)), 1e-300)
    assert np.all(np.abs(d - fd) <= 1e-5 * scale), (what, np.abs(d - fd) / scale)
    gd = r["greek_d"][0, 4, 0]
    gfd = (plus["greek"][4, 0] - minus["greek"][4, 0]) / (2 * h)
    assert np.all(np.abs(gd - gfd) <= 1e-5 * np.maximum(np.abs(gfd), 1e-3)), what
    pd = r["phase_d"][0, 1, 0]
    pfd = (plus["phase"][1, 0] - minus["phase"][1, 0]) / (2 * h)
    f11 = r["phase"][0, 0]
    assert np.all(np.abs(pd - pfd) <= 1e-5 * np.maximum(np.abs(pfd), f11 / max(abs(value), 1e-3))), what


def _one(d, m=M):
    return [(d, None, 1.0, np.array([m]))]


@pytest.mark.parametrize("what,make,param,value", [
    ("median_radius", lambda v: _one(O.dist(1, v, 1.6)), (0, -1, PD, 0), 0.2),
    ("width", lambda v: _one(O.dist(1, 0.2, v)), (0, -1, PD, 1), 1.6),
    ("m_real", lambda v: _one(O.dist(1, 0.2, 1.6), complex(v, 0.02)), (0, -1, RE, 0), 1.45),
    ("m_imag", lambda v: _one(O.dist(1, 0.2, 1.6), complex(1.45, v)), (0, -1, IM, 0), 0.02),
    ("effective_radius", lambda v: _one(O.dist(2, v, 0.1)), (0, -1, PD, 0), 0.5),
    ("effective_variance", lambda v: _one(O.dist(2, 0.5, v)), (0, -1, PD, 1), 0.1),
    ("b", lambda v: _one(O.dist(3, 2.0, v, 0.5)), (0, -1, PD, 1), 15.0),
    ("gamma", lambda v: _one(O.dist(3, 2.0, 15.0, v)), (0, -1, PD, 2), 0.5),
    ("exponent", lambda v: _one(O.dist(4, v, 0.02, 1.0)), (0, -1, PD, 0), 3.0),
])
def test_jacobians_match_finite_differences(what, make, param, value):
    _check(make, param, value, what)


def _mix(w0, m1=1.53 + 0.01j):
    return [(O.dist(1, 0.1, 1.5), None, w0, np.array([1.45 + 0j])),
            (O.dist(1, 0.8, 1.3), None, 0.5, np.array([m1]))]


def _bimodal(v0, width0=1.5):
    return [(O.join(O.dist(1, 0.1, width0), O.dist(1, 0.8, 1.3)), [v0, 0.5], 1.0,
             np.array([M]))]


@pytest.mark.parametrize("what,make,param,value", [
    ("c0.weight", lambda v: _mix(v), (0, -1, W, 0), 2.0),
    ("c1.m_real", lambda v: _mix(2.0, complex(v, 0.01)), (1, -1, RE, 0), 1.53),
    ("mode0.weight", lambda v: _bimodal(v), (0, 0, W, 0), 2.0),
    ("mode0.width", lambda v: _bimodal(2.0, v), (0, 0, PD, 1), 1.5),
])
def test_mixture_jacobians_match_finite_differences(what, make, param, value):
    _check(make, param, value, what)


@pytest.mark.parametrize("dist,m,lam", [
    (O.dist(1, 0.08, 1.6), 1.43 + 1e-8j, 0.5),
    (O.dist(2, 2.0, 0.1), 1.33 + 1e-3j, 0.65),
    (O.dist(4, 3.5, 0.01, 5.0), 1.5 + 0.01j, 0.5),
])
def test_error_estimates_bound_the_true_errors(dist, m, lam):
    """ensemble.rs:469-647 on the derivatives: every parameter, backscattering refined."""
    n_theta = {1: 2, 2: 2, 4: 1}[int(dist["kind"][0])]
    ps = O.params(*[(0, -1, PD, k) for k in range(n_theta)], (0, -1, RE, 0), (0, -1, IM, 0))
    mu = np.array([1.0, 0.7, 0.0, -1.0])
    run = lambda rtol, mp: O.ensemble_mixture_d(  # noqa: E731
        _one(dist, m), [lam], ps, mu=mu, greek_order=24, rtol=rtol, max_panels=mp,
        refine_backscatter=True)
    a, b = run(1e-6, 4096), run(1e-11, 50_000)
    assert a["converged"][0] and b["converged"][0]
    true = np.abs(a["d"] - b["d"])
    assert np.all(true <= 2.0 * a["d_err"] + 1e-14 * np.abs(b["d"])), np.argwhere(
        true > 2.0 * a["d_err"] + 1e-14 * np.abs(b["d"]))
    for key in ("greek_d", "phase_d"):
        t = np.abs(a[key] - b[key])
        assert np.all(t <= 2.0 * a[key + "_err"] + 1e-13 * np.abs(b[key]).max(axis=-1,
                                                                            keepdims=True))


def test_unresolvable_derivatives_are_flagged():
    """ensemble.rs:666-680."""
    d = O.dist(2, 2.0, 0.1)
    r = O.ensemble_mixture_d(_one(d, 1.33 + 0j), [0.65], O.params((0, -1, IM, 0)),
                             max_panels=512)
    assert not r["converged"][0] and r["panels"][0] <= 512
    assert O.ensemble_mixture_d(_one(d, 1.33 + 0j), [0.65], np.zeros(0, O.PARAM_DTYPE))[
        "converged"][0]


def test_a_single_radius_has_its_m_derivatives_and_its_radius():
    r = O.ensemble_mixture_d(_one(O.dist(O.MONODISPERSE, 0.3)), [LAMBDA],
                             O.params((0, -1, RE, 0)), mu=MU, greek_order=6)
    h = 1e-6
    p = O.ensemble_mixture_d(_one(O.dist(O.MONODISPERSE, 0.3), M + h), [LAMBDA],
                             np.zeros(0, O.PARAM_DTYPE), mu=MU, greek_order=6)
    q = O.ensemble_mixture_d(_one(O.dist(O.MONODISPERSE, 0.3), M - h), [LAMBDA],
                             np.zeros(0, O.PARAM_DTYPE), mu=MU, greek_order=6)
    fd = (p["values"] - q["values"]) / (2 * h)
    assert np.allclose(r["d"][0], fd, rtol=1e-6, atol=1e-9 * np.abs(r["values"]).max())
    assert np.all(r["d_err"] == 0.0)
    _check(lambda v: _one(O.dist(O.MONODISPERSE, v)), (0, -1, PD, 0), 0.3, "radius")
    # x = 24 with a nearly real m: ripple resonances make the 1e-4 step's truncation error
    # about 5e-4 relative, so the step is 5e-6 relative here.
    _check(lambda v: _one(O.dist(O.MONODISPERSE, v), 1.33 + 1e-8j), (0, -1, PD, 0), 2.1,
           "radius, nearly real m", step=5e-6)
    r = O.ensemble_mixture_d(_one(O.dist(O.MONODISPERSE, 0.3)), [LAMBDA],
                             O.params((0, -1, PD, 0)), mu=MU, greek_order=6)
    assert np.all(r["d_err"] == 0.0) and r["converged"][0]
