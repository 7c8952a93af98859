"""Derivatives of mixtures of different particles on the GPU (scatrs_ensemble_mixture_d through
mixture_hetero_d: each part on its own engine with its derivative blocks, mixed with the weight
derivatives and assembled on the host): the reference's own mixture cases
(scatrs/tests/ensemble_spheroid.rs:335-348, a sphere component and a spheroid component along the
spheroid's aspect ratio; scatrs/tests/ensemble_layered.rs:258-274, a sphere component and a
coated sphere along its radius fraction), and along a sphere component's index, a component's
weight and a spheroid mode's weight, against central differences of the same GPU path's values
at h = 1e-4 of the parameter within 1e-5 (every scalar, alpha1 and beta1 where the Greek
coefficients are asked for, the phase matrix)."""

import numpy as np
import pytest

from scatrs_b200 import _scatrs
from scatrs_b200.errors import InvalidInputError

pytestmark = pytest.mark.gpu

DUST = 1.53 + 0.008j
CORE = 1.95 + 0.79j
SHELL = 1.43 + 0.01j


def _check(run, index, value, what):
    r = run(value, [index])
    h = 1e-4 * max(abs(value), 1e-3)
    plus, minus = run(value + h, []), run(value - h, [])
    d = r["d"][0][:, 0]
    v = r["values"][:, 0]
    for k in range(11):
        fd = (plus["values"][k, 0] - minus["values"][k, 0]) / (2 * h)
        scale = max(abs(fd), abs(v[k]) / max(abs(value), 1e-3), 1e-300)
        assert abs(d[k] - fd) <= 1e-5 * scale, (what, "scalar", k, d[k], fd)
    for k in (0, 4):
        gd = r["greek_d"][0][k, 0]
        fd = (plus["greek"][k, 0] - minus["greek"][k, 0]) / (2 * h)
        assert np.all(np.abs(gd - fd) <= 1e-5 * np.maximum(np.abs(fd), 1e-3)), (what, "greek", k)
    f11 = r["phase"][0, 0]
    pd = r["phase_d"][0][:, 0]
    fd = (plus["phase"][:, 0] - minus["phase"][:, 0]) / (2 * h)
    scale = np.maximum(np.abs(fd), f11[None, :] / max(abs(value), 1e-3))
    assert np.all(np.abs(pd - fd) <= 1e-5 * scale), (what, "phase", np.abs(pd - fd) / scale)
    assert abs(d[0]) > 1e-5 * abs(v[0]) / max(abs(value), 1e-3), (what, d[0], v[0])
    assert np.all(np.isfinite(r["d_errors"])) and np.all(r["d_errors"] >= 0)


def _spheroid_mix(eps=0.5, m_sphere=1.45 + 0j, w1=0.5, rtol=1e-9):
    def run(derivatives):
        items = [(("lognormal", 0.05, 1.5), ("sphere", np.array([m_sphere])), 2.0),
                 (("lognormal", 0.03, 1.4), ("spheroid", eps, np.array([DUST])), w1)]
        return _scatrs.ensemble_compute(items, np.array([1.0]), True, 6, False,
                                        np.array([0.8, -0.6, -1.0]), True, list(derivatives),
                                        rtol, 50_000, False, False)
    return run


def test_names():
    items = [(("lognormal", 0.05, 1.5), ("sphere", [1.45]), 2.0),
             (("lognormal", 0.03, 1.4), ("spheroid", 0.5, [DUST]), 0.5)]
    names = _scatrs.ensemble_parameters(items, True)
    assert names[9] == "c1.aspect_ratio" and names[10] == "c1.weight" and names[2] == "c0.m_real"


def test_spheroid_component_aspect_ratio(gpu):
    _check(lambda v, d: _spheroid_mix(eps=v)(d), 9, 0.5, "c1.aspect_ratio")


def test_sphere_component_index_and_weight(gpu):
    _check(lambda v, d: _spheroid_mix(m_sphere=complex(v, 0.0))(d), 2, 1.45, "c0.m_real")
    _check(lambda v, d: _spheroid_mix(w1=v)(d), 10, 0.5, "c1.weight")


def test_layered_component_radius_fraction(gpu):
    def run(f, derivatives):
        items = [(("lognormal", 0.1, 1.5), ("sphere", np.array([1.45 + 0j])), 2.0),
                 (("lognormal", 0.3, 1.4), ("layered", [f], np.array([[CORE], [SHELL]])), 0.5)]
        return _scatrs.ensemble_compute(items, np.array([0.55]), True, 6, False,
                                        np.array([0.8, -0.6]), True, list(derivatives), 1e-11,
                                        50_000, False, False)
    # c0: median, width, m_real, m_imag, weight; c1: median, width, layer0/1 (Re, Im), fraction.
    _check(run, 11, 0.5, "c1.layer0.radius_fraction")


def test_multimodal_spheroid_mode_weight(gpu):
    """A multimodal spheroid beside a sphere: the weight of the spheroid's second mode."""
    def run(v, derivatives):
        modes = ("multimodal", [(1.0, ("lognormal", 0.03, 1.4)), (v, ("lognormal", 0.06, 1.3))])
        items = [(("lognormal", 0.05, 1.5), ("sphere", np.array([1.45 + 0j])), 2.0),
                 (modes, ("spheroid", 1.8, np.array([DUST])), 0.5)]
        return _scatrs.ensemble_compute(items, np.array([1.0]), True, 6, False,
                                        np.array([0.8, -0.6, -1.0]), True, list(derivatives),
                                        1e-9, 50_000, False, False)
    names = _scatrs.ensemble_parameters(
        [(("lognormal", 0.05, 1.5), ("sphere", [1.45]), 2.0),
         (("multimodal", [(1.0, ("lognormal", 0.03, 1.4)), (0.7, ("lognormal", 0.06, 1.3))]),
          ("spheroid", 1.8, [DUST]), 0.5)], True)
    k = names.index("c1.mode1.weight")
    _check(run, k, 0.7, "c1.mode1.weight")


def test_greek_all(gpu):
    """greek='all' (every wavelength's order 2 N_max over every part, engine.rs:2016-2036): at
    each wavelength the derivatives and coefficients equal a call at that order alone, zero
    above it (pass 1 does not refine on the Greek coefficients, so the panels are the same)."""
    items = [(("lognormal", 0.05, 1.5), ("sphere", np.array([1.45 + 0j, 1.45 + 0j])), 2.0),
             (("lognormal", 0.03, 1.4), ("spheroid", 0.5, np.array([DUST, DUST])), 0.5)]
    wl = np.array([1.0, 0.5])
    a = _scatrs.ensemble_compute(items, wl, True, None, True, None, True, [9, 2], 1e-6, 4096,
                                 False, False)
    width = a["greek"].shape[-1]
    for i in range(wl.size):
        one = [(spec, (p[0],) + p[1:-1] + (p[-1][i:i + 1],), w) for spec, p, w in items]
        order = int(np.max(np.nonzero(np.any(a["greek"][:, i] != 0, axis=0))[0]))
        b = _scatrs.ensemble_compute(one, wl[i:i + 1], True, order, False, None, True, [9, 2],
                                     1e-6, 4096, False, False)
        np.testing.assert_allclose(a["d"][:, :, i], b["d"][:, :, 0], rtol=1e-12, atol=0)
        np.testing.assert_allclose(a["greek"][:, i, :order + 1], b["greek"][:, 0], rtol=1e-12,
                                   atol=1e-300)
        np.testing.assert_allclose(a["greek_d"][:, :, i, :order + 1], b["greek_d"][:, :, 0],
                                   rtol=1e-12, atol=1e-300)
        assert not a["greek_d"][:, :, i, order + 1:].any() and order + 1 <= width


def test_single_sphere_radius_in_a_mixture(gpu):
    """A single sphere radius beside a spheroid: its radius derivative (engine.rs:1158-1170,
    the x pass placed in the part's parameter block) through the mixture's assembly."""
    def run(r, derivatives):
        items = [(("monodisperse", r), ("sphere", np.array([1.45 + 0.01j])), 2.0),
                 (("lognormal", 0.03, 1.4), ("spheroid", 0.5, np.array([DUST])), 0.5)]
        return _scatrs.ensemble_compute(items, np.array([1.0]), True, 6, False,
                                        np.array([0.8, -0.6, -1.0]), True, list(derivatives),
                                        1e-9, 50_000, False, False)
    _check(run, 0, 0.2, "c0.radius")


def test_layered_mixture_against_the_oracle_differences(gpu):
    """A sphere and a coated sphere: the derivatives along the sphere's index, the coating's
    fraction and index and the coated component's weight against central differences of the
    oracle's own mixture (its panels and values at rtol 1e-11)."""
    from oracle import oracle as O

    wl = np.array([0.55])
    mu = np.array([0.8, -0.6])
    base = {"m0": 1.45, "f": 0.5, "si": SHELL.imag, "w1": 0.5}

    def items(p):
        return [(("lognormal", 0.1, 1.5), ("sphere", np.array([complex(p["m0"], 0.0)])), 2.0),
                (("lognormal", 0.3, 1.4),
                 ("layered", [p["f"]], np.array([[CORE], [complex(SHELL.real, p["si"])]])),
                 p["w1"])]

    def oracle(p):
        comps = []
        for (kind, *par), particle, w in items(p):
            d = np.zeros(1, dtype=O.DIST_DTYPE)
            d["kind"], d["p"][0, :2] = 1, par
            m = particle[1] if particle[0] == "sphere" else particle
            comps.append((d, None, w, m))
        return O.ensemble_mixture_d(comps, wl, np.zeros(0, dtype=O.PARAM_DTYPE), mu, 6,
                                    rtol=1e-11, max_panels=50_000)

    names = _scatrs.ensemble_parameters(items(base), True)
    cols = {"m0": names.index("c0.m_real"), "f": names.index("c1.layer0.radius_fraction"),
            "si": names.index("c1.layer1.m_imag"), "w1": names.index("c1.weight")}
    got = _scatrs.ensemble_compute(items(base), wl, True, 6, False, mu, True,
                                   list(cols.values()), 1e-11, 50_000, False, False)
    v = got["values"][:, 0]
    for c, (key, value) in enumerate(base.items()):
        h = 1e-4 * abs(value)
        op, om = oracle({**base, key: value + h}), oracle({**base, key: value - h})
        for j in range(11):
            fd = (op["values"][j, 0] - om["values"][j, 0]) / (2 * h)
            scale = max(abs(fd), abs(v[j]) / abs(value), 1e-300)
            assert abs(got["d"][c][j, 0] - fd) <= 1e-5 * scale, (key, j, got["d"][c][j, 0], fd)
        fd = (op["greek"][0, 0] - om["greek"][0, 0]) / (2 * h)
        assert np.all(np.abs(got["greek_d"][c][0, 0] - fd)
                      <= 1e-5 * np.maximum(np.abs(fd), 1e-3)), (key, "alpha1")
        fd = (op["phase"][:, 0] - om["phase"][:, 0]) / (2 * h)
        scale = np.maximum(np.abs(fd), got["phase"][0, 0][None, :] / abs(value))
        assert np.all(np.abs(got["phase_d"][c][:, 0] - fd) <= 1e-5 * scale), (key, "phase")
