"""Derivatives of the adaptive layered-sphere ensemble on the GPU (one layered component through
scatrs_ensemble_mixture_d: pass 1 refines each requested direction's group from
pass1_layered_deriv_kernel, pass 2 runs the derivative pipeline once per direction group):
every scalar output, beta1 and the phase matrix's F11 and F12 along each layer's Re m and Im m,
the radius fractions and the distribution's median radius, against central differences of the
same GPU path's values at h = 1e-4 of the parameter, with the bounds and the cases of the
reference's own test (scatrs/tests/ensemble_layered.rs:117-276: rtol 1e-11, Greek order 6,
cosines 0.8 and -0.6, a coated sphere with core 1.95 + 0.79i and shell 1.43 + 0.01i at a
wavelength of 0.55, and three layers). The values are pinned to the oracle in
test_gpu_adaptive_layered.py."""

import numpy as np
import pytest

from scatrs_b200 import _scatrs
from scatrs_b200.errors import OutsideValidatedDomainError

pytestmark = pytest.mark.gpu

CORE = 1.95 + 0.79j
SHELL = 1.43 + 0.01j
WL = np.array([0.55])
MU = np.array([0.8, -0.6])
LOGN = ("lognormal", 0.15, 1.5)


def _run(dist, fractions, ms, derivatives=(), rtol=1e-11):
    particle = ("layered", list(fractions), np.array([[m] for m in ms]))
    return _scatrs.ensemble_compute([(dist, particle, 1.0)], WL, False, 6, False, MU, True,
                                    list(derivatives), rtol, 50_000, False, False)


def _check(run, index, value, what):
    """run(v, derivatives) at the parameter's value v; index: its position among the
    parameters (scatrs/tests/ensemble_layered.rs:117-195)."""
    r = run(value, [index])
    h = 1e-4 * max(abs(value), 1e-3)
    plus, minus = run(value + h, []), run(value - h, [])
    d = r["d"][0][:, 0]
    v = r["values"][:, 0]
    for k in range(11):
        fd = (plus["values"][k, 0] - minus["values"][k, 0]) / (2 * h)
        scale = max(abs(fd), abs(v[k]) / max(abs(value), 1e-3), 1e-300)
        assert abs(d[k] - fd) <= 1e-5 * scale, (what, "scalar", k, d[k], fd)
    gd = r["greek_d"][0][4, 0]
    fd = (plus["greek"][4, 0] - minus["greek"][4, 0]) / (2 * h)
    assert np.all(np.abs(gd - fd) <= 1e-5 * np.maximum(np.abs(fd), 1e-3)), (what, "beta1")
    f11 = r["phase"][0, 0]
    for el in (0, 1):
        pd = r["phase_d"][0][el, 0]
        fd = (plus["phase"][el, 0] - minus["phase"][el, 0]) / (2 * h)
        scale = np.maximum(np.abs(fd), f11 / max(abs(value), 1e-3))
        assert np.all(np.abs(pd - fd) <= 1e-5 * scale), (what, "phase", el)
    # The parameter moves C_ext (the check is not passed by zeros).
    assert abs(d[0]) > 1e-4 * abs(v[0]) / max(abs(value), 1e-3), (what, d[0], v[0])
    assert np.all(np.isfinite(r["d_errors"])) and np.all(r["d_errors"] >= 0)


def test_parameter_names():
    names = _scatrs.ensemble_parameters(
        [(LOGN, ("layered", [0.6], np.array([[CORE], [SHELL]])), 1.0)], False)
    assert names == ["median_radius", "width", "layer0.m_real", "layer0.m_imag",
                     "layer1.m_real", "layer1.m_imag", "layer0.radius_fraction"]


def test_radius_fraction(gpu):
    _check(lambda v, d: _run(LOGN, [v], [CORE, SHELL], d), 6, 0.6, "layer0.radius_fraction")


def test_core_index(gpu):
    _check(lambda v, d: _run(LOGN, [0.6], [complex(v, CORE.imag), SHELL], d), 2, CORE.real,
           "layer0.m_real")
    _check(lambda v, d: _run(LOGN, [0.6], [complex(CORE.real, v), SHELL], d), 3, CORE.imag,
           "layer0.m_imag")


def test_shell_index(gpu):
    _check(lambda v, d: _run(LOGN, [0.6], [CORE, complex(v, SHELL.imag)], d), 4, SHELL.real,
           "layer1.m_real")
    _check(lambda v, d: _run(LOGN, [0.6], [CORE, complex(SHELL.real, v)], d), 5, SHELL.imag,
           "layer1.m_imag")


def test_distribution(gpu):
    _check(lambda v, d: _run(("lognormal", v, 1.5), [0.6], [CORE, SHELL], d), 0, 0.15,
           "median_radius")


def test_three_layers(gpu):
    ms = lambda m1: [1.6 + 0.3j, m1, 1.33 + 1e-6j]  # noqa: E731
    # Parameters: median_radius, width, layer0..2 (Re, Im), layer0..1 fractions.
    _check(lambda v, d: _run(LOGN, [0.3, v], ms(2.0 + 0.05j), d), 9, 0.7,
           "three layers: layer1.radius_fraction")
    _check(lambda v, d: _run(LOGN, [0.3, 0.7], ms(complex(2.0, v)), d), 5, 0.05,
           "three layers: layer1.m_imag")


def test_every_direction_at_once(gpu):
    """All seven parameters in one call: each column equals its single call's within the
    refinement (the direction groups refine together)."""
    every = _run(LOGN, [0.6], [CORE, SHELL], range(7), rtol=1e-9)
    for i in (3, 6):
        one = _run(LOGN, [0.6], [CORE, SHELL], [i], rtol=1e-9)
        d_all, d_one = every["d"][i][:, 0], one["d"][0][:, 0]
        scale = np.maximum(np.abs(d_one), 1e-6 * np.abs(every["values"][:, 0]))
        assert np.all(np.abs(d_all - d_one) <= 1e-5 * scale), i


def test_derivatives_need_the_layered_derivative_domain(gpu):
    """x_L near 2e3 at a wavelength of 0.5: the derivatives are validated up to x_L = 1000
    (scatrs/tests/ensemble_layered.rs:379-396); the values alone are validated there."""
    d = ("lognormal", 80.0, 1.1)
    particle = ("layered", [0.5], np.array([[CORE], [SHELL]]))
    wl = np.array([0.5])
    with pytest.raises(OutsideValidatedDomainError, match="derivatives"):
        _scatrs.ensemble_compute([(d, particle, 1.0)], wl, False, None, False, None, True, [6],
                                 1e-3, 4096, False, False)
    ok = _scatrs.ensemble_compute([(d, particle, 1.0)], wl, False, None, False, None, True, [],
                                  1e-3, 4096, False, False)
    assert np.all(np.isfinite(ok["values"]))


def test_single_radius(gpu):
    """A monodisperse ensemble's radius at fixed fractions (particle.rs:221-237, the sum over the
    interfaces of f_l d/dx_l and the outer surface's d/dx_L; scatrs/tests/ensemble_layered.rs:
    237-240): the particle with a vacuum shell of zero thickness gives the outer surface's
    direction."""
    _check(lambda v, d: _run(("monodisperse", v), [0.6], [CORE, SHELL], d), 0, 0.3, "radius")
    ms = [1.6 + 0.3j, 2.0 + 0.05j, 1.33 + 1e-6j]
    _check(lambda v, d: _run(("monodisperse", v), [0.3, 0.7], ms, d), 0, 0.25,
           "three layers: radius")


def test_against_the_oracle_differences(gpu):
    """Every direction of one call against central differences of the oracle's adaptive layered
    ensemble (its own panels and values at rtol 1e-11): a pin of the GPU's derivative blocks
    that does not go through the GPU's values."""
    from oracle import oracle as O

    def oracle(p):  # p: median radius, width, core Re, Im, shell Re, Im, fraction
        d = np.zeros(1, dtype=O.DIST_DTYPE)
        d["kind"] = 1
        d["p"][0, :2] = p[0], p[1]
        ml = np.array([[[complex(p[2], p[3])], [complex(p[4], p[5])]]])
        return O.ensemble_adaptive_layered(d, WL, np.array([[p[6]]]), ml, MU, 6, rtol=1e-11,
                                           max_panels=50_000)

    base = [0.15, 1.5, CORE.real, CORE.imag, SHELL.real, SHELL.imag, 0.6]
    got = _run(LOGN, [0.6], [CORE, SHELL], range(7))
    v = got["values"][:, 0]
    f11 = got["phase"][0, 0]
    for k, value in enumerate(base):
        h = 1e-4 * abs(value)
        plus, minus = list(base), list(base)
        plus[k] += h
        minus[k] -= h
        op, om = oracle(plus), oracle(minus)
        for j in range(11):
            fd = (op["values"][j, 0] - om["values"][j, 0]) / (2 * h)
            scale = max(abs(fd), abs(v[j]) / abs(value), 1e-300)
            assert abs(got["d"][k][j, 0] - fd) <= 1e-5 * scale, (k, j, got["d"][k][j, 0], fd)
        fd = (op["greek"][4, 0] - om["greek"][4, 0]) / (2 * h)
        gd = got["greek_d"][k][4, 0]
        assert np.all(np.abs(gd - fd) <= 1e-5 * np.maximum(np.abs(fd), 1e-3)), (k, "beta1")
        for el in (0, 1):
            fd = (op["phase"][el, 0] - om["phase"][el, 0]) / (2 * h)
            scale = np.maximum(np.abs(fd), f11 / abs(value))
            assert np.all(np.abs(got["phase_d"][k][el, 0] - fd) <= 1e-5 * scale), (k, el)
