"""Derivatives of the adaptive spheroid ensemble on the GPU (one spheroid component through
scatrs_ensemble_mixture_d): every scalar output, the Greek coefficients alpha1 and beta1 and the
phase matrix along the aspect ratio (oblate and prolate), Re m, Im m, the lognormal's median
radius and width, and a single radius's radius, against central differences of the same GPU
path's values at h = 1e-4 of the parameter, with the bounds and the case of the reference's
own test (scatrs/tests/ensemble_spheroid.rs:227-350: rtol 1e-9, Greek order 6, cosines 0.8,
-0.6, -1, m = 1.53 + 0.008i at a wavelength of 1). The values themselves are pinned to the
oracle in test_gpu_adaptive_spheroid.py."""

import numpy as np
import pytest

from scatrs_b200 import _scatrs
from scatrs_b200.errors import InvalidInputError

pytestmark = pytest.mark.gpu

DUST = 1.53 + 0.008j
WL = np.array([1.0])
MU = np.array([0.8, -0.6, -1.0])


def _run(dist, eps, m, derivatives=()):
    item = (dist, ("spheroid", eps, np.array([m])), 1.0)
    return _scatrs.ensemble_compute([item], WL, False, 6, False, MU, True, list(derivatives),
                                    1e-9, 50_000, False, False)


def _check(run, index, value, what):
    """run(v, derivatives) at the parameter's value v; index: its position among the
    parameters (scatrs/tests/ensemble_spheroid.rs:229-290)."""
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
    # The parameter moves C_ext (the check is not passed by zeros).
    assert abs(d[0]) > 1e-4 * abs(v[0]) / max(abs(value), 1e-3), (what, d[0], v[0])
    # The derivative call's error estimates are there and finite.
    assert np.all(np.isfinite(r["d_errors"])) and np.all(r["d_errors"] >= 0)
    return r


LOGN = ("lognormal", 0.03, 1.4)


@pytest.mark.parametrize("eps", [2.0, 0.5])
def test_aspect_ratio(gpu, eps):
    names = _scatrs.ensemble_parameters([(LOGN, ("spheroid", eps, [DUST]), 1.0)], False)
    assert names == ["median_radius", "width", "m_real", "m_imag", "aspect_ratio"]
    _check(lambda v, d: _run(LOGN, v, DUST, d), 4, eps, "aspect_ratio")


def test_refractive_index(gpu):
    _check(lambda v, d: _run(LOGN, 2.0, complex(v, DUST.imag), d), 2, DUST.real, "m_real")
    _check(lambda v, d: _run(LOGN, 2.0, complex(DUST.real, v), d), 3, DUST.imag, "m_imag")


def test_distribution(gpu):
    _check(lambda v, d: _run(("lognormal", v, 1.4), 2.0, DUST, d), 0, 0.03, "median_radius")
    _check(lambda v, d: _run(("lognormal", 0.03, v), 2.0, DUST, d), 1, 1.4, "width")


def test_single_radius(gpu):
    """A monodisperse ensemble's radius at a fixed aspect ratio (monodisperse_direct,
    engine.rs:1896-1961): 2/r times the values plus (2 pi / lambda) d/dx."""
    _check(lambda v, d: _run(("monodisperse", v), 2.0, DUST, d), 0, 0.2, "radius")


def test_every_direction_at_once(gpu):
    """All five parameters in one call give each one's derivative of the single calls (the
    direction blocks refine together; each column's values agree within the refinement)."""
    all5 = _run(LOGN, 2.0, DUST, [0, 1, 2, 3, 4])
    for i in (2, 4):
        one = _run(LOGN, 2.0, DUST, [i])
        d_all, d_one = all5["d"][i][:, 0], one["d"][0][:, 0]
        scale = np.maximum(np.abs(d_one), 1e-6 * np.abs(all5["values"][:, 0]))
        assert np.all(np.abs(d_all - d_one) <= 1e-6 * scale), i


def test_a_sphere_has_no_aspect_ratio(gpu):
    d = gpu.dist_records(1)
    d["kind"][0] = gpu.KINDS["lognormal"]
    d["param"][0, :2] = (0.2, 1.5)
    comps = [(d, None, 1.0, np.array([1.5 + 0j]))]
    bad = np.array([(0, -1, gpu.PARAM_ASPECT_RATIO, 0)], dtype=gpu.PARAM_DTYPE)
    with pytest.raises(InvalidInputError, match="no parameter aspect_ratio"):
        gpu.ensemble_mixture_d(comps, [0.5], bad)


def test_against_the_oracle_differences(gpu):
    """The aspect ratio, Re m, Im m and median radius in one call against central differences
    of the oracle's own adaptive spheroid ensemble (its panels, its double-precision EBCM and
    Racah-based orientation average per node, rtol 1e-9): a pin of the GPU's derivative blocks
    that does not go through the GPU's values."""
    from oracle import oracle as O

    base = [0.03, 2.0, DUST.real, DUST.imag]  # median radius, aspect ratio, Re m, Im m

    def oracle(p):
        d = np.zeros(1, dtype=O.DIST_DTYPE)
        d["kind"] = 1
        d["p"][0, :2] = p[0], 1.4
        return O.ensemble_adaptive_spheroid(d, WL, p[1], np.array([complex(p[2], p[3])]), MU, 6,
                                            rtol=1e-9, max_panels=50_000)

    got = _run(LOGN, 2.0, DUST, [0, 4, 2, 3])
    v = got["values"][:, 0]
    for c, value in enumerate(base):
        h = 1e-4 * abs(value)
        plus, minus = list(base), list(base)
        plus[c] += h
        minus[c] -= h
        op, om = oracle(plus), oracle(minus)
        for j in range(11):
            fd = (op["values"][j, 0] - om["values"][j, 0]) / (2 * h)
            scale = max(abs(fd), abs(v[j]) / abs(value), 1e-300)
            assert abs(got["d"][c][j, 0] - fd) <= 1e-5 * scale, (c, j, got["d"][c][j, 0], fd)
        fd = (op["greek"][0, 0] - om["greek"][0, 0]) / (2 * h)
        assert np.all(np.abs(got["greek_d"][c][0, 0] - fd)
                      <= 1e-5 * np.maximum(np.abs(fd), 1e-3)), (c, "alpha1")
        fd = (op["phase"][:, 0] - om["phase"][:, 0]) / (2 * h)
        scale = np.maximum(np.abs(fd), got["phase"][0, 0][None, :] / abs(value))
        assert np.all(np.abs(got["phase_d"][c][:, 0] - fd) <= 1e-5 * scale), (c, "phase")
