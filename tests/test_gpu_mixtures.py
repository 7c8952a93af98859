"""Mixtures of different particles on the GPU (scatrs_ensemble_mixture with layered and
spheroid components: each class on its own engine, the parts' averages mixed and assembled on
one layout) against the oracle's restatement of the reference's single-layout engine: the same
panels and flags; values, phase matrix and Greek coefficients within the tolerance of the
slower particle's own path (1e-11 with layered spheres; 1e-9 with spheroids, whose nodes the two
solve in different arithmetic), error estimates as those paths'. And the reference-facing call
routes mixtures and multimodal layered or spheroid components through this path."""

import numpy as np
import pytest

from oracle import oracle as O
from scatrs_b200 import _native, _scatrs
from test_gpu_adaptive import _dists, _odist

pytestmark = pytest.mark.gpu

MU = np.array([1.0, 0.4, -0.5, -1.0])
NONE = np.zeros(0, O.PARAM_DTYPE)


def _compare(got, ref, tol, etol):
    assert np.array_equal(got["panels"], ref["panels"])
    assert np.array_equal(got["converged"], ref["converged"])
    v, rv = got["values"], ref["values"]
    scale = np.abs(rv).copy()
    scale[2] = np.abs(rv[0])  # C_abs against C_ext
    scale[3] = np.maximum(scale[3], np.abs(rv[1]))
    scale[7] = np.maximum(scale[7], 1e-300)
    assert np.all(np.abs(v - rv) <= tol * scale), np.abs(v - rv) / scale
    e, re = got["errors"], ref["errors"]
    assert np.all(np.abs(e - re) <= etol * np.abs(re) + 1e-13 * scale)
    for key in ("phase", "greek"):
        size = np.abs(ref[key][0]).max(axis=1, keepdims=True)[None]
        assert np.all(np.abs(got[key] - ref[key]) <= tol * size), key


def _both(comps, wl, L, **kw):
    got = _native.ensemble_mixture(comps, wl, MU, L, **kw)
    ref = O.ensemble_mixture_d([(_odist(d), mw, w, m) for d, mw, w, m in comps], wl, NONE,
                               mu=MU, greek_order=L, **kw)
    return got, ref


def test_spheres_and_layered_spheres(gpu):
    wl = np.array([0.45, 0.8])
    core = np.array([1.95 + 0.79j, 1.9 + 0.7j])
    shell = np.array([1.43 + 0.01j, 1.42 + 0.01j])
    comps = [(_dists((1, 0.1, 1.5)), None, 2.0, np.array([1.45 + 0j, 1.44 + 1e-5j])),
             (_dists((1, 0.3, 1.4)), None, 0.5, ("layered", [0.5], np.stack([core, shell]))),
             (_dists((2, 0.2, 0.1), (1, 0.5, 1.3)), [1.0, 0.3], 0.7,
              ("layered", [0.4, 0.8], np.stack([core, shell, shell * 0 + 1.33])))]
    got, ref = _both(comps, wl, 10)
    _compare(got, ref, 1e-11, 1e-9)


@pytest.mark.parametrize("normalized", [True, False])
def test_spheres_and_spheroids(gpu, normalized):
    wl = np.array([1.0])
    dust = np.array([1.53 + 0.008j])
    comps = [(_dists((1, 0.05, 1.5)), None, 2.0, np.array([1.45 + 0j])),
             (_dists((1, 0.08, 1.4)), None, 0.5, ("spheroid", 1.5, dust)),
             (_dists((1, 0.06, 1.3)), None, 0.4, ("spheroid", 0.7, dust))]
    got, ref = _both(comps, wl, 6, normalized=normalized, rtol=1e-4)
    _compare(got, ref, 1e-9, 1e-6)
    assert np.all(got["values"][7] > 0.0)


def _orders(greek):
    """The order of each wavelength's coefficients: the last nonzero alpha1."""
    return np.array([np.flatnonzero(g)[-1] for g in greek[0]])


def test_all_orders_with_layered_spheres(gpu):
    """greek='all': each wavelength's order is 2 N_max over every part (engine.rs:2016-2036),
    the layered class's pass 1 included."""
    wl = np.array([0.45, 0.8])
    core = np.array([1.95 + 0.79j, 1.9 + 0.7j])
    shell = np.array([1.43 + 0.01j, 1.42 + 0.01j])
    comps = [(_dists((1, 0.1, 1.5)), None, 2.0, np.array([1.45 + 0j, 1.44 + 1e-5j])),
             (_dists((1, 0.12, 1.4)), None, 0.5, ("layered", [0.5], np.stack([core, shell])))]
    got = _native.ensemble_mixture(comps, wl, MU, _native.GREEK_ALL)
    ref = O.ensemble_mixture_d([(_odist(d), mw, w, m) for d, mw, w, m in comps], wl, NONE,
                               mu=MU, greek_order="all")
    assert got["greek"].shape == ref["greek"].shape
    assert np.array_equal(_orders(got["greek"]), _orders(ref["greek"]))
    _compare(got, ref, 1e-11, 1e-9)


def test_all_orders_with_spheroids(gpu):
    """The spheroids' N enters the order; the spheres' bands project to min(2 N_max, 2 N_band)
    and the spheroids' direct segment to 2 N of their own."""
    wl = np.array([0.8, 1.0])
    dust = np.array([1.53 + 0.008j, 1.52 + 0.01j])
    comps = [(_dists((1, 0.03, 1.5)), None, 2.0, np.array([1.45 + 0j, 1.44 + 0j])),
             (_dists((1, 0.08, 1.4)), None, 0.5, ("spheroid", 1.5, dust))]
    got = _native.ensemble_mixture(comps, wl, MU, _native.GREEK_ALL, rtol=1e-4)
    ref = O.ensemble_mixture_d([(_odist(d), mw, w, m) for d, mw, w, m in comps], wl, NONE,
                               mu=MU, greek_order="all", rtol=1e-4)
    assert got["greek"].shape == ref["greek"].shape
    assert np.array_equal(_orders(got["greek"]), _orders(ref["greek"]))
    _compare(got, ref, 1e-9, 1e-6)


def test_the_reference_call(gpu):
    wl = np.array([0.6])
    m = np.array([1.5 + 0.02j])
    layered = ("layered", [0.6], np.array([[1.8 + 0.3j], [1.4 + 0.001j]]))
    items = [(("lognormal", 0.1, 1.5), ("sphere", m), 1.0),
             (("gamma", 0.2, 0.1), layered, 0.5)]
    raw = _scatrs.ensemble_compute(items, wl, True, 6, False, MU, True, [], 1e-6, 4096, False,
                                   False)
    ref = _native.ensemble_mixture([(_dists((1, 0.1, 1.5)), None, 1.0, m),
                                    (_dists((2, 0.2, 0.1)), None, 0.5, layered)], wl, MU, 6)
    assert np.array_equal(raw["values"], ref["values"])
    assert np.array_equal(raw["greek"], ref["greek"])
    bimodal = [(("multimodal", [(2.0, ("lognormal", 0.1, 1.5)), (1.0, ("lognormal", 0.4, 1.3))]),
                layered, 1.0)]
    one = _scatrs.ensemble_compute(bimodal, wl, False, 6, False, None, True, [], 1e-6, 4096,
                                   False, False)
    d = _native.dist_records(2)
    d[0]["kind"] = d[1]["kind"] = 1
    d[0]["param"][:2], d[1]["param"][:2] = (0.1, 1.5), (0.4, 1.3)
    ref = O.ensemble_mixture_d([(_odist(d), [2.0, 1.0], 1.0, layered)], wl, NONE, greek_order=6)
    assert np.allclose(one["values"], ref["values"], rtol=1e-11, atol=0)
