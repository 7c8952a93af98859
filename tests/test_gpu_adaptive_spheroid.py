"""The adaptive ensemble of randomly oriented spheroids on the GPU
(scatrs_ensemble_adaptive_spheroid: pass-1 nodes as spheroid batches with their orientation
average, pass 2 on the engine's direct path) against the oracle's adaptive engine with its
double-precision EBCM and Racah-based orientation average per node: the same panels and
convergence flags; values within 1e-9 and error estimates within 1e-6 of their size (the two
solve each node's T-matrix to rtol / 100 in different arithmetic, double-double here and
double there, so a node's N or n_theta may settle one step apart)."""

import numpy as np
import pytest

from oracle import oracle as O
from scatrs_b200 import _scatrs
from test_gpu_adaptive import _dists, _odist

pytestmark = pytest.mark.gpu

MU = np.array([-0.5, 0.5])


def _compare(got, ref):
    assert np.array_equal(got["panels"], ref["panels"])
    assert np.array_equal(got["converged"], ref["converged"])
    v, rv = got["values"], ref["values"]
    scale = np.abs(rv)
    scale[2] = np.abs(rv[0])  # C_abs against C_ext
    assert np.all(np.abs(v - rv) <= 1e-9 * scale), np.abs(v - rv) / scale
    e, re = got["errors"], ref["errors"]
    assert np.all(np.abs(e - re) <= 1e-6 * np.abs(re) + 1e-12 * scale)
    for key in ("phase", "greek"):
        size = np.abs(ref[key][0]).max(axis=1, keepdims=True)[None]
        assert np.all(np.abs(got[key] - ref[key]) <= 1e-9 * size), key


def test_matches_the_oracle(gpu):
    d = _dists((1, 0.1, 1.5), (5, 0.15))
    wl = np.array([0.5, 0.8])
    m = np.array([1.5 + 0.01j, 1.45 + 0.001j])
    got = gpu.ensemble_adaptive_spheroid(d, wl, 1.6, m, MU, 6, rtol=1e-4)
    ref = O.ensemble_adaptive_spheroid(_odist(d), wl, 1.6, m, MU, 6, rtol=1e-4)
    _compare(got, ref)
    assert np.all(got["values"][7] > 0)  # spheroids depolarize


def test_drop_in_spec(gpu):
    """('spheroid', eps, m) through the reference's ensemble_compute signature."""
    wl = np.array([0.6])
    raw = _scatrs.ensemble_compute([(("lognormal", 0.08, 1.5), ("spheroid", 0.7,
                                                                 np.array([1.5 + 0.02j])), 1.0)],
                                   wl, False, 4, False, None, True, [], 1e-3, 4096, False, False)
    ref = O.ensemble_adaptive_spheroid(_odist(_dists((1, 0.08, 1.5))), wl, 0.7,
                                       np.array([1.5 + 0.02j]), None, 4, rtol=1e-3)
    assert np.allclose(raw["values"], ref["values"], rtol=1e-9, atol=0)
    assert raw["greek"].shape == (6, 1, 5)


def test_each_distribution_has_its_own_direct_order(gpu):
    """Every distribution of a call is a call of its own (engine.rs:1987-2030): its direct order,
    to which the phase matrix's expansion and its error bounds run, follows its own N_max over
    its final panels."""
    d = _dists((1, 0.03, 1.3), (1, 0.2, 1.4))
    wl = np.array([0.6])
    m = np.array([1.5 + 0.01j])
    got = gpu.ensemble_adaptive_spheroid(d, wl, 1.4, m, MU, 4, rtol=1e-4)
    ref = O.ensemble_adaptive_spheroid(_odist(d), wl, 1.4, m, MU, 4, rtol=1e-4)
    _compare(got, ref)


def test_all_orders(gpu):
    """greek='all': every order to 2 N_max of each distribution, padded to the longest."""
    from scatrs_b200 import _native

    d = _dists((1, 0.05, 1.4), (1, 0.15, 1.3))
    wl = np.array([0.5, 0.9])
    m = np.array([1.5 + 0.01j, 1.45 + 0.001j])
    got = gpu.ensemble_adaptive_spheroid(d, wl, 0.8, m, MU, _native.GREEK_ALL, rtol=1e-4)
    ref = O.ensemble_adaptive_spheroid(_odist(d), wl, 0.8, m, MU, "all", rtol=1e-4)
    assert got["greek"].shape == ref["greek"].shape
    _compare(got, ref)
