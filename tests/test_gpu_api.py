"""The reference-facing mirror (scatrs_b200._scatrs.ensemble_compute_fixed): the dict of
scatrs-py/src/ensemble.rs:289-294, 432-450 with its keys, dtypes and shapes, derivative
selection by ensemble_parameters index, and the layered particle spec."""

import numpy as np
import pytest

from scatrs_b200 import _native, _scatrs

pytestmark = pytest.mark.gpu


def test_dict_layout_and_derivative_selection(gpu):
    specs = [("lognormal", 0.1, 1.6), ("lognormal", 0.3, 1.4)]
    wl = np.array([0.4, 0.6, 0.9])
    m = np.array([1.45 + 0.01j, 1.44 + 0.005j, 1.43 + 0.001j])
    mu = np.array([1.0, 0.2, -0.5])
    raw = _scatrs.ensemble_compute_fixed(specs, ("sphere", m), wl, 10, False, mu, True,
                                         n_nodes=64, spread=4.0, derivatives=[3, 0])
    n = 6
    assert raw["values"].shape == (11, n) and raw["errors"].shape == (11, n)
    assert raw["d"].shape == (2, 11, n) and raw["d_errors"].shape == (2, 11, n)
    assert raw["greek"].shape == (6, n, 11) and raw["greek_d"].shape == (2, 6, n, 11)
    assert raw["phase"].shape == (6, n, 3) and raw["phase_d"].shape == (2, 6, n, 3)
    assert raw["converged"].dtype == bool and raw["panels"].dtype == np.uint64
    full = _native.ensemble_fixed_d(_scatrs._dist_array(specs, 4.0), wl,
                                    np.broadcast_to(m, (2, 3)), mu, 64, 10)
    assert np.array_equal(raw["d"], full[3][[3, 0]])
    assert np.array_equal(raw["greek_d"], full[5][[3, 0]])
    plain = _scatrs.ensemble_compute_fixed(specs, ("sphere", m), wl, 10, False, mu, True,
                                           n_nodes=64, spread=4.0)
    assert plain["d"].shape == (0, 11, n) and plain["greek_d"].shape == (0, 6, n, 11)


def test_layered_spec(gpu):
    specs = [("lognormal", 0.2, 1.5)]
    wl = np.array([0.5, 0.8])
    ml = np.array([[1.6 + 0.1j, 1.6 + 0.1j], [1.4 + 0.01j, 1.4 + 0.01j], [1.33 + 0j, 1.33 + 0j]])
    raw = _scatrs.ensemble_compute_fixed(specs, ("layered", [0.5, 0.9], ml), wl, 8, False, None,
                                         True, n_nodes=64, spread=4.0)
    v, _, g = _native.ensemble_fixed_layered(_scatrs._dist_array(specs, 4.0), wl, [[0.5, 0.9]],
                                             ml[None], None, 64, 8)
    assert np.array_equal(raw["values"], v) and np.array_equal(raw["greek"], g)


def test_adaptive_calls_mirror_the_reference(gpu):
    """ensemble_compute / ensemble_compute_batch: the reference dict from the adaptive engine,
    equal to the raw binding's arrays."""
    wl = np.array([0.4, 0.7])
    m = np.array([1.45 + 0.01j, 1.40 + 1e-4j])
    mu = np.array([1.0, -0.3])
    items = [(("gamma", 0.4, 0.1), ("sphere", m), 1.0)]
    raw = _scatrs.ensemble_compute(items, wl, False, 12, False, mu, True, [], 1e-6, 4096, False,
                                   False)
    ref = _native.ensemble_adaptive(_scatrs._adaptive_dists([items[0][0]]), wl, m, mu, 12)
    assert np.array_equal(raw["values"], ref["values"])
    assert np.array_equal(raw["greek_errors"], ref["greek_err"])
    assert raw["d"].shape == (0, 11, 2) and raw["panels"].dtype == np.uint64
    specs = [("lognormal", 0.1, 1.5), ("monodisperse", 0.3)]
    b = _scatrs.ensemble_compute_batch(specs, ("sphere", m), wl, None, False, mu, True, 1e-6,
                                       4096, False, False)
    assert b["values"].shape == (11, 4) and "greek" not in b and b["phase"].shape == (6, 4, 2)
    assert np.all(b["panels"][2:] == 0) and np.all(b["converged"])


def test_mixture_call_mirrors_the_reference(gpu):
    wl = np.array([0.5])
    m1, m2 = np.array([1.45 + 0j]), np.array([1.53 + 0.01j])
    items = [(("multimodal", [(2.0, ("lognormal", 0.1, 1.5)), (0.5, ("lognormal", 1.0, 1.3))]),
              ("sphere", m1), 1.0)]
    bi = _scatrs.ensemble_compute(items, wl, False, 10, False, None, True, [], 1e-6, 4096, False,
                                  False)
    both = _scatrs.ensemble_compute([(("lognormal", 0.1, 1.5), ("sphere", m1), 2.0),
                                     (("lognormal", 1.0, 1.3), ("sphere", m1), 0.5)], wl, True,
                                    10, False, None, True, [], 1e-6, 4096, False, False)
    assert np.array_equal(bi["values"], both["values"])
    mix = _scatrs.ensemble_compute([(("lognormal", 0.1, 1.5), ("sphere", m1), 2.0),
                                    (("lognormal", 1.0, 1.3), ("sphere", m2), 0.5)], wl, True,
                                   10, False, None, True, [], 1e-6, 4096, False, False)
    assert mix["values"].shape == (11, 1) and mix["greek"].shape == (6, 1, 11)
