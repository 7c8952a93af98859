"""greek='all' (GreekOrder::All) on the GPU: every order up to 2 N_max at each wavelength, the
arrays padded with zeros to the longest, against the oracle (same widths, same zeros, values and
error estimates as the adaptive path's tolerances), alone, batched, in a mixture with
derivatives, and through the reference-facing call (spheroids, and mixtures of different
particles, too)."""

import numpy as np
import pytest

from oracle import oracle as O
from scatrs_b200 import _native, _scatrs
from scatrs_b200.errors import InvalidInputError
from test_gpu_adaptive import MU, _compare, _dists, _odist

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("batch", [False, True])
def test_all_orders_match_the_oracle(gpu, batch):
    d = _dists((1, 0.3, 1.4), (2, 0.5, 0.12))
    wl = np.array([0.4, 0.9, 1.6])
    m = np.array([1.45 + 0.01j, 1.44 + 1e-3j, 1.43 + 1e-5j])
    got = gpu.ensemble_adaptive(d, wl, m, MU, _native.GREEK_ALL, batch=batch)
    ref = O.ensemble_adaptive(_odist(d), wl, m, mu=MU, greek_order="all", batch=batch)
    assert got["greek"].shape == ref["greek"].shape
    assert np.array_equal(got["greek"] == 0.0, ref["greek"] == 0.0)
    _compare(got, ref)


def test_a_mixture_with_derivatives(gpu):
    wl = np.array([0.45, 1.2])
    comps = [(_dists((1, 0.1, 1.5)), None, 2.0, np.array([1.45 + 0j, 1.44 + 1e-5j])),
             (_dists((1, 0.8, 1.3)), None, 0.5, np.array([1.53 + 0.01j, 1.5 + 0.02j]))]
    params = [(0, -1, 0, 1), (1, -1, 1, 0), (0, -1, 3, 0)]
    got = gpu.ensemble_mixture_d(comps, wl, np.array(params, dtype=_native.PARAM_DTYPE), MU,
                                 _native.GREEK_ALL)
    ref = O.ensemble_mixture_d([(_odist(d), mw, w, m) for d, mw, w, m in comps], wl,
                               O.params(*params), mu=MU, greek_order="all")
    assert got["greek_d"].shape == ref["greek_d"].shape
    _compare(got, ref)
    size = np.abs(ref["greek_d"]).max(axis=-1, keepdims=True) + 1e-300
    assert np.all(np.abs(got["greek_d"] - ref["greek_d"]) <= 1e-9 * size)


def test_the_reference_call(gpu):
    wl = np.array([0.5, 2.0])
    m = np.array([1.5 + 0.01j, 1.45 + 0.002j])
    items = [(("lognormal", 0.2, 1.5), ("sphere", m), 1.0)]
    raw = _scatrs.ensemble_compute(items, wl, False, None, True, MU, True, [], 1e-6, 4096, False,
                                   False)
    ref = gpu.ensemble_adaptive(_dists((1, 0.2, 1.5)), wl, m, MU, _native.GREEK_ALL)
    assert np.array_equal(raw["greek"], ref["greek"])
    assert raw["greek"].shape[-1] > 1 and np.all(raw["greek"][0, :, 0] == 1.0)
    spheroid = [(("lognormal", 0.05, 1.3), ("spheroid", 1.5, m), 1.0)]
    sph = _scatrs.ensemble_compute(spheroid, wl, False, None, True, None, True, [], 1e-4, 4096,
                                   False, False)
    assert sph["greek"].shape[-1] > 1 and np.all(sph["greek"][0, :, 0] == 1.0)
    mixed = spheroid + [(("lognormal", 0.2, 1.5), ("sphere", m), 1.0)]
    mix = _scatrs.ensemble_compute(mixed, wl, True, None, True, None, True, [], 1e-4, 4096,
                                   False, False)
    ref = _native.ensemble_mixture([(_dists((1, 0.05, 1.3)), None, 1.0, ("spheroid", 1.5, m)),
                                    (_dists((1, 0.2, 1.5)), None, 1.0, m)], wl, None,
                                   _native.GREEK_ALL, rtol=1e-4)
    assert np.array_equal(mix["greek"], ref["greek"]) and np.all(mix["greek"][0, :, 0] == 1.0)
