"""The reference's edge-case checks of the adaptive engine (scatrs/tests/ensemble.rs) on the GPU
path, against the oracle where it runs them too: backscattering refinement is optional and
costs panels (649-663); narrow distributions are the single sphere and broad or steep ones stay
finite (839-880); number tails need no Mie solutions and every gamma parameter converges
(935-948); invalid inputs are rejected (881-934); and the results do not depend on how the work
is laid out (682-715 for the threads there): the same call twice, and a distribution alone or
among others, give the same bits."""

import numpy as np
import pytest

from oracle import oracle as O
from scatrs_b200 import _native
from scatrs_b200.errors import InvalidInputError
from test_gpu_adaptive import _compare, _dists, _odist

pytestmark = pytest.mark.gpu


def test_backscattering_refinement_is_optional(gpu):
    d = _dists((1, 1.0, 2.0))
    m = np.array([1.33 + 1e-4j])
    plain = gpu.ensemble_adaptive(d, [1.0], m)
    refined = gpu.ensemble_adaptive(d, [1.0], m, refine_backscatter=True)
    assert plain["converged"][0] and refined["panels"][0] > plain["panels"][0]
    assert abs(refined["values"][0, 0] / plain["values"][0, 0] - 1) < 2e-6
    for got, rb in ((plain, False), (refined, True)):
        ref = O.ensemble_adaptive(_odist(d), [1.0], m, refine_backscatter=rb)
        _compare(got, ref)


def test_narrow_and_extreme_distributions(gpu):
    m = np.array([1.45 + 0.001j])
    mono = gpu.ensemble_adaptive(_dists((5, 0.3)), [0.5], m, None, 4)
    for spec in ((1, 0.3, 1.000001), (2, 0.3, 1e-9)):
        d = _dists(spec)
        r = gpu.ensemble_adaptive(d, [0.5], m, None, 4)
        assert r["converged"][0] and np.all(np.isfinite(r["values"]))
        assert np.all(np.isfinite(r["greek"]))
        assert abs(r["values"][0, 0] / mono["values"][0, 0] - 1) < 1e-4, spec
        _compare(r, O.ensemble_adaptive(_odist(d), [0.5], m, greek_order=4))
    for spec in ((2, 0.3, 0.45), (4, -200.0, 0.01, 1.0)):
        r = gpu.ensemble_adaptive(_dists(spec), [0.5], m, None, 4, allow_unvalidated=True)
        assert np.all(np.isfinite(r["values"])) and np.all(np.isfinite(r["greek"])), spec


def test_number_tails_need_no_mie_solutions(gpu):
    m = np.array([1.45 + 0.01j])
    d = _dists((2, 0.5, 0.3))
    assert gpu.ensemble_adaptive(d, [10.0], m)["converged"][0]
    params = np.array([(0, -1, 0, 0), (0, -1, 0, 1)], dtype=_native.PARAM_DTYPE)
    r = gpu.ensemble_mixture_d([(d, None, 1.0, m)], [0.55], params)
    assert r["converged"][0]


def test_invalid_inputs_are_rejected(gpu):
    d = _dists((1, 0.3, 1.5))
    with pytest.raises(InvalidInputError, match="does m = 1"):
        gpu.ensemble_adaptive(d, [0.5], np.array([1.0 + 0j]))
    with pytest.raises(InvalidInputError):
        gpu.ensemble_adaptive(d, [1e-7], np.array([1.45 + 0.001j]), allow_unvalidated=True)
    huge = [(d, None, np.finfo(float).max, np.array([1.45 + 0j])),
            (d, None, np.finfo(float).max, np.array([1.45 + 0j]))]
    with pytest.raises(InvalidInputError, match="finite, positive sum"):
        gpu.ensemble_mixture(huge, [0.5])


def test_results_do_not_depend_on_the_layout(gpu):
    wl = np.array([0.4, 0.7, 1.3])
    m = np.array([1.45 + 0.01j, 1.44 + 1e-3j, 1.43 + 1e-5j])
    mu = np.array([1.0, 0.0, -1.0])
    d = _dists((1, 0.1, 1.6), (2, 0.6, 0.15), (1, 1.2, 1.3))
    a = gpu.ensemble_adaptive(d, wl, m, mu, 16)
    b = gpu.ensemble_adaptive(d, wl, m, mu, 16)
    alone = gpu.ensemble_adaptive(_dists((2, 0.6, 0.15)), wl, m, mu, 16)
    for key in ("values", "errors", "phase", "greek", "panels"):
        assert np.array_equal(a[key], b[key]), key
        # Units are distribution-major: the second distribution's are 3..5.
        mine = a[key][3:6] if key == "panels" else a[key][:, 3:6]
        assert np.array_equal(mine, alone[key]), key
