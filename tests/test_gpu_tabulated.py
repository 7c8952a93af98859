"""Tabulated size distributions on the GPU (n(r) linear between the table's points, 0 outside;
scatrs/src/ensemble/distribution.rs:55-62) against the oracle: the adaptive engine alone, in a
batch sharing panels with other kinds, as a multimodal mode and a mixture component, on layered
spheres; the fixed grid with and without the Re m / Im m derivatives; and the reference-facing
spec ("tabulated", radii, densities). Tolerances are those of the same paths for the
parametric kinds."""

import numpy as np
import pytest

from oracle import oracle as O
from scatrs_b200 import _native, _scatrs
from scatrs_b200.errors import InvalidInputError
from test_gpu_adaptive import MU, _compare, _odist
from test_gpu_derivatives import _compare as _compare_d
from test_gpu_ensemble import _compare as _compare_fixed

pytestmark = pytest.mark.gpu

REF_TABLE = ([0.05, 0.1, 0.4, 1.0], [0.0, 3.0, 1.0, 0.2])
SPIKE = ([0.1, 0.2, 0.2001, 0.2002, 0.5], [0.0, 0.0, 1.0, 0.0, 0.0])


def _records(*entries):
    """Distribution records: (radii, densities) tables or (kind, params...) tuples."""
    d = _native.dist_records(len(entries))
    for k, e in enumerate(entries):
        if isinstance(e[0], (list, np.ndarray)):
            _native.set_table(d, k, *e)
        else:
            d[k]["kind"] = e[0]
            d[k]["param"][: len(e) - 1] = e[1:]
    return d


@pytest.mark.parametrize("batch", [False, True])
def test_adaptive_matches_the_oracle(gpu, batch):
    d = _records(REF_TABLE, (1, 0.2, 1.5), SPIKE)
    wl = np.array([0.4, 0.7])
    m = np.array([2.0 + 0.5j, 1.45 + 1e-4j])
    got = gpu.ensemble_adaptive(d, wl, m, MU, 12, batch=batch)
    ref = O.ensemble_adaptive(_odist(d), wl, m, mu=MU, greek_order=12, batch=batch)
    _compare(got, ref)


def test_spike_with_one_panel(gpu):
    d = _records(SPIKE)
    got = gpu.ensemble_adaptive(d, [0.5], 1.5 + 0j, MU, 6, max_panels=1)
    ref = O.ensemble_adaptive(_odist(d), [0.5], 1.5 + 0j, mu=MU, greek_order=6, max_panels=1)
    _compare(got, ref)
    assert np.all(np.isfinite(got["values"])) and got["values"][0, 0] > 0.0


def test_mixture_with_a_table_matches_the_oracle(gpu):
    wl = np.array([0.45, 0.8])
    comps = [(_records(REF_TABLE, (1, 0.8, 1.3)), [2.0, 1.0], 1.0,
              np.array([1.5 + 0.01j, 1.48 + 0.005j])),
             (_records(SPIKE), None, 0.5, np.array([1.33 + 0j, 1.33 + 1e-6j]))]
    got = gpu.ensemble_mixture(comps, wl, MU, 10)
    ref = O.ensemble_mixture([(_odist(d), mw, w, m) for d, mw, w, m in comps], wl, mu=MU,
                             greek_order=10)
    _compare(got, ref)


def test_layered_on_a_table_matches_the_oracle(gpu):
    d = _records(REF_TABLE)
    wl = np.array([0.5, 0.9])
    fr = np.array([[0.6]])
    ml = np.array([[[1.95 + 0.79j, 1.9 + 0.7j], [1.43 + 1e-8j, 1.42 + 1e-8j]]])
    got = gpu.ensemble_adaptive_layered(d, wl, fr, ml, MU, 8)
    ref = O.ensemble_adaptive_layered(_odist(d), wl, fr, ml, MU, 8)
    _compare(got, ref, tol=1e-11)


def test_fixed_grid_matches_the_oracle(gpu):
    # (A fixed grid does not resolve SPIKE: its nodes miss the 2e-4 wide peak.)
    d = _records(REF_TABLE, ([0.1, 0.3, 0.6], [1.0, 2.0, 0.0]))
    wl = np.array([0.4, 0.7, 1.1])
    m = np.array([[2.0 + 0.5j, 1.9 + 0.4j, 1.8 + 0.3j], [1.33 + 0j, 1.33 + 1e-7j, 1.32 + 1e-6j]])
    got = gpu.ensemble_fixed(d, wl, m, MU, 80, 12)
    ref = O.ensemble_fixed(_odist(d), wl, m, 80, MU, 12)
    _compare_fixed(got, ref)
    got_d = gpu.ensemble_fixed_d(d, wl, m, MU, 80, 12)
    ref_d = O.ensemble_fixed_d(_odist(d), wl, m, 80, MU, 12)
    assert got_d[3].shape[0] == 2  # no distribution parameters: Re m, Im m
    _compare_d(got_d, ref_d)


def test_the_reference_spec(gpu):
    wl = np.array([0.4, 0.7])
    m = np.array([2.0 + 0.5j, 1.9 + 0.4j])
    spec = ("tabulated", REF_TABLE[0], REF_TABLE[1])
    raw = _scatrs.ensemble_compute([(spec, ("sphere", m), 1.0)], wl, False, 10, False, MU, True,
                                   [], 1e-6, 4096, False, False)
    ref = gpu.ensemble_adaptive(_records(REF_TABLE), wl, m, MU, 10)
    assert np.array_equal(raw["values"], ref["values"])
    assert np.array_equal(raw["greek"], ref["greek"])
    assert _scatrs.ensemble_parameters([(spec, ("sphere", m), 1.0)], False) == [
        "m_real", "m_imag"]
    with pytest.raises(InvalidInputError, match="at least 2 points"):
        _scatrs.ensemble_compute([(("tabulated", [0.1, 0.2], [1.0]), ("sphere", m), 1.0)], wl,
                                 False, None, False, None, True, [], 1e-6, 4096, False, False)
    with pytest.raises(InvalidInputError, match="must increase"):
        _scatrs.ensemble_compute([(("tabulated", [0.2, 0.1], [1.0, 1.0]), ("sphere", m), 1.0)],
                                 wl, False, None, False, None, True, [], 1e-6, 4096, False,
                                 False)
