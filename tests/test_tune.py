"""The autotuner's selection rules and error measure (no GPU)."""

import numpy as np

from scatrs_b200 import tune


def test_choose_keeps_only_identical_settings():
    ms = {(2, 1): 3.0, (4, 1): 5.0, (8, 1): 1.0}
    identical = {(2, 1): True, (4, 1): True, (8, 1): False}  # (8, 1) changed a result
    assert tune.choose(ms, identical, (4, 1)) == (2, 1)
    assert tune.choose({(4, 1): 5.0}, {}, (4, 1)) == (4, 1)


def test_choose_threshold_respects_tolerance():
    ms = {0: 10.0, 16: 6.0, 32: 7.0, 64: 8.0}
    errors = {0: 0.0, 16: 2e-10, 32: 5e-11, 64: 1e-12}
    assert tune.choose_threshold(ms, errors, 1e-10) == 32
    assert tune.choose_threshold(ms, errors, 1e-9) == 16
    assert tune.choose_threshold({0: 10.0, 16: 6.0}, {16: np.nan}, 1e-10) == 0


def test_output_errors_measures():
    n_units, n_mu, order = 2, 3, 2
    rv = np.array([1.0, 2.0, 4.0])
    rp = np.ones(6 * n_units * n_mu)
    rg = np.ones(6 * n_units * (order + 1))
    ref = (rv, rp, rg)
    gp = rp.copy()
    gp[5] += 1e-9  # F11 of unit 0 is 1: relative to it
    gg = rg.copy()
    gg[-1] += 3e-9  # relative to alpha_1 at order 0 of unit 1
    assert tune.output_errors(ref, (rv * (1 + 1e-12), rp, rg), n_units, n_mu, order) < 2e-12
    assert abs(tune.output_errors(ref, (rv, gp, rg), n_units, n_mu, order) - 1e-9) < 1e-15
    assert abs(tune.output_errors(ref, (rv, rp, gg), n_units, n_mu, order) - 3e-9) < 1e-15


def test_sample_wavelengths_spans_the_range():
    idx = tune.sample_wavelengths(1024, 64)
    assert idx[0] == 0 and idx[-1] == 1023 and 60 <= idx.size <= 64
    assert np.all(np.diff(idx) > 0)
    assert np.array_equal(tune.sample_wavelengths(10, 64), np.arange(10))


def test_tuning_settings_are_validated_and_restored():
    """scatrs_set_tuning through the C ABI (no GPU needed): accepted ranges, 0 for the
    defaults, refusals with the library's messages."""
    import pytest

    from scatrs_b200 import _native
    from scatrs_b200.errors import InvalidInputError

    before = _native.get_tuning()
    try:
        _native.set_tuning(8, 1 << 20)
        assert _native.get_tuning() == {"split": 8, "arena_rows": 1 << 20}
        _native.set_tuning(0, 0)
        assert _native.get_tuning() == {"split": 4, "arena_rows": 1 << 22}
        with pytest.raises(InvalidInputError, match="split"):
            _native.set_tuning(65, 0)
        with pytest.raises(InvalidInputError, match="arena_rows"):
            _native.set_tuning(4, 1 << 30)
        assert _native.get_tuning() == {"split": 4, "arena_rows": 1 << 22}
    finally:
        _native.set_tuning(before["split"], before["arena_rows"])
