"""The oracle's refractive-index models against the reference package's own (fixture
tests/golden/refractive.json, made by tests/golden/make_fixtures.py from
python/scatrs/refractive.py): m and dm/dtheta to rounding."""

import json
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.join(os.path.dirname(__file__), "golden")


def records():
    with open(os.path.join(HERE, "refractive.json")) as f:
        return json.load(f)


def spec_of(rec):
    """A fixture's model spec in the form of oracle.refractive_index / _native models."""
    s = rec["spec"]
    kind = s[0]
    if kind == "constant":
        return (kind, complex(*s[1]))
    if kind.startswith("table"):
        return (kind, s[1], [complex(a, b) for a, b in s[2]])
    return tuple([kind] + s[1:])


@pytest.mark.parametrize("k", range(5))
def test_oracle_models_match_the_reference(k):
    rec = records()[k]
    m, dm = O.refractive_index(spec_of(rec), rec["wavelength"])
    want_m = np.array(rec["m"]).view(np.complex128).reshape(-1)
    want_dm = np.array(rec["dm"], dtype=np.float64).reshape(
        len(rec["parameters"]), 2 * len(rec["wavelength"])).view(np.complex128)
    np.testing.assert_allclose(m, want_m, rtol=4e-16, atol=0)
    assert dm.shape == want_dm.shape
    np.testing.assert_allclose(dm, want_dm, rtol=4e-16, atol=0)


def test_oracle_models_refuse_what_the_reference_refuses():
    rec = records()[1]
    with pytest.raises(ValueError):
        O.refractive_index(spec_of(rec), [0.2])
    with pytest.raises(ValueError):
        O.refractive_index(("sellmeier", [1.0], [0.25], 0.0), [0.5])  # at the pole
