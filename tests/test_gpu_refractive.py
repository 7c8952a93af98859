"""Refractive-index models evaluated on the device (scatrs_refractive_index_device) against the
reference package's own models (tests/golden/refractive.json, from
python/scatrs/refractive.py): m and dm/dtheta within 1e-15 relative (the device's pow, log and
exp may differ from the host's in the last bit), and the reference's refusals."""

import numpy as np
import pytest

from scatrs_b200 import _native
from scatrs_b200.errors import InvalidInputError
from test_oracle_refractive import records, spec_of

pytestmark = pytest.mark.gpu


def _device(specs, lam, p_max=8):
    import torch

    dev = torch.device("cuda", 0)
    wl = torch.tensor(lam, dtype=torch.float64, device=dev)
    m = torch.zeros(len(specs), len(lam), 2, dtype=torch.float64, device=dev)
    dm = torch.zeros(len(specs), p_max, len(lam), 2, dtype=torch.float64, device=dev)
    _native.refractive_index_device(specs, wl.data_ptr(), len(lam), m.data_ptr(), dm.data_ptr(),
                                    p_max)
    return (m.cpu().numpy().view(np.complex128)[..., 0],
            dm.cpu().numpy().view(np.complex128)[..., 0])


def test_models_match_the_reference(gpu):
    recs = records()
    lam = recs[0]["wavelength"]
    assert all(r["wavelength"] == lam for r in recs)
    m, dm = _device([spec_of(r) for r in recs], lam)
    for k, rec in enumerate(recs):
        want = np.array(rec["m"]).view(np.complex128).reshape(-1)
        np.testing.assert_allclose(m[k], want, rtol=1e-15, atol=0, err_msg=rec["spec"][0])
        P = len(rec["parameters"])
        assert _native.refractive_parameter_count(spec_of(rec)) == P
        if P:
            want_dm = np.array(rec["dm"], dtype=np.float64).reshape(P, 2 * len(lam)).view(
                np.complex128)
            np.testing.assert_allclose(dm[k, :P], want_dm, rtol=1e-15, atol=1e-300,
                                       err_msg=rec["spec"][0])
        assert np.all(dm[k, P:] == 0)


def test_refusals(gpu):
    table = spec_of(records()[1])
    with pytest.raises(InvalidInputError, match="outside the Table's range"):
        _device([("constant", 1.5), table], [0.5, 3.0])
    with pytest.raises(InvalidInputError, match="n\\^2"):
        _device([("sellmeier", [1.0], [0.25], 0.0)], [0.4, 0.5])
    with pytest.raises(InvalidInputError, match="Im m"):
        _device([("cauchy", 1.5, 0.0, 0.0, -1.0)], [0.5])
    with pytest.raises(InvalidInputError, match="increasing"):
        _device([("table", [0.5, 0.4], [1.5, 1.5])], [0.45])
