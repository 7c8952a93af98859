"""The adaptive ensemble on the GPU (scatrs_ensemble_adaptive) against the oracle's restatement
of the reference's adaptive engine (itself checked against the reference's ensemble
identities): the same panels (pass-1 decisions on the same per-node quantities), values within
1e-12 (scalars relative; phase matrix relative to max F11; Greek relative to alpha1_0), error
estimates within 1e-9 of their own size or 1e-13 of the value (they are sums of
|Kronrod - Gauss| differences, which cancel), converged flags and panel counts equal."""

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

MU = np.array([1.0, 0.7, 0.0, -0.4, -1.0])


def _odist(d):
    """The oracle's records of d (tables are shared: d must outlive the oracle call)."""
    o = np.zeros(d.size, dtype=O.DIST_DTYPE)
    o["kind"], o["p"] = d["kind"], d["param"]
    o["r_lo"], o["r_hi"] = d["r_lo"], d["r_hi"]
    o["table"], o["table_len"] = d["table"], d["table_len"]
    return o


def _dists(*specs):
    from scatrs_b200._native import DIST_DTYPE

    d = np.zeros(len(specs), dtype=DIST_DTYPE)
    for k, (kind, *p) in enumerate(specs):
        d["kind"][k] = kind
        d["param"][k, :len(p)] = p
    return d


def _compare(got, ref, tol=1e-12):
    assert np.array_equal(got["panels"], ref["panels"])
    assert np.array_equal(got["converged"], ref["converged"])
    v, rv = got["values"], ref["values"]
    scale = np.maximum(np.abs(rv), 1e-300)
    scale[3] = np.maximum(scale[3], np.abs(rv[1]))
    err = np.abs(v - rv) / scale
    err[7] = np.abs(v[7] - rv[7])
    assert err.max() <= tol, (np.unravel_index(err.argmax(), err.shape), err.max())
    e, re = got["errors"], ref["errors"]
    assert np.all(np.abs(e - re) <= 1e-9 * np.abs(re) + 1e-13 * scale)
    for key in ("phase", "greek"):
        if key in ref:
            size = np.abs(ref[key][0]).max(axis=1, keepdims=True)[None]
            d = np.abs(got[key] - ref[key]) / size
            assert d.max() <= tol, (key, np.unravel_index(d.argmax(), d.shape), d.max())
            de = np.abs(got[key + "_err"] - ref[key + "_err"])
            assert np.all(de <= 1e-9 * np.abs(ref[key + "_err"]) + 1e-13 * size), key


@pytest.mark.parametrize("batch", [False, True])
def test_matches_the_oracle(gpu, batch):
    d = _dists((1, 0.08, 1.6), (2, 0.5, 0.15), (3, 2.0, 15.0, 0.5), (4, 3.0, 0.02, 1.0),
               (5, 0.3))
    wl = np.array([0.35, 0.55, 1.0])
    m = np.array([1.43 + 1e-8j, 1.5 + 0.01j, 1.33 + 0.0j])
    got = gpu.ensemble_adaptive(d, wl, m, MU, 24, batch=batch)
    ref = O.ensemble_adaptive(_odist(d), wl, m, mu=MU, greek_order=24, batch=batch)
    _compare(got, ref)


def test_tight_tolerance_and_unnormalized(gpu):
    d = _dists((1, 0.3, 1.5), (1, 1.2, 1.3))
    wl = np.array([0.5, 0.8])
    m = np.array([1.33 + 1e-6j, 1.45 + 1e-3j])
    got = gpu.ensemble_adaptive(d, wl, m, MU, 16, normalized=False, rtol=1e-9,
                                refine_backscatter=True)
    ref = O.ensemble_adaptive(_odist(d), wl, m, mu=MU, greek_order=16, normalized=False,
                              rtol=1e-9, refine_backscatter=True)
    _compare(got, ref)


def test_errors_name_the_node(gpu):
    from scatrs_b200.errors import InvalidInputError, OutsideValidatedDomainError

    d = _dists((1, 0.1, 1.5))
    with pytest.raises(OutsideValidatedDomainError, match="at wavelength"):
        gpu.ensemble_adaptive(d, [0.5], 1.5 + 20j)
    with pytest.raises(InvalidInputError, match="rtol"):
        gpu.ensemble_adaptive(d, [0.5], 1.5, rtol=0.5)
    with pytest.raises(InvalidInputError, match="distribution 0"):
        gpu.ensemble_adaptive(_dists((1, -0.1, 1.5)), [0.5], 1.5)


def test_mixture_and_multimodal_match_the_oracle(gpu):
    wl = np.array([0.45, 0.8])
    comps = [(_dists((1, 0.1, 1.5)), None, 2.0, np.array([1.45 + 0j, 1.44 + 1e-5j])),
             (_dists((1, 1.0, 1.3), (2, 0.4, 0.1)), [3.0, 1.0], 0.5,
              np.array([1.53 + 0.01j, 1.50 + 0.02j])),
             (_dists((5, 0.35)), None, 0.25, np.array([1.6 + 0.1j, 1.6 + 0.1j]))]
    got = gpu.ensemble_mixture(comps, wl, MU, 14)
    ref = O.ensemble_mixture([(_odist(d), mw, w, m) for d, mw, w, m in comps], wl, mu=MU,
                             greek_order=14)
    _compare(got, ref)
