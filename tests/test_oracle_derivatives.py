"""The oracle's forward-mode derivatives of the fixed-grid ensemble (the reference's
`derivatives=` outputs: scatrs/src/ensemble/engine.rs:1047-1200 per node, 1782-1836 for the
averages, lin.rs for the ratios) against central differences of its own values, the node grid
held fixed, for every distribution kind: the distribution's parameters, then Re m and Im m."""

import numpy as np
import pytest

from oracle import oracle as O

MU = np.array([1.0, 0.6, 0.0, -0.35, -1.0])
WL = np.array([0.45, 0.9])
M = np.array([[1.45 + 0.02j, 1.38 + 1e-4j]])

CASES = {
    "lognormal": (1, [0.15, 1.7, 0.0], 0.15 * 1.7 ** -4, 0.15 * 1.7 ** 4),
    "gamma": (2, [0.3, 0.12, 0.0], 0.01, 2.0),
    "modified_gamma": (3, [2.0, 8.0, 1.0, ], 0.01, 2.5),
    "power_law": (4, [3.5, 0.05, 1.5], 0.05, 1.5),
}


def _dist(kind, p, lo, hi):
    d = np.zeros(1, dtype=O.DIST_DTYPE)
    d["kind"] = kind
    d["p"][0, :len(p)] = p
    d["r_lo"], d["r_hi"] = lo, hi
    return d


def _values(d, m, normalized):
    return O.ensemble_fixed(d, WL, m, 48, MU, 10, normalized=normalized)


@pytest.mark.parametrize("normalized", [True, False])
@pytest.mark.parametrize("name", list(CASES))
def test_derivatives_match_central_differences(name, normalized):
    kind, p, lo, hi = CASES[name]
    d = _dist(kind, p, lo, hi)
    got = O.ensemble_fixed_d(d, WL, M, 48, MU, 10, normalized=normalized)
    plain = _values(d, M, normalized)
    for k in ("values", "phase", "greek"):
        assert np.array_equal(got[k], plain[k])
    n_theta = got["d_values"].shape[0] - 2
    assert n_theta == {1: 2, 2: 2, 3: 3, 4: 1}[kind]
    h = 1e-6
    for q in range(n_theta + 2):
        dp, dm, mp, mm = d.copy(), d.copy(), M.copy(), M.copy()
        if q < n_theta:
            s = h * max(abs(p[q]), 1e-3)
            dp["p"][0, q] += s
            dm["p"][0, q] -= s
        elif q == n_theta:
            s = h
            mp, mm = M + s, M - s
        else:
            s = h * M.imag.min()
            mp, mm = M + 1j * s, M - 1j * s
        a, b = _values(dp, mp, normalized), _values(dm, mm, normalized)
        for k in ("values", "phase", "greek"):
            fd = (a[k] - b[k]) / (2 * s)
            an = got["d_" + k][q]
            if k == "values":
                size = np.abs(an) + np.abs(plain["values"]) * 1e-3
                size[7] = 1.0  # depolarization: 0 for spheres
            else:
                size = np.abs(an).max(axis=-1, keepdims=True) + 1e-300
            err = np.abs(fd - an) / size
            assert err.max() <= 2e-5, (name, q, k, np.unravel_index(err.argmax(), err.shape))


def test_mixed_kinds_rejected():
    d = np.concatenate([_dist(*CASES["lognormal"]), _dist(*CASES["modified_gamma"])])
    with pytest.raises(O.OracleError):
        O.ensemble_fixed_d(d, WL, np.repeat(M, 2, axis=0), 16, MU, 4)
