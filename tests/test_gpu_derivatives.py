"""The derivatives of the fixed-grid ensemble through the C ABI (scatrs_ensemble_fixed_d)
against the oracle's forward-mode restatement (itself checked against central differences).

Tolerance: the GPU projects each block's raw sums and averages after the projection, the
oracle averages first (the projection is linear), and the sums run in other orders; the
derivatives agree to 1e-9 of the largest derivative of the same output and unit (or 1e-6 of
the value for a derivative that vanishes), the values to 1e-12 as in the plain path. A ratio
x/y (albedo, g, lidar ratio, effective radius) has the derivative (dx - (x/y) dy)/y, whose
rounding is relative to |v| (|dx/x| + |dy/y|), its scale here."""

import numpy as np
import pytest

from oracle import oracle as O
from scatrs_b200 import workloads as W

pytestmark = pytest.mark.gpu

MU = np.array([1.0, 0.6, 0.0, -0.35, -1.0, 0.35])


def _odists(d):
    o = np.zeros(d.size, dtype=O.DIST_DTYPE)
    o["kind"], o["p"], o["r_lo"], o["r_hi"] = d["kind"], d["param"], d["r_lo"], d["r_hi"]
    return o


def _dists(kind, params, lo, hi):
    from scatrs_b200._native import DIST_DTYPE

    d = np.zeros(len(params), dtype=DIST_DTYPE)
    d["kind"] = kind
    for k, p in enumerate(params):
        d["param"][k, :len(p)] = p
    d["r_lo"], d["r_hi"] = lo, hi
    return d


def _compare(got, ref, tol=1e-9):
    v, ph, g, dv, dph, dg = got
    assert np.allclose(v, ref["values"], rtol=1e-12, atol=0)
    pairs = [(dv, ref["d_values"], ref["values"])]
    if ph is not None:
        pairs.append((dph, ref["d_phase"], ref["phase"]))
    if g is not None:
        pairs.append((dg, ref["d_greek"], ref["greek"]))
    for a, b, val in pairs:
        if a.ndim == 3:  # scalars: per output and unit
            size = np.maximum(np.abs(b), 1e-6 * np.abs(val)[None])
            rel = np.abs(b) / np.maximum(np.abs(val)[None], 1e-300)  # |d ln v|
            for k, (x, y) in {4: (1, 0), 5: (1, 1), 6: (0, 3), 8: (10, 9)}.items():
                size[:, k] = np.maximum(size[:, k], np.abs(val[k]) * (rel[:, x] + rel[:, y]))
            size[:, 7] = 1.0
        else:
            # Normalized by c_sca (phase) or alpha1_0 (Greek): the same ratio rule.
            vmax = np.abs(val).max(axis=-1, keepdims=True)[None]
            rsca = (np.abs(ref["d_values"][:, 1]) / ref["values"][1][None])[:, None, :, None]
            size = np.maximum(np.abs(b).max(axis=-1, keepdims=True),
                              vmax * np.maximum(1e-6, rsca))
        err = np.abs(a - b) / np.maximum(size, 1e-300)
        assert err.max() <= tol, (np.unravel_index(err.argmax(), err.shape), err.max())


@pytest.mark.parametrize("normalized", [True, False])
def test_lognormal_matches_oracle(gpu, normalized):
    w = W.batched_spheres(seed=5, scale=0.03)  # 2 distributions x 31 wavelengths
    w.n_nodes = 96
    got = gpu.ensemble_fixed_d(w.dists, w.wavelengths, w.m, MU, w.n_nodes, 24,
                               normalized=normalized)
    ref = O.ensemble_fixed_d(_odists(w.dists), w.wavelengths, w.m, w.n_nodes, MU, 24,
                             normalized=normalized)
    _compare(got, ref)


@pytest.mark.parametrize("kind,params,lo,hi", [
    (2, [[0.3, 0.12], [0.8, 0.2]], 0.01, 3.0),
    (3, [[2.0, 8.0, 1.0], [1.0, 3.0, 0.5]], 0.01, 2.5),
    (4, [[3.5, 0.05, 1.5], [2.0, 0.05, 1.5]], 0.05, 1.5),
])
def test_other_kinds_match_oracle(gpu, kind, params, lo, hi):
    d = _dists(kind, params, lo, hi)
    wl = np.array([0.4, 0.7, 1.1])
    m = np.array([[1.5 + 0.01j, 1.45 + 1e-5j, 1.33 + 0.0j], [1.6 + 0.1j, 1.52 + 1e-3j,
                                                             1.4 + 1e-8j]])
    got = gpu.ensemble_fixed_d(d, wl, m, MU, 70, 16)
    ref = O.ensemble_fixed_d(_odists(d), wl, m, 70, MU, 16)
    _compare(got, ref)


def test_values_match_the_plain_path(gpu):
    w = W.small_spheres()
    got = gpu.ensemble_fixed_d(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, w.greek_order)
    plain = gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, w.greek_order)
    for a, b in zip(got[:3], plain):
        size = np.abs(b).max(axis=-1, keepdims=True)
        assert np.all(np.abs(a - b) <= 1e-12 * size)
    assert np.all(got[2][0, :, 0] == 1.0) and np.all(got[5][:, 0, :, 0] == 0.0)


def test_no_outputs_and_errors(gpu):
    from scatrs_b200.errors import InvalidInputError

    w = W.small_spheres()
    got = gpu.ensemble_fixed_d(w.dists, w.wavelengths, w.m, None, w.n_nodes, -1)
    assert got[1] is None and got[2] is None and got[4] is None and got[5] is None
    ref = O.ensemble_fixed_d(_odists(w.dists), w.wavelengths, w.m, w.n_nodes)
    assert np.allclose(got[0], ref["values"], rtol=1e-12, atol=0)
    mixed = np.concatenate([w.dists, _dists(3, [[2.0, 8.0, 1.0]], 0.01, 2.5)])
    with pytest.raises(InvalidInputError, match="one kind"):
        gpu.ensemble_fixed_d(mixed, w.wavelengths, np.repeat(w.m, 2, axis=0), None, 16, -1)
