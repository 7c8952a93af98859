"""Spheroid T-matrices on the GPU (scatrs_spheroid_tmatrix, scatrs_spheroid_efficiencies: the
EBCM assembled in double-double, FP64 LU with double-double residual refinement) against the
oracle's quadruple-precision EBCM and the reference's Arb records.

Tolerances: T within 1e-13 of the mode's largest element of the quadruple-precision oracle
(the double-double elements and the refined solve leave rounding of that order after the
cancellation), and within 1e-13 of the records' largest element; the converged efficiencies at
rtol 1e-10 within 1e-9 of the records, for every record, including the elongated and flattened
shapes (eps = 0.2, 5, 1/3) where plain FP64 does not converge."""

import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from scatrs_b200 import _native
from scatrs_b200.errors import InvalidInputError

pytestmark = pytest.mark.gpu

RECORDS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "spheroid.json")))
FIXED = [r for r in RECORDS if ",N=" in r["case"]]
CONVERGED = [r for r in RECORDS if r["case"].endswith(",converged")]


@pytest.mark.parametrize("r", FIXED, ids=[r["case"] for r in FIXED])
def test_fixed_tmatrix_matches_the_oracle_and_the_records(gpu, r):
    from test_oracle_tmatrix import compare_fixed
    x, eps, s, N, nt = r["x"], r["eps"], complex(*r["m"]), r["n_terms"], r["n_theta"]
    for mm in sorted({0, 1, N // 2, N}):
        g = _native.spheroid_tmatrix(x, eps, s, mm, N, nt)
        o = O.tmatrix_mode(x, eps, s, mm, N, nt, quad=True)
        assert g.shape == o.shape
        assert np.abs(g - o).max() <= 1e-13 * np.abs(o).max(), mm
    assert compare_fixed(r, _native.spheroid_tmatrix) <= 1e-13


def test_a_sphere_gives_the_mie_coefficients(gpu):
    x, s = 3.0, 1.5 + 0.01j
    mie = O.mie(x, s, n_max=12)
    for mm in (0, 1, 5, 12):
        T = _native.spheroid_tmatrix(x, 1.0, s, mm, 12, 20)
        k = T.shape[0] // 2
        n0 = max(mm, 1)
        for i in range(k):
            assert abs(T[i, i] + mie["b"][n0 + i - 1]) <= 1e-14
            assert abs(T[k + i, k + i] + mie["a"][n0 + i - 1]) <= 1e-14
        assert np.abs(T - np.diag(np.diag(T))).max() <= 1e-14


def test_converged_efficiencies_in_one_batch(gpu):
    """Every converged record in one call, at rtol 1e-10: Q within 1e-9 of the records'."""
    x = np.array([r["x"] for r in CONVERGED])
    eps = np.array([r["eps"] for r in CONVERGED])
    m = np.array([complex(*r["m"]) for r in CONVERGED])
    q, n, nth = _native.spheroid_efficiencies(x, eps, m, 1e-10)
    for i, r in enumerate(CONVERGED):
        qe = r["q_ext"][0][0] + r["q_ext"][0][1]
        qs = r["q_sca"][0][0] + r["q_sca"][0][1]
        qa = r["q_abs"][0][0] + r["q_abs"][0][1]
        assert abs(q[i, 0] - qe) <= 1e-9 * qe, r["case"]
        assert abs(q[i, 1] - qs) <= 1e-9 * qs, r["case"]
        assert abs(q[i, 2] - qa) <= 1e-9 * qe, r["case"]
        assert nth[i] >= 2 * n[i]


def test_a_batch_equals_its_members(gpu):
    x = np.array([0.7, 2.5, 4.0])
    eps = np.array([1.7, 0.6, 2.2])
    m = np.array([1.5 + 0.01j, 1.33 + 0j, 1.53 + 0.1j])
    q, n, nth = _native.spheroid_efficiencies(x, eps, m, 1e-9)
    for i in range(3):
        qi, ni, nthi = _native.spheroid_efficiencies(x[i:i + 1], eps[i:i + 1], m[i:i + 1], 1e-9)
        assert (ni[0], nthi[0]) == (n[i], nth[i])
        assert np.array_equal(qi[0], q[i])


def test_invalid_inputs(gpu):
    with pytest.raises(InvalidInputError):
        _native.spheroid_tmatrix(1.0, 2.0, 1.5, 0, 0, 10)
    with pytest.raises(InvalidInputError):
        _native.spheroid_tmatrix(1.0, -2.0, 1.5, 0, 5, 10)
    with pytest.raises(InvalidInputError):
        _native.spheroid_efficiencies([1.0], [2.0], [1.5 - 0.1j], 1e-8)
