"""Spheroid T-matrices on the GPU (scatrs_spheroid_tmatrix, scatrs_spheroid_efficiencies)
against the oracle's EBCM (the same FP64 formulation, summed and pivoted in another order:
T within 1e-10 of the mode's largest element, the cross sections within 1e-11) and against the
reference's Arb records (the bounds of the plain FP64 method: 5e-8, and 1e-9 for the
converged efficiencies)."""

import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from scatrs_b200 import _native
from scatrs_b200.errors import InvalidInputError, NotConvergedError

pytestmark = pytest.mark.gpu

RECORDS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "spheroid.json")))
FIXED = [r for r in RECORDS if ",N=" in r["case"]]
CONVERGED = [r for r in RECORDS if r["case"].endswith(",converged")]


def _settles(r):
    eps = r["eps"]
    far = max(eps, 1 / eps) - 1
    return far < 1.999 or (far < 2.001 and abs(complex(*r["m"]).imag) < 0.1)


@pytest.mark.parametrize("r", FIXED, ids=[r["case"] for r in FIXED])
def test_fixed_tmatrix_matches_the_oracle_and_the_records(gpu, r):
    from test_oracle_tmatrix import compare_fixed
    x, eps, s, N, nt = r["x"], r["eps"], complex(*r["m"]), r["n_terms"], r["n_theta"]
    # The cancellation that bounds the method's accuracy also amplifies the rounding of two
    # summation orders: 1e-10 for moderate shapes, 1e-7 where max(eps, 1/eps) >= 3.
    tol = 1e-10 if max(eps, 1 / eps) < 2.999 else 1e-7
    for mm in sorted({0, 1, N // 2, N}):
        g = _native.spheroid_tmatrix(x, eps, s, mm, N, nt)
        o = O.tmatrix_mode(x, eps, s, mm, N, nt)
        assert g.shape == o.shape
        assert np.abs(g - o).max() <= tol * np.abs(o).max()
    assert compare_fixed(r, _native.spheroid_tmatrix) <= 5e-8


def test_a_sphere_gives_the_mie_coefficients(gpu):
    x, s = 3.0, 1.5 + 0.01j
    mie = O.mie(x, s, n_max=12)
    for mm in (0, 1, 5, 12):
        T = _native.spheroid_tmatrix(x, 1.0, s, mm, 12, 20)
        k = T.shape[0] // 2
        n0 = max(mm, 1)
        for i in range(k):
            assert abs(T[i, i] + mie["b"][n0 + i - 1]) <= 1e-13
            assert abs(T[k + i, k + i] + mie["a"][n0 + i - 1]) <= 1e-13
        assert np.abs(T - np.diag(np.diag(T))).max() <= 1e-13


def test_converged_efficiencies_in_one_batch(gpu):
    """Every settling record in one call: Q equal to the oracle's loop to 10 rtol (the last
    step's change can sit at rtol's own level, where rounding decides whether one more n_theta
    step is taken) and to the records' to 1e-9."""
    recs = [r for r in CONVERGED if _settles(r)]
    rt = [1e-10 if max(r["eps"], 1 / r["eps"]) < 2.999 else 1e-8 for r in recs]
    for rtol in sorted(set(rt)):
        sel = [r for r, t in zip(recs, rt) if t == rtol]
        x = np.array([r["x"] for r in sel])
        eps = np.array([r["eps"] for r in sel])
        m = np.array([complex(*r["m"]) for r in sel])
        q, n, nth = _native.spheroid_efficiencies(x, eps, m, rtol)
        for i, r in enumerate(sel):
            qo, no, ntho = O.spheroid_converged(r["x"], r["eps"], complex(*r["m"]), rtol)
            assert n[i] == no and nth[i] >= 2 * n[i], r["case"]
            assert np.abs(q[i] - qo).max() <= 10 * rtol * qo[0], r["case"]
            qe = r["q_ext"][0][0] + r["q_ext"][0][1]
            qs = r["q_sca"][0][0] + r["q_sca"][0][1]
            assert abs(q[i, 0] - qe) <= 1e-9 * qe
            assert abs(q[i, 1] - qs) <= 1e-9 * qs


def test_unsettled_spheroids_report_not_converged(gpu):
    r = next(r for r in CONVERGED if not _settles(r))
    with pytest.raises(NotConvergedError):
        _native.spheroid_efficiencies([r["x"]], [r["eps"]], [complex(*r["m"])], 1e-8)


def test_invalid_inputs(gpu):
    with pytest.raises(InvalidInputError):
        _native.spheroid_tmatrix(1.0, 2.0, 1.5, 0, 0, 10)
    with pytest.raises(InvalidInputError):
        _native.spheroid_tmatrix(1.0, -2.0, 1.5, 0, 5, 10)
    with pytest.raises(InvalidInputError):
        _native.spheroid_efficiencies([1.0], [2.0], [1.5 - 0.1j], 1e-8)
