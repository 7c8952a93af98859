"""The adaptive ensemble with derivatives on the GPU (scatrs_ensemble_mixture_d: pass 1 with the
parameter blocks and the derivatives along m from pass1_kernel, pass 2's derivative blocks with
per-panel error sums, averaged per node before the Greek projection, mixed on the host with the
weight derivatives) against the oracle's restatement (itself checked against central
differences): the same panels and flags; values as the adaptive path's (1e-12); derivatives as
the fixed grid's derivative path (1e-9 of the largest derivative of the same output, the ratio
rule of test_gpu_derivatives); error estimates within 1e-9 of their size or 1e-13 of the
value's scale."""

import numpy as np
import pytest

from oracle import oracle as O
from scatrs_b200 import _native, _scatrs
from scatrs_b200.errors import InvalidInputError
from test_gpu_adaptive import _compare, _odist
from test_gpu_derivatives import _compare as _compare_d

pytestmark = pytest.mark.gpu

MU = np.array([1.0, 0.6, 0.0, -0.35, -1.0])
PD, RE, IM, W = 0, 1, 2, 3


def _dist(kind, *p):
    d = _native.dist_records(1)
    d[0]["kind"] = kind
    d[0]["param"][: len(p)] = p
    return d


def _both(comps, params, wl, L=12, **kw):
    got = _native.ensemble_mixture_d(comps, wl, np.array(params, dtype=_native.PARAM_DTYPE), MU,
                                     L, **kw)
    oc = [(_odist(d), mw, w, m) for d, mw, w, m in comps]
    ref = O.ensemble_mixture_d(oc, wl, O.params(*params), mu=MU, greek_order=L, **kw)
    return got, ref


def _check(got, ref):
    _compare(got, ref)
    tup = (got["values"], got["phase"], got["greek"], got["d"], got["phase_d"], got["greek_d"])
    r = {"values": ref["values"], "phase": ref["phase"], "greek": ref["greek"],
         "d_values": ref["d"], "d_phase": ref["phase_d"], "d_greek": ref["greek_d"]}
    _compare_d(tup, r)
    for key in ("d", "phase_d", "greek_d"):
        e, re_ = got[key + "_err"], ref[key + "_err"]
        scale = np.abs(ref[key]).max(axis=-1, keepdims=True)
        assert np.all(np.abs(e - re_) <= 1e-9 * np.abs(re_) + 1e-13 * scale), key


def test_a_lognormal_matches_the_oracle(gpu):
    wl = np.array([0.45, 0.8])
    m = np.array([1.5 + 0.01j, 1.45 + 0.002j])
    got, ref = _both([(_dist(1, 0.2, 1.5), None, 1.0, m)],
                     [(0, -1, PD, 0), (0, -1, PD, 1), (0, -1, RE, 0), (0, -1, IM, 0)], wl)
    _check(got, ref)


@pytest.mark.parametrize("dist,params", [
    ((2, 0.5, 0.1), [(0, -1, PD, 1)]),                       # a parameter alone
    ((3, 2.0, 15.0, 0.5), [(0, -1, IM, 0), (0, -1, PD, 2)]),  # Im m and gamma
    ((4, 3.0, 0.02, 1.0), [(0, -1, PD, 0), (0, -1, RE, 0)]),  # finite support
    ((5, 0.3), [(0, -1, IM, 0), (0, -1, RE, 0)]),             # a single radius along m
    ((5, 0.3), [(0, -1, PD, 0)]),                             # its radius (engine.rs:1158-1170)
])
def test_other_kinds_match_the_oracle(gpu, dist, params):
    wl = np.array([0.55, 0.9])
    m = np.array([1.45 + 0.02j, 1.44 + 0.01j])
    got, ref = _both([(_dist(*dist), None, 1.0, m)], params, wl, L=10, refine_backscatter=True)
    _check(got, ref)


@pytest.mark.parametrize("radius,m", [(2.1, 1.33 + 1e-8j), (0.05, 1.6 + 0.3j), (6.0, 1.5 + 0.1j)])
def test_a_single_radius_along_its_radius_and_m(gpu, radius, m):
    """The single radius's derivative along r (the Mie pass along x at fixed m) beside those
    along Re m and Im m, from x = 0.3 to x = 75, nearly real to strongly absorbing m."""
    wl = np.array([0.5, 1.0])
    got, ref = _both([(_dist(5, radius), None, 1.0, np.array([m, m]))],
                     [(0, -1, RE, 0), (0, -1, PD, 0), (0, -1, IM, 0)], wl, L=10)
    _check(got, ref)
    assert np.all(got["d_err"] == 0.0)


def test_a_single_radius_in_a_mixture(gpu):
    """A monodisperse component's radius, the other component's width and the weights."""
    comps = [(_dist(5, 0.4), None, 0.3, np.array([1.5 + 0.01j])),
             (_dist(1, 0.2, 1.5), None, 1.0, np.array([1.45 + 0.001j]))]
    got, ref = _both(comps, [(0, -1, PD, 0), (1, -1, PD, 1), (0, -1, W, 0)], np.array([0.6]))
    _check(got, ref)


def test_mixtures_and_modes_match_the_oracle(gpu):
    wl = np.array([0.5, 0.75])
    bi = _native.dist_records(2)
    bi[0]["kind"], bi[1]["kind"] = 1, 2
    bi[0]["param"][:2] = (0.1, 1.5)
    bi[1]["param"][:2] = (0.6, 0.12)
    comps = [(bi, [2.0, 0.5], 1.5, np.array([1.45 + 0j, 1.44 + 1e-5j])),
             (_dist(4, 3.5, 0.05, 1.5), None, 0.5, np.array([1.53 + 0.01j, 1.52 + 0.02j]))]
    params = [(0, 0, PD, 1), (0, 1, W, 0), (0, -1, W, 0), (1, -1, RE, 0), (1, -1, PD, 0),
              (0, 1, PD, 0), (1, -1, W, 0)]
    got, ref = _both(comps, params, wl, L=16)
    _check(got, ref)


def test_a_table_along_m(gpu):
    d = _native.dist_records(1)
    _native.set_table(d, 0, [0.05, 0.1, 0.4, 1.0], [0.0, 3.0, 1.0, 0.2])
    got, ref = _both([(d, None, 1.0, np.array([2.0 + 0.5j]))], [(0, -1, RE, 0), (0, -1, IM, 0)],
                     np.array([0.4]), L=8)
    _check(got, ref)


def test_the_reference_call(gpu):
    """ensemble_compute(deriv_idx=...) through the reference-facing mirror: the dict's d blocks
    are the raw binding's in the order asked, and its parameter errors."""
    wl = np.array([0.5, 0.8])
    m = np.array([1.5 + 0.01j, 1.45 + 0.002j])
    items = [(("lognormal", 0.2, 1.5), ("sphere", m), 1.0)]
    raw = _scatrs.ensemble_compute(items, wl, False, 8, False, MU, True, [3, 1], 1e-6, 4096,
                                   False, False)
    ref = _native.ensemble_mixture_d([(_dist(1, 0.2, 1.5), None, 1.0, m)], wl,
                                     np.array([(0, -1, IM, 0), (0, -1, PD, 1)],
                                              dtype=_native.PARAM_DTYPE), MU, 8)
    assert np.array_equal(raw["d"], ref["d"]) and np.array_equal(raw["d_errors"], ref["d_err"])
    assert np.array_equal(raw["greek_d"], ref["greek_d"])
    assert raw["phase_d_errors"].shape == (2, 6, 2, MU.size)
    with pytest.raises(InvalidInputError, match="no parameter 9"):
        _scatrs.ensemble_compute(items, wl, False, None, False, None, True, [9], 1e-6, 4096,
                                 False, False)
    with pytest.raises(InvalidInputError, match="width requested twice"):
        _scatrs.ensemble_compute(items, wl, False, None, False, None, True, [1, 1], 1e-6, 4096,
                                 False, False)
    # A layered sphere's directions (its checks against differences are in
    # test_gpu_adaptive_layered_derivatives.py).
    layered = [(("lognormal", 0.2, 1.5), ("layered", [0.5], np.stack([m, m])), 1.0)]
    lay = _scatrs.ensemble_compute(layered, wl, False, None, False, None, True, [2], 1e-6, 4096,
                                   False, False)
    assert lay["d"].shape == (1, 11, wl.size) and np.all(np.isfinite(lay["d"]))
    mono = _scatrs.ensemble_compute([(("monodisperse", 0.3), ("sphere", m), 1.0)], wl, False,
                                    None, False, None, True, [0], 1e-6, 4096, False, False)
    ref = _native.ensemble_mixture_d([(_dist(5, 0.3), None, 1.0, m)], wl,
                                     np.array([(0, -1, PD, 0)], dtype=_native.PARAM_DTYPE), None,
                                     -1)
    assert np.array_equal(mono["d"], ref["d"]) and not mono["d_errors"].any()


def test_invalid_parameters_are_rejected(gpu):
    comps = [(_dist(1, 0.2, 1.5), None, 1.0, np.array([1.5 + 0j]))]
    for bad, msg in [([(0, -1, PD, 2)], "no parameter"), ([(1, -1, RE, 0)], "no parameter"),
                     ([(0, 0, PD, 0)], "no parameter"), ([(0, 0, W, 0)], "no parameter"),
                     ([(0, -1, RE, 0), (0, -1, RE, 0)], "requested twice")]:
        with pytest.raises(InvalidInputError, match=msg):
            _native.ensemble_mixture_d(comps, [0.5], np.array(bad, dtype=_native.PARAM_DTYPE))
