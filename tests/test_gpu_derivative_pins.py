"""The GPU's derivative blocks pinned to the reference's Arb derivative records
(reference/data/mie_derivatives.jsonl and layered_derivatives.jsonl, committed as
tests/golden/mie_jacobian.json and layered_derivatives.json).

A fixed grid of one node (a lognormal on [r / 1.5, 1.5 r], whose one Gauss node is r) makes the
ensemble's outputs a single sphere's: c = pi r^2 Q, and the derivative blocks along m (and along
a layered sphere's radius fractions, f_l = x_l / x_L) are pi r^2 times the efficiency Jacobian
that the records hold. The bound is the reference's declared one for the efficiency Jacobian,
256 (kappa max(1, |m|/|m - 1|)) 2^-52 (scatrs/src/mie/domain.rs:150-199;
scatrs/src/layered/domain.rs:117-163 with the layered kappa), relative to max(|dQ|, |Q|).
"""

import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from scatrs_b200 import _native

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(__file__), "golden")
EPS = 2.0 ** -52
NAMES = ("q_ext", "q_sca", "q_abs", "q_back")


def load(name):
    with open(os.path.join(HERE, name + ".json")) as f:
        return json.load(f)


def val(pairs, i=0):
    return pairs[i][0] + pairs[i][1]


def single_node(x, lam=1.0):
    r = x * lam / (2.0 * np.pi)
    d = np.zeros(1, dtype=_native.DIST_DTYPE)
    d["kind"] = 1
    d["param"][0, :2] = (r, 1.5)
    d["r_lo"], d["r_hi"] = r / 1.5, r * 1.5
    return d, r


def near_one(m):
    return max(abs(m) / abs(m - 1), 1.0) if m != 1 else np.inf


def check(got, ref, q, q_sca, tol, what):
    qs = max(abs(q), abs(q_sca)) if what.startswith("q_back") else abs(q)
    scale = max(abs(ref), qs, 1e-300)
    err = abs(got - ref) / scale
    assert err <= tol, (what, got, ref, err, tol)
    return err / tol


def test_sphere_jacobian_matches_arb(gpu):
    worst = 0.0
    for r in load("mie_jacobian"):
        x, m = r["x"], complex(*r["m"])
        d, rad = single_node(x)
        v, _, _, dv, _, _ = gpu.ensemble_fixed_d(d, np.array([1.0]), np.array([[m]]), None, 1,
                                                 -1, allow_unvalidated=True)
        area = np.pi * rad * rad
        q = v[:4, 0] / area
        kappa = (1.0 + max(abs(m), 1.0) * x) * near_one(m)
        tol = 256.0 * kappa * near_one(m) * EPS
        for p, key in ((2, "dm_re"), (3, "dm_im")):
            for k, name in enumerate(NAMES):
                worst = max(worst, check(dv[p, k, 0] / area, val(r[f"{name}_{key}"]), q[k],
                                         q[1], tol, f"{r['case']} {name}_{key}"))
        # and the oracle's, computed the same way, to rounding
        od = np.zeros(1, dtype=O.DIST_DTYPE)
        od["kind"], od["p"], od["r_lo"], od["r_hi"] = d["kind"], d["param"], d["r_lo"], d["r_hi"]
        ref = O.ensemble_fixed_d(od, np.array([1.0]), np.array([[m]]), 1, None, -1,
                                 allow_unvalidated=True)
        s = np.maximum(np.abs(ref["d_values"][2:4, :4, 0]), np.abs(ref["values"][None, :4, 0]))
        s[:, 3] = np.maximum(s[:, 3], np.abs(ref["values"][1, 0]))  # C_back against C_sca
        assert np.all(np.abs(dv[2:4, :4, 0] - ref["d_values"][2:4, :4, 0]) <= 1e-12 * s), r["case"]
    assert worst > 0.0


def test_layered_jacobian_matches_arb(gpu):
    """Per layer l: dQ/dRe m_l, dQ/dIm m_l; per inner interface l: dQ/dx_l (the fraction
    block over x_L); Q_ext, Q_sca, Q_abs, Q_back and g."""
    worst = 0.0
    for r in load("layered_derivatives"):
        xs = np.array(r["x"], dtype=float)
        m = np.array([complex(a, b) for a, b in zip(r["m_re"], r["m_im"])])
        L, xL = xs.size, xs[-1]
        d, rad = single_node(xL)
        fr = (xs[:-1] / xL)[None, :]
        ml = m.reshape(1, L, 1)
        v, _, _, dv, _, _ = gpu.ensemble_fixed_layered_d(d, np.array([1.0]), fr, ml, None, 1,
                                                         -1, allow_unvalidated=True)
        area = np.pi * rad * rad
        q = v[:4, 0] / area
        g = v[5, 0]
        big = max(1.0, max(abs(z) for z in m))
        near = max(near_one(z) for z in m if z != 1)
        kappa = (1.0 + big * xL) * near
        tol = 256.0 * kappa * near * EPS
        rows = []
        for layer in range(L):
            rows.append((2 + 2 * layer, f"dm_re{layer}", 1.0))
            rows.append((2 + 2 * layer + 1, f"dm_im{layer}", 1.0))
        for f in range(L - 1):
            rows.append((2 + 2 * L + f, f"dx{f}", 1.0 / xL))
        for blk, key, factor in rows:
            for k, name in enumerate(NAMES):
                if f"{name}_{key}" not in r:
                    continue
                got = dv[blk, k, 0] / area * factor
                worst = max(worst, check(got, val(r[f"{name}_{key}"]), q[k], q[1], tol,
                                         f"{r['case']} {name}_{key}"))
            gk = "g_" + key
            if gk in r:
                worst = max(worst, check(dv[blk, 5, 0] * factor, val(r[gk]), g, g, tol,
                                         f"{r['case']} {gk}"))
    assert worst > 0.0
