"""The oracle against the reference's Arb golden data (reference/data/*.jsonl, committed as
tests/golden/*.json), within the reference's declared tolerances C (kappa' + cond) 2^-52
(scatrs/src/mie/domain.rs:145-199): the same checks as scatrs/tests/mie_reference.rs, with the
condition numbers from the oracle's closed-form derivatives or central differences."""

import json
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.join(os.path.dirname(__file__), "golden")
EPS = 2.0 ** -52


def load(name):
    with open(os.path.join(HERE, name + ".json")) as f:
        return json.load(f)


def val(pairs, i):
    return pairs[i][0] + pairs[i][1]


def kappa(x, m):
    """condition_factor (domain.rs:145-147): (1 + max(1,|m|) x) max(1, |m|/|m-1|)."""
    near = max(abs(m) / abs(m - 1), 1.0) if m != 1 else np.inf
    return (1.0 + max(abs(m), 1.0) * x) * near


def test_coefficients_within_declared_tolerance():
    worst = 0.0
    for r in load("mie_coefficients"):
        x, m = r["x"], complex(*r["m"])
        orders = np.array(r["orders"])
        n_max = max(O.default_n_max(x), int(orders.max()))
        s = O.mie(x, m, n_max=n_max, derivatives=True)
        for stem in ("a", "b"):
            ref = np.array([complex(val(r[stem + "_re"], i), val(r[stem + "_im"], i))
                            for i in range(orders.size)])
            got = s[stem][orders - 1]
            scale = np.abs(ref).max()
            if scale == 0.0:
                continue
            dx, dm = s[f"d{stem}_dx"][orders - 1], s[f"d{stem}_dm"][orders - 1]
            cond = (x * np.abs(dx).max() + abs(m) * np.abs(dm).max()) / scale
            tol = 16.0 * (kappa(x, m) + cond) * EPS
            err = np.abs(got - ref).max() / scale
            worst = max(worst, err / tol)
            assert err <= tol, (r["case"], stem, err, tol)
    assert worst > 0.0


def _q(x, m):
    s = O.mie(x, m)
    return np.array([s["q_ext"], s["q_sca"], s["q_abs"], s["q_back"], s["g"]])


def test_efficiencies_and_amplitudes_within_declared_tolerance():
    names = ("q_ext", "q_sca", "q_abs", "q_back", "g")
    for r in load("mie_series"):
        x, m = r["x"], complex(*r["m"])
        q = _q(x, m)
        h = 1e-6
        dqx = (_q(x * (1 + h), m) - _q(x * (1 - h), m)) / (2 * h)  # x dQ/dx
        dqr = (_q(x, m + h * m.real) - _q(x, m - h * m.real)) / (2 * h)
        dqi = (_q(x, m + 1j * h * m.imag) - _q(x, m - 1j * h * m.imag)) / (2 * h) \
            if m.imag > 0 else 0.0 * q
        for k, name in enumerate(names):
            ref = val(r[name], 0)
            if name == "q_abs" and m.imag == 0.0:
                assert q[k] == 0.0
                continue
            if name == "q_back":
                s = max(abs(ref), q[1])
            elif name == "g":
                s = max(abs(ref), 1e-3 * min(1.0, x * x))
            else:
                s = abs(ref)
            if s == 0.0:
                continue
            cond = (abs(dqx[k]) + abs(dqr[k]) + abs(dqi[k])) / s
            tol = 16.0 * (kappa(x, m) + cond) * EPS + 1e-15
            assert abs(q[k] - ref) / s <= tol, (r["case"], name, q[k], ref)
        mu = np.array(r["mu"])
        s1, s2 = O.amplitudes(x, m, mu)
        srms = x * np.sqrt(q[1]) / 2
        for stem, arr in (("s1", s1), ("s2", s2)):
            ref = np.array([complex(val(r[stem + "_re"], j), val(r[stem + "_im"], j))
                            for j in range(mu.size)])
            err = np.abs(arr - ref) / np.maximum(np.abs(ref), srms)
            # amplitudes: C = 128; their condition is bounded here by kappa (no derivatives)
            tol = 128.0 * kappa(x, m) * EPS * 8
            assert err.max() <= tol, (r["case"], stem, err.max(), tol)


def test_gauss_legendre_matches_arb():
    for r in load("gauss_legendre"):
        n = r["n"]
        x, w = O.gauss_legendre(n)
        rx = np.array([val(r["nodes"], i) for i in range(n)])
        rw = np.array([val(r["weights"], i) for i in range(n)])
        assert np.abs(x - rx).max() <= (1.0 if n <= 100 else 32.0) * EPS
        assert (np.abs(w - rw) / rw).max() <= (1.0 if n <= 100 else 32.0) * EPS
        assert np.array_equal(x, -x[::-1]) and np.array_equal(w, w[::-1])


def test_wigner_d_matches_arb():
    for r in load("wigner_d"):
        d = O.wigner_d(r["m"], r["n"], r["x"], r["l_max"])
        ref = np.array([val(r["d"], l) for l in range(r["l_max"] + 1)])
        bound = 16.0 * (np.arange(ref.size) + 1) * EPS
        assert np.all(np.abs(d - ref) <= bound), (r["m"], r["n"], r["x"])


def test_greek_coefficients_within_declared_tolerance():
    names = ("alpha1", "alpha2", "alpha3", "alpha4", "beta1", "beta2")
    for r in load("mie_greek"):
        x, m, L = r["x"], complex(*r["m"]), r["order"]
        g = O.mie_greek(x, m, L)
        A = max(abs(val(r["alpha1"], l)) for l in range(L + 1))
        quad = ((L + 1) ** 2 + x * x) / 8.0
        tol = 8.0 * (kappa(x, m) + quad) * EPS * 16  # cond not tabulated: slack 16
        for k, name in enumerate(names):
            ref = np.array([val(r[name], l) for l in range(L + 1)])
            assert np.abs(g[k] - ref).max() / A <= tol, (r["case"], name)


def test_phase_matrix_matches_arb():
    for r in load("mie_phase"):
        x, m, mu = r["x"], complex(*r["m"]), np.array(r["mu"])
        s1, s2 = O.amplitudes(x, m, mu)
        q = _q(x, m)
        c = 4.0 / (x * x) / q[1]  # normalized
        n1, n2 = np.abs(s1) ** 2, np.abs(s2) ** 2
        p = s2 * np.conj(s1)
        f = {"f11": c * 0.5 * (n1 + n2), "f12": c * 0.5 * (n2 - n1), "f33": c * p.real,
             "f34": c * p.imag}
        ref11 = np.array([val(r["f11"], j) for j in range(mu.size)])
        scale = np.maximum(ref11, 1.0)
        for name, got in f.items():
            ref = np.array([val(r[name], j) for j in range(mu.size)])
            assert np.all(np.abs(got - ref) / scale <= 32.0 * kappa(x, m) * EPS * 16), \
                (r["case"], name)


def kappa_layered(x_outer, ms):
    """layered condition_factor (layered/domain.rs:95-110): the largest index and the largest
    near-unity factor of any layer whose index is not exactly 1."""
    big = max([1.0] + [abs(m) for m in ms])
    near = max([1.0] + [abs(m) / abs(m - 1) for m in ms if m != 1])
    return (1.0 + big * x_outer) * near


def test_layered_within_declared_tolerance():
    for r in load("layered_coefficients"):
        x = np.array(r["x"])
        ms = np.array(r["m_re"]) + 1j * np.array(r["m_im"])
        s = O.layered(x, ms)
        orders = np.array(r["orders"])
        if orders.max() > s["n"]:
            continue
        tol = 16.0 * kappa_layered(x[-1], ms) * EPS * 4  # cond not tabulated: slack 4
        for stem in "ab":
            ref = np.array([complex(val(r[stem + "_re"], i), val(r[stem + "_im"], i))
                            for i in range(orders.size)])
            scale = np.abs(ref).max()
            if scale == 0.0:
                continue
            assert np.abs(s[stem][orders - 1] - ref).max() / scale <= tol, (r["case"], stem)
    for r in load("layered_series"):
        x = np.array(r["x"])
        ms = np.array(r["m_re"]) + 1j * np.array(r["m_im"])
        s = O.layered(x, ms)
        names = ("q_ext", "q_sca", "q_abs", "q_back", "g")
        q = np.array([s[k] for k in names])
        # cond by central differences in every layer's x, Re m and Im m (relative step 1e-6)
        cond_num = np.zeros(5)
        h = 1e-6
        for l in range(x.size):
            for kind in ("x", "re", "im"):
                if kind == "x" and l > 0 and x[l] == x[l - 1]:
                    continue
                xp, xm, mp, mm = x.copy(), x.copy(), ms.copy(), ms.copy()
                if kind == "x":
                    xp[l] *= 1 + h
                    xm[l] *= 1 - h
                    if (l + 1 < x.size and xp[l] > x[l + 1]) or (l > 0 and xm[l] < x[l - 1]):
                        continue
                elif kind == "re":
                    mp[l] += h * ms[l].real
                    mm[l] -= h * ms[l].real
                else:
                    if ms[l].imag == 0.0:
                        continue
                    mp[l] += 1j * h * ms[l].imag
                    mm[l] -= 1j * h * ms[l].imag
                sp, sm = O.layered(xp, mp), O.layered(xm, mm)
                cond_num += np.abs(np.array([sp[k] - sm[k] for k in names])) / (2 * h)
        for i, k in enumerate(names):
            ref = val(r[k], 0)
            if ref == 0.0:
                continue
            scale = max(abs(ref), s["q_sca"]) if k == "q_back" else abs(ref)
            if k == "q_abs":
                scale = max(abs(ref), 1e-3 * s["q_ext"])
            tol = 16.0 * (kappa_layered(x[-1], ms) + cond_num[i] / scale) * EPS * 4
            assert abs(q[i] - ref) / scale <= tol, (r["case"], k, q[i], ref)


def test_coefficient_derivatives_within_declared_tolerance():
    """da/dx, da/dm, db/dx, db/dm against the Arb records (reference/data/mie_derivatives.jsonl)
    within 512 (1 + max(1, |m|) x + cond) 2^-52 of the largest |value| of each array
    (scatrs/src/mie/domain.rs:150-199, CoefficientDerivatives), cond from central differences
    of the oracle's own derivatives (x |d/dx| + |m| |d/dm|, relative)."""
    worst = 0.0
    for r in load("mie_coefficient_derivatives"):
        x, m = r["x"], complex(*r["m"])
        orders = np.array(r["orders"])
        n_max = max(O.default_n_max(x), int(orders.max()))
        s = O.mie(x, m, n_max=n_max, derivatives=True)
        h = 1e-5
        sp = O.mie(x * (1 + h), m, n_max=n_max, derivatives=True)
        sm = O.mie(x * (1 - h), m, n_max=n_max, derivatives=True)
        mp = O.mie(x, m * (1 + h), n_max=n_max, derivatives=True)
        mm = O.mie(x, m * (1 - h), n_max=n_max, derivatives=True)
        for key in ("da_dx", "da_dm", "db_dx", "db_dm"):
            ref = np.array([complex(val(r[key + "_re"], i), val(r[key + "_im"], i))
                            for i in range(orders.size)])
            got = s[key][orders - 1]
            scale = np.abs(ref).max()
            if scale == 0.0:
                continue
            ddx = (sp[key][orders - 1] - sm[key][orders - 1]) / (2 * h)   # x d/dx
            ddm = (mp[key][orders - 1] - mm[key][orders - 1]) / (2 * h)   # m d/dm
            cond = (np.abs(ddx).max() + np.abs(ddm).max()) / scale
            tol = 512.0 * (1.0 + max(abs(m), 1.0) * x + cond) * EPS
            err = np.abs(got - ref).max() / scale
            worst = max(worst, err / tol)
            assert err <= tol, (r["case"], key, err, tol)
    assert worst > 0.0


def single_node(x, lam=1.0):
    """A fixed grid whose one node is a sphere of size parameter x at wavelength lam: a
    lognormal on [r / 1.5, 1.5 r], whose one Gauss node is the midpoint in ln r."""
    r = x * lam / (2.0 * np.pi)
    d = np.zeros(1, dtype=O.DIST_DTYPE)
    d["kind"] = 1
    d["p"][0, :2] = (r, 1.5)
    d["r_lo"], d["r_hi"] = r / 1.5, r * 1.5
    return d, r


JAC_NAMES = ("q_ext", "q_sca", "q_abs", "q_back")


def jacobian_errors(r, q, dq):
    """Errors of dQ/dRe m, dQ/dIm m (dq[p][k], p = 0 Re, 1 Im) against a record, relative to
    max(|dQ|, |Q|) (Q_back against max(Q_back, Q_sca)), and their bounds
    256 (kappa max(1, |m|/|m-1|)) 2^-52 (scatrs/src/mie/domain.rs:150-199, EfficiencyJacobian)."""
    x, m = r["x"], complex(*r["m"])
    near = max(abs(m) / abs(m - 1), 1.0) if m != 1 else np.inf
    tol = 256.0 * kappa(x, m) * near * EPS
    out = []
    for p, key in enumerate(("dm_re", "dm_im")):
        for k, name in enumerate(JAC_NAMES):
            ref = val(r[f"{name}_{key}"], 0)
            qs = max(abs(q[k]), abs(q[1])) if name == "q_back" else abs(q[k])
            scale = max(abs(ref), qs, 1e-300)
            out.append((name + "_" + key, abs(dq[p][k] - ref) / scale, tol))
    return out


def test_efficiency_jacobian_of_the_oracle_within_declared_tolerance():
    """The oracle's dQ/dRe m and dQ/dIm m through its one-node fixed-grid ensemble with
    derivatives (d c / dm = pi r^2 dQ/dm) against the Arb records' efficiency Jacobian."""
    worst = 0.0
    for r in load("mie_jacobian"):
        x, m = r["x"], complex(*r["m"])
        d, rad = single_node(x)
        out = O.ensemble_fixed_d(d, np.array([1.0]), np.array([[m]]), 1, None, -1,
                                 allow_unvalidated=True)
        area = np.pi * rad * rad
        q = out["values"][:4, 0] / area
        dq = out["d_values"][2:4, :4, 0] / area
        for name, err, tol in jacobian_errors(r, q, dq):
            worst = max(worst, err / tol)
            assert err <= tol, (r["case"], name, err, tol)
    assert worst > 0.0
