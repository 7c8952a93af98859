"""Derivatives of a randomly oriented spheroid's outputs along x, the aspect ratio, Re m and Im m
(scatrs_spheroid_compute_d) against central differences of the oracle's EBCM at the same N and
n_theta, with the bound of the reference's own check (tmatrix/mod.rs:965-1040): |d - fd| within
1e-6 of the output's scale over the parameter's size."""

import numpy as np
import pytest

from oracle import oracle as O
from scatrs_b200 import _native, _scatrs

pytestmark = pytest.mark.gpu

ORDER = 8


def oracle_outputs(x, eps, m, n, nth):
    """The efficiencies (Q_ext, Q_sca, Q_abs, Q_back, g) and the unnormalized Greek coefficients
    (times 4 / x^2, orders 0..ORDER) of the oracle at a fixed discretization."""
    modes = O.tmatrix_modes(x, eps, m, n, nth)
    q_ext, q_sca = O.spheroid_q(x, eps, m, n, nth)
    raw = O.random_greek(modes, 2 * n)
    f11 = np.sum(raw[0] * (-1.0) ** np.arange(raw.shape[1]))
    q_back = 4.0 * np.pi * f11 / (np.pi * x * x)
    g = raw[0, 1] / (3.0 * raw[0, 0])
    greek = np.zeros((6, ORDER + 1))
    k = min(ORDER + 1, raw.shape[1])
    greek[:, :k] = raw[:, :k] * 4.0 / (x * x)
    return np.array([q_ext, q_sca, q_ext - q_sca, q_back, g]), greek


def oracle_fd(x, eps, m, n, nth, direction, h):
    """Richardson-extrapolated central differences (steps h, h / 2); forward fourth-order
    differences along Im m when Im m < 4 h."""
    def at(step):
        args = [x, eps, m]
        if direction == 0:
            args[0] = x + step
        elif direction == 1:
            args[1] = eps + step
        elif direction == 2:
            args[2] = m + step
        else:
            args[2] = m + 1j * step
        return oracle_outputs(*args, n, nth)

    if direction == 3 and m.imag < 4 * h:
        f = [at(k * h) for k in range(5)]
        c = (-25.0, 48.0, -36.0, 16.0, -3.0)
        return tuple(sum(ci * fk[j] for ci, fk in zip(c, f)) / (12 * h) for j in range(2))
    a, b = at(h), at(-h)
    a2, b2 = at(h / 2), at(-h / 2)
    return tuple((4 * (a2[j] - b2[j]) / h - (a[j] - b[j]) / (2 * h)) / 3 for j in range(2))


CASES = [(0.6, 3.0, 1.45 + 0.03j), (2.0, 5.0, 1.33 + 0.001j), (1.5, 2.0, 1.5 + 0.0j)]


@pytest.mark.parametrize("eps,x,m", CASES)
def test_spheroid_derivatives_match_differences(gpu, eps, x, m):
    r = _native.spheroid_compute_d([x], [eps], [m], rtol=1e-10, greek_order=ORDER,
                                   normalized=False)
    n, nth = int(r["n_terms"][0]), int(r["n_theta"][0])
    # the values are compute's at the same discretization
    ref = _native.spheroid_compute([x], [eps], [m], rtol=1e-10, greek_order=ORDER,
                                   normalized=False)
    assert np.allclose(r["efficiencies"], ref["efficiencies"], rtol=1e-13, atol=0)
    eff0, greek0 = oracle_outputs(x, eps, m, n, nth)
    assert np.allclose(r["efficiencies"][0], eff0, rtol=1e-10, atol=1e-14)
    sizes = (x, eps, abs(m), abs(m))
    for d in range(4):
        h = 1e-4 * sizes[d]
        fd_eff, fd_greek = oracle_fd(x, eps, m, n, nth, d, h)
        got_eff, got_greek = r["d_efficiencies"][d, 0], r["d_greek"][d, 0]
        scale = np.maximum(np.abs(eff0), 1e-300)
        scale[2] = max(scale[2], abs(eff0[0]))  # Q_abs = Q_ext - Q_sca: on Q_ext's scale
        assert np.all(np.abs(got_eff - fd_eff) <= 1e-6 * scale / sizes[d]), (
            d, got_eff, fd_eff)
        gscale = np.abs(greek0).max()
        assert np.all(np.abs(got_greek - fd_greek) <= 1e-6 * gscale / sizes[d]), (
            d, np.abs(got_greek - fd_greek).max(), gscale)
        assert np.abs(got_eff).max() > 0.0


def test_spheroid_derivatives_normalized_greek(gpu):
    """Normalized coefficients: alpha1_0 = 1 has no derivative; the rest follow the quotient."""
    eps, x, m = 0.6, 3.0, 1.45 + 0.03j
    u = _native.spheroid_compute_d([x], [eps], [m], rtol=1e-10, greek_order=ORDER,
                                   normalized=False)
    v = _native.spheroid_compute_d([x], [eps], [m], rtol=1e-10, greek_order=ORDER,
                                   normalized=True)
    g, dg = u["greek"][0], u["d_greek"][:, 0]
    expect = (dg - (g / g[0, 0])[None] * dg[:, :1, :1]) / g[0, 0]
    assert np.allclose(v["d_greek"][:, 0], expect, rtol=0, atol=1e-8)
    assert np.all(v["d_greek"][:, 0, 0, 0] == 0.0)


def _small_ensemble():
    d = np.zeros(1, dtype=_native.DIST_DTYPE)
    d["kind"] = 1
    d["param"][0, :2] = (0.12, 1.5)
    d["r_lo"], d["r_hi"] = 0.12 / 1.5 ** 3, 0.12 * 1.5 ** 3
    return d, np.array([0.5]), 1.6, np.array([[1.5 + 0.01j]]), np.array([-0.9, 0.1, 0.8])


def _oracle_ensemble(d, wl, eps, m, terms, mu, L):
    od = np.zeros(d.size, dtype=O.DIST_DTYPE)
    od["kind"], od["p"], od["r_lo"], od["r_hi"] = d["kind"], d["param"], d["r_lo"], d["r_hi"]
    r = O.ensemble_fixed_spheroid(od, wl, eps, m, terms.shape[1], terms, mu, L, True)
    return r["values"], r["phase"], r["greek"]


def test_spheroid_ensemble_derivatives_match_differences(gpu):
    """Every block (median, width, aspect ratio, Re m, Im m) of the spheroid ensemble against
    Richardson-extrapolated central differences of the oracle's ensemble at the same per-node
    (N, n_theta), within 1e-6 of each output's scale over the parameter's size."""
    d, wl, eps, m, mu = _small_ensemble()
    n_nodes, L = 6, 8
    v, ph, g, dv, dph, dg, terms = _native.ensemble_fixed_spheroid_d(d, wl, eps, m, mu, n_nodes,
                                                                     L, True, 1e-10)
    v0, ph0, g0, _ = _native.ensemble_fixed_spheroid(d, wl, eps, m, mu, n_nodes, L, True, 1e-10)
    assert np.allclose(v, v0, rtol=1e-13, atol=0) and np.allclose(g, g0, rtol=0, atol=1e-13)
    assert np.allclose(ph, ph0, rtol=1e-12, atol=0)
    ov, oph, og = _oracle_ensemble(d, wl, eps, m, terms, mu, L)
    assert np.allclose(v, ov, rtol=1e-9, atol=0)

    def at(k, step):
        dd, e, mm = d.copy(), eps, m.copy()
        if k < 2:
            dd["param"][0, k] += step
        elif k == 2:
            e = eps + step
        elif k == 3:
            mm = m + step
        else:
            mm = m + 1j * step
        return _oracle_ensemble(dd, wl, e, mm, terms, mu, L)

    sizes = (0.12, 1.5, eps, abs(m[0, 0]), abs(m[0, 0]))
    for k in range(5):
        h = 1e-4 * sizes[k]
        a, b, a2, b2 = at(k, h), at(k, -h), at(k, h / 2), at(k, -h / 2)
        fd = [(4 * (a2[q] - b2[q]) / h - (a[q] - b[q]) / (2 * h)) / 3 for q in range(3)]
        for got, ref, val, name in ((dv[k], fd[0], v, "values"), (dph[k], fd[1], ph, "phase"),
                                    (dg[k], fd[2], g, "greek")):
            scale = np.maximum(np.abs(val), np.abs(val).max(axis=tuple(range(1, val.ndim)),
                                                           keepdims=True) * 1e-3)
            err = np.abs(got - ref) / scale * sizes[k]
            assert err.max() <= 1e-6, (k, name, err.max())


def test_spheroid_autograd_aspect_ratio_gradient(gpu):
    """The torch gradient of a loss along the aspect ratio (and the other inputs) equals the
    Jacobian contraction, checked by central differences of the loss on the GPU path at fixed
    discretization through the derivative entry's own values."""
    import torch

    from scatrs_b200 import autograd as A

    d, wl, eps, m, mu = _small_ensemble()
    theta = torch.tensor([[0.12, 1.5]], dtype=torch.float64, requires_grad=True)
    e = torch.tensor([eps], dtype=torch.float64, requires_grad=True)
    m_re = torch.tensor(m.real, requires_grad=True)
    m_im = torch.tensor(m.imag, requires_grad=True)
    ranges = [[d["r_lo"][0], d["r_hi"][0]]]
    v, ph, g = A.ensemble_fixed_spheroid(theta, e, m_re, m_im, kind="lognormal", ranges=ranges,
                                         wavelengths=wl, mu=mu, n_nodes=6, greek_order=8,
                                         tmatrix_rtol=1e-10)
    loss = (v[0] ** 2 + v[5] + (g[0, :, 1:5] ** 2).sum() + ph[1].sum())
    loss.sum().backward()
    res = _native.ensemble_fixed_spheroid_d(d, wl, eps, m, mu, 6, 8, True, 1e-10)
    dv, dph, dg = res[3], res[4], res[5]
    vv, pp, gg = res[0], res[1], res[2]
    # dL/dp = 2 v0 dv0 + dv5 + 2 sum g dg + sum dph[1]
    expect = [2 * vv[0, 0] * dv[k, 0, 0] + dv[k, 5, 0] + 2 * (gg[0, 0, 1:5] * dg[k, 0, 0, 1:5]).sum()
              + dph[k, 1].sum() for k in range(5)]
    got = [theta.grad[0, 0].item(), theta.grad[0, 1].item(), e.grad[0].item(),
           m_re.grad[0, 0].item(), m_im.grad[0, 0].item()]
    assert np.allclose(got, expect, rtol=1e-12, atol=1e-15)
    assert abs(got[2]) > 0.0


def test_fixed_grid_binding_takes_spheroid_derivatives(gpu):
    """ensemble_compute_fixed with a spheroid and derivatives: its columns, in
    ensemble_parameters' order (median_radius, width, m_real, m_imag, aspect_ratio), are the
    library's blocks (the distribution's, the aspect ratio, Re m, Im m) bit for bit."""
    d, wl, eps, m, mu = _small_ensemble()
    spec = ("lognormal", 0.12, 1.5)
    particle = ("spheroid", eps, m[0])
    raw = _scatrs.ensemble_compute_fixed([spec], particle, wl, 8, False, mu, True, n_nodes=6,
                                         ranges=[(d["r_lo"][0], d["r_hi"][0])],
                                         derivatives=[4, 2, 0], tmatrix_rtol=1e-10)
    res = _native.ensemble_fixed_spheroid_d(d, wl, eps, m, mu, 6, 8, True, 1e-10)
    assert np.array_equal(raw["values"], res[0])
    for got, want in ((raw["d"], res[3]), (raw["phase_d"], res[4]), (raw["greek_d"], res[5])):
        assert np.array_equal(got, want[[2, 3, 0]])
