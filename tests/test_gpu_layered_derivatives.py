"""Derivatives of the layered-sphere ensemble on the GPU (scatrs_ensemble_fixed_layered_d: the
layered recursion carried in forward mode, one derivative pass per layer index and per radius
fraction) against Richardson-extrapolated central differences of the oracle's layered ensemble
(an independent double-precision restatement; steps 2e-5 and 1e-5 relative, so the differences'
truncation error is O(h^4); larger steps cross the layered recursion's switches between forms): the scalars, phase matrix and Greek coefficients along the
distribution's parameters, Re m_l and Im m_l of every layer and the fractions, within 1e-6 of
each output row's scale. Values equal the plain layered ensemble. The derivatives themselves are
pinned to the reference's Arb records in test_gpu_derivative_pins.py."""

import numpy as np
import pytest

from oracle import oracle as O
from scatrs_b200 import _native

pytestmark = pytest.mark.gpu

MU = np.array([-0.9, -0.2, 0.4, 0.95])
L = 8


def _case():
    d = np.zeros(2, dtype=_native.DIST_DTYPE)
    d["kind"] = 1
    d["param"][0, :2] = [0.12, 1.5]
    d["param"][1, :2] = [0.2, 1.4]
    for i in range(2):
        rg, sg = d["param"][i, :2]
        d["r_lo"][i], d["r_hi"][i] = rg * sg ** -3, rg * sg ** 3
    wl = np.array([0.45, 0.7])
    fr = np.array([[0.55, 0.85], [0.4, 0.92]])
    ml = np.empty((2, 3, 2), dtype=complex)
    ml[0] = [[1.9 + 0.05j, 1.85 + 0.04j], [1.45 + 0.002j, 1.44 + 0.002j], [1.34 + 1e-3j, 1.33 + 1e-3j]]
    ml[1] = [[1.6 + 0.2j, 1.6 + 0.2j], [2.1 + 0.01j, 2.0 + 0.01j], [1.5 + 0.003j, 1.5 + 0.003j]]
    return d, wl, fr, ml


def _oracle(d, wl, fr, ml):
    out = O.ensemble_fixed_layered(d.view(O.DIST_DTYPE), wl, fr, ml, 48, mu=MU, greek_order=L)
    return out["values"], out["phase"], out["greek"]


def test_matches_finite_differences(gpu):
    d, wl, fr, ml = _case()
    v, ph, g, dv, dph, dg = gpu.ensemble_fixed_layered_d(d, wl, fr, ml, MU, 48, L)
    pv, pph, pg = gpu.ensemble_fixed_layered(d, wl, fr, ml, MU, 48, L)
    assert np.allclose(v, pv, rtol=1e-12, atol=0)
    n_wl = wl.size
    blocks = []  # (block index, perturbation of (d, fr, ml) by h, its size)
    for p in range(2):
        blocks.append((p, "param", p))
    for layer in range(3):
        blocks.append((2 + 2 * layer, "re", layer))
        blocks.append((3 + 2 * layer, "im", layer))
    for f in range(2):
        blocks.append((8 + f, "fr", f))
    assert dv.shape[0] == 10
    for blk, kind, k in blocks:
        for dist in range(2):
            def perturbed(sign, rel):
                dd, ff, mm = d.copy(), fr.copy(), ml.copy()
                if kind == "param":
                    h = rel * dd["param"][dist, k]
                    dd["param"][dist, k] += sign * h
                elif kind == "re":
                    h = rel * abs(mm[dist, k, 0])
                    mm[dist, k, :] += sign * h
                elif kind == "im":
                    h = rel * abs(mm[dist, k, 0])
                    mm[dist, k, :] += sign * 1j * h
                else:
                    h = rel * ff[dist, k]
                    ff[dist, k] += sign * h
                return _oracle(dd, wl, ff, mm), h

            def central(rel):
                (vp, php, gp), h = perturbed(+1, rel)
                (vm, phm, gm), _ = perturbed(-1, rel)
                return [(p_ - m_) / (2 * h) for p_, m_ in ((vp, vm), (php, phm), (gp, gm))]

            coarse, fine = central(2e-5), central(1e-5)
            sl = slice(dist * n_wl, (dist + 1) * n_wl)
            for got, dc, df in zip((dv[blk], dph[blk], dg[blk]), coarse, fine):
                fd = (4.0 * df - dc) / 3.0  # Richardson: the h^2 terms cancel
                g_, f_ = got[:, sl], fd[:, sl]
                # Each output row (a scalar, a phase element, a Greek array) against its own
                # largest derivative in the unit slice.
                scale = np.abs(f_).reshape(f_.shape[0], -1).max(axis=1)
                err = np.abs(g_ - f_).reshape(f_.shape[0], -1).max(axis=1)
                assert np.all(err <= 1e-6 * np.maximum(scale, 1e-300)), (blk, kind, k, dist,
                                                                         err / scale)


def test_autograd_gradient_of_a_loss(gpu):
    """A loss of the layered-adjoint shape (weighted squared differences of c_ext, ssa, g and
    alpha1[0:16] from targets) differentiated by torch through scatrs_ensemble_fixed_layered_d:
    the gradient along the medians, widths, fractions and every layer's n and k (the same at
    every wavelength) against Richardson-extrapolated central differences of the loss (steps
    1e-4 and 5e-5 relative), 1e-6 relative."""
    import torch
    from scatrs_b200 import autograd

    d, wl, fr, ml = _case()
    ranges = np.stack([d["r_lo"], d["r_hi"]], axis=1)
    rng = np.random.default_rng(4)
    targets = rng.uniform(0.5, 1.5, (19, d.size * wl.size))

    def loss_of(theta, frac, n_re, n_im):
        m_re = n_re[:, :, None].expand(-1, -1, wl.size)
        m_im = n_im[:, :, None].expand(-1, -1, wl.size)
        v, _, g = autograd.ensemble_fixed_layered(theta, frac, m_re, m_im, kind="lognormal",
                                                  ranges=ranges, wavelengths=wl, n_nodes=48,
                                                  greek_order=16)
        rows = torch.cat([v[[0, 4, 5]], g[0, :, :16].transpose(0, 1)], dim=0)
        t = torch.from_numpy(targets).to(rows)
        return ((rows / t - 1.0) ** 2).sum()

    base = [torch.tensor(d["param"][:, :2].copy(), dtype=torch.float64),
            torch.tensor(fr.copy(), dtype=torch.float64),
            torch.tensor(ml[:, :, 0].real.copy(), dtype=torch.float64),
            torch.tensor(ml[:, :, 0].imag.copy(), dtype=torch.float64)]
    ml[:, :, 1] = ml[:, :, 0]  # one index per (distribution, layer) at both wavelengths
    params = [b.clone().requires_grad_(True) for b in base]
    loss = loss_of(*params)
    loss.backward()
    for which, p in enumerate(params):
        flat = p.grad.reshape(-1)
        for idx in range(flat.numel()):
            x0 = max(abs(float(base[which].reshape(-1)[idx])), 1e-3)

            def central(h):
                vals = []
                for sign in (1, -1):
                    args = [b.clone() for b in base]
                    args[which].view(-1)[idx] += sign * h
                    with torch.no_grad():
                        vals.append(float(loss_of(*args)))
                return (vals[0] - vals[1]) / (2 * h)

            fd = (4.0 * central(5e-5 * x0) - central(1e-4 * x0)) / 3.0
            assert abs(float(flat[idx]) - fd) <= 1e-6 * max(abs(fd), 1e-3 * abs(loss.item())), (
                which, idx, float(flat[idx]), fd)


def test_fixed_binding_selects_the_layered_blocks(gpu):
    """_scatrs.ensemble_compute_fixed with derivatives of a layered sphere: the blocks of
    scatrs_ensemble_fixed_layered_d in ensemble_parameters' order, selected by index."""
    from scatrs_b200 import _scatrs

    wl = np.array([0.5, 0.8])
    fr = np.array([0.6, 0.9])
    ml = np.array([[1.8 + 0.1j, 1.8 + 0.1j], [1.5 + 0.01j, 1.5 + 0.01j],
                   [1.34 + 1e-4j, 1.33 + 1e-4j]])
    spec = ("lognormal", 0.15, 1.5)
    names = _scatrs.ensemble_parameters([(spec, ("layered", fr, ml), 1.0)], False)
    assert names[:4] == ["median_radius", "width", "layer0.m_real", "layer0.m_imag"]
    assert names[-2:] == ["layer0.radius_fraction", "layer1.radius_fraction"]
    pick = [1, names.index("layer1.m_imag"), names.index("layer1.radius_fraction")]
    out = _scatrs.ensemble_compute_fixed([spec], ("layered", fr, ml), wl, 8, False, MU, True,
                                         n_nodes=48, spread=3.0, derivatives=pick)
    d = np.zeros(1, dtype=_native.DIST_DTYPE)
    d["kind"] = 1
    d["param"][0, :2] = (0.15, 1.5)
    d["r_lo"], d["r_hi"] = 0.15 * 1.5 ** -3, 0.15 * 1.5 ** 3
    ref = gpu.ensemble_fixed_layered_d(d, wl, fr[None], ml[None], MU, 48, 8)
    assert np.array_equal(out["values"], ref[0])
    assert np.array_equal(out["d"], ref[3][pick])
    assert np.array_equal(out["greek_d"], ref[5][pick])
    assert np.array_equal(out["phase_d"], ref[4][pick])
