"""Gradients through scatrs_b200.autograd (forward-mode Jacobians from the GPU, contracted in
the backward pass) against central finite differences of the same GPU forward pass, step 1e-6
relative, for a loss shaped like the layered benchmark's: a weighted squared difference of
c_ext, ssa, g and alpha1_0..15 against seeded targets. Agreement: 1e-6 relative (norm-wise and
per component against the largest component)."""

import numpy as np
import pytest
import torch

from scatrs_b200 import autograd as A
from scatrs_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _setup():
    rng = np.random.default_rng(11)
    n_dist, n_wl = 3, 4
    med = rng.uniform(0.08, 0.4, n_dist)
    wid = rng.uniform(1.3, 1.8, n_dist)
    wl = np.geomspace(0.4, 1.2, n_wl)
    m = rng.uniform(1.35, 1.6, (n_dist, n_wl)) + 1j * np.exp(rng.uniform(-9, -2, (n_dist, n_wl)))
    ranges = np.stack([med * wid ** -4.0, med * wid ** 4.0], axis=1)
    targets = rng.uniform(0.5, 1.5, 3 + 16)
    return med, wid, wl, m, ranges, targets


def test_gradients_match_central_differences():
    med, wid, wl, m, ranges, targets = _setup()
    dev = "cuda"
    theta = torch.tensor(np.stack([med, wid], axis=1), dtype=torch.float64, device=dev,
                         requires_grad=True)
    m_re = torch.tensor(m.real, dtype=torch.float64, device=dev, requires_grad=True)
    m_im = torch.tensor(m.imag, dtype=torch.float64, device=dev, requires_grad=True)
    # c_ext normalized by a constant so that the loss is smooth in every parameter.
    scale = None

    def f(th, re, im):
        nonlocal scale
        v, ph, g = A.ensemble_fixed(th, re, im, kind="lognormal", ranges=ranges,
                                    wavelengths=wl, mu=np.array([0.9, -0.2]), n_nodes=96,
                                    greek_order=20)
        if scale is None:
            scale = float(v[0].detach().mean())
        loss = ((v[0] / scale - targets[0]) ** 2).sum()
        loss = loss + ((v[4] - targets[1]) ** 2).sum() + ((v[5] - targets[2]) ** 2).sum()
        a1 = g[0, :, :16]
        loss = loss + ((a1 - torch.as_tensor(targets[3:], device=a1.device)[None]) ** 2).sum()
        return loss + 1e-3 * (ph[0] ** 2).sum()

    loss = f(theta, m_re, m_im)
    loss.backward()
    grads = [theta.grad.cpu().numpy(), m_re.grad.cpu().numpy(), m_im.grad.cpu().numpy()]
    base = [theta.detach().clone(), m_re.detach().clone(), m_im.detach().clone()]
    h = 1e-6
    for which, g_ad in enumerate(grads):
        fd = np.zeros_like(g_ad)
        for idx in np.ndindex(g_ad.shape):
            args_p = [b.clone() for b in base]
            args_m = [b.clone() for b in base]
            x0 = float(base[which][idx])
            step = h * abs(x0)
            args_p[which][idx] = x0 + step
            args_m[which][idx] = x0 - step
            with torch.no_grad():
                fd[idx] = (float(f(*args_p)) - float(f(*args_m))) / (2 * step)
        err = np.abs(g_ad - fd)
        assert np.linalg.norm(g_ad - fd) <= 1e-6 * np.linalg.norm(fd), (which, err.max())
        assert err.max() <= 1e-6 * np.abs(fd).max() + 1e-9 * np.abs(g_ad).max(), which


def test_device_path_equals_the_host_entry():
    """With CUDA tensors the forward pass runs scatrs_ensemble_fixed_d_device on the tensors'
    storage (no host round trip): the same bits as the host-buffer entry point, outputs and
    Jacobians left on the device."""
    from scatrs_b200 import _native as N

    med, wid, wl, m, ranges, _ = _setup()
    theta = torch.tensor(np.stack([med, wid], axis=1), dtype=torch.float64, device="cuda")
    re = torch.tensor(m.real, dtype=torch.float64, device="cuda", requires_grad=True)
    im = torch.tensor(m.imag, dtype=torch.float64, device="cuda")
    mu = np.array([0.9, -0.2, 0.35])
    v, ph, g = A.ensemble_fixed(theta, re, im, kind="lognormal", ranges=ranges, wavelengths=wl,
                                mu=mu, n_nodes=64, greek_order=12)
    assert v.is_cuda and ph.is_cuda and g.is_cuda
    d = np.zeros(med.size, dtype=N.DIST_DTYPE)
    d["kind"] = N.KINDS["lognormal"]
    d["param"][:, 0], d["param"][:, 1] = med, wid
    d["r_lo"], d["r_hi"] = ranges[:, 0], ranges[:, 1]
    ref = N.ensemble_fixed_d(d, wl, m, mu, 64, 12)
    for got, want in zip((v, ph, g), ref[:3]):
        assert np.array_equal(got.detach().cpu().numpy(), want)
    (v[0].sum() + g[0, :, 3].sum()).backward()
    assert re.grad.is_cuda
    want_grad = ref[3][2, 0].reshape(med.size, wl.size) + ref[5][2, 0, :, 3].reshape(
        med.size, wl.size)
    np.testing.assert_allclose(re.grad.cpu().numpy(), want_grad, rtol=1e-14, atol=0)


def test_gradient_through_a_cauchy_model():
    """m(lambda) from Cauchy's law on the device (refractive_index), its parameters
    differentiable through the ensemble: the gradient of a loss against Richardson-extrapolated
    central differences, 1e-6 relative."""
    med, wid, wl, _, ranges, targets = _setup()
    theta = torch.tensor(np.stack([med, wid], axis=1), dtype=torch.float64, device="cuda")
    params = torch.tensor([[1.45, 4.2e-3, 1.1e-4, 2e-4], [1.52, 3.0e-3, 0.0, 1e-5],
                           [1.38, 5.0e-3, 2.0e-5, 3e-3]], dtype=torch.float64, device="cuda")

    def loss_of(p):
        re, im = A.refractive_index("cauchy", p, wl)
        v, _, g = A.ensemble_fixed(theta, re, im, kind="lognormal", ranges=ranges,
                                   wavelengths=wl, n_nodes=64, greek_order=8)
        return ((v[4] - targets[1]) ** 2).sum() + ((g[0, :, 1] / 3 - targets[2]) ** 2).sum()

    p = params.clone().requires_grad_(True)
    loss_of(p).backward()
    grad = p.grad.cpu().numpy()
    for idx in np.ndindex(grad.shape):
        x0 = max(abs(float(params[idx])), 1e-4)

        def central(h):
            out = []
            for sign in (1, -1):
                q = params.clone()
                q[idx] += sign * h
                with torch.no_grad():
                    out.append(float(loss_of(q)))
            return (out[0] - out[1]) / (2 * h)

        fd = (4.0 * central(5e-5 * x0) - central(1e-4 * x0)) / 3.0
        assert abs(grad[idx] - fd) <= 1e-6 * max(abs(fd), 1e-6 * np.abs(grad).max()), (
            idx, grad[idx], fd)
