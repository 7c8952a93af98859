"""Gradients of the fixed-grid sphere ensemble for torch: a torch.autograd.Function whose
forward pass is one scatrs_ensemble_fixed_d call (values and their forward-mode derivatives
along the distribution parameters and Re m, Im m, all on the GPU) and whose backward pass
contracts the incoming gradients with those derivatives (J^T g).

With at most 5 directions per unit (3 distribution parameters, Re m, Im m) the forward-mode
blocks cost about one extra GEMM tile per block on the GPU, so no separate adjoint pass is run;
the reference returns the same forward-mode Jacobians from `derivatives=`
(scatrs/src/ensemble/mod.rs:515-521).
"""

from __future__ import annotations

import numpy as np
import torch

from . import _native


class _FixedEnsemble(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, m_re, m_im, spec):
        dists, wl, mu, n_nodes, greek_order, normalized, allow = spec
        d = dists.copy()
        n_th = {3: 3, 4: 1}.get(int(d["kind"][0]), 2) if d.size else 2
        d["param"][:, :n_th] = theta.detach().to("cpu", torch.float64).numpy()
        m = (m_re.detach().to("cpu", torch.float64).numpy()
             + 1j * m_im.detach().to("cpu", torch.float64).numpy())
        v, ph, g, dv, dph, dg = _native.ensemble_fixed_d(d, wl, m, mu, n_nodes, greek_order,
                                                         normalized, allow)
        dev = theta.device
        ctx.n_dist, ctx.n_wl, ctx.n_th = d.size, wl.size, n_th
        ctx.jac = [torch.from_numpy(a).to(dev) if a is not None else None for a in (dv, dph, dg)]
        empty = torch.zeros(0, dtype=torch.float64, device=dev)
        out = [torch.from_numpy(a).to(dev) if a is not None else empty for a in (v, ph, g)]
        return tuple(out)

    @staticmethod
    def backward(ctx, gv, gph, gg):
        # sum over every output of one unit: (P, n_units)
        total = None
        for grad, jac in zip((gv, gph, gg), ctx.jac):
            if jac is None or grad is None or grad.numel() == 0:
                continue
            # jac: (P, K, n, ...) and grad: (K, n, ...) -> (P, n)
            g = grad.to(jac.dtype)
            dims = [k for k in range(g.dim()) if k != 1]
            contrib = (jac * g.unsqueeze(0)).sum(dim=[k + 1 for k in dims])
            total = contrib if total is None else total + contrib
        n_th = ctx.n_th
        if total is None:
            return None, None, None, None
        per_unit = total.reshape(total.shape[0], ctx.n_dist, ctx.n_wl)
        g_theta = per_unit[:n_th].sum(dim=2).transpose(0, 1)   # (n_dist, n_th)
        g_re, g_im = per_unit[n_th], per_unit[n_th + 1]         # (n_dist, n_wl)
        return g_theta, g_re, g_im, None


def ensemble_fixed(theta: torch.Tensor, m_re: torch.Tensor, m_im: torch.Tensor, *, kind: str,
                   ranges, wavelengths, mu=None, n_nodes: int = 256, greek_order: int = -1,
                   normalized: bool = True, allow_unvalidated: bool = False):
    """Differentiable fixed-grid ensemble of homogeneous spheres.

    ``theta`` (n_dist, P) holds each distribution's parameters in ensemble_parameters order
    (lognormal: median_radius, width; gamma: effective_radius, effective_variance; modified
    gamma: alpha, b, gamma; power law: exponent, with its range in ``ranges``), ``m_re``,
    ``m_im`` (n_dist, n_wl) the index per distribution and wavelength, ``ranges`` (n_dist, 2)
    the fixed grid [r_lo, r_hi] (for a power law also its [min_radius, max_radius]). Returns
    (values (11, n), phase (6, n, n_mu), greek (6, n, L + 1)) as float64 tensors on theta's
    device, empty where not requested; gradients flow to theta, m_re and m_im."""
    if kind not in _native.KINDS:
        raise TypeError(f"unknown distribution kind {kind!r}")
    ranges = np.asarray(ranges, dtype=np.float64).reshape(-1, 2)
    d = np.zeros(ranges.shape[0], dtype=_native.DIST_DTYPE)
    d["kind"] = _native.KINDS[kind]
    d["r_lo"], d["r_hi"] = ranges[:, 0], ranges[:, 1]
    if kind == "power_law":
        d["param"][:, 1], d["param"][:, 2] = ranges[:, 0], ranges[:, 1]
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    spec = (d, wl, mu, int(n_nodes), int(greek_order), bool(normalized), bool(allow_unvalidated))
    return _FixedEnsemble.apply(theta, m_re, m_im, spec)


class _LayeredEnsemble(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, fractions, m_re, m_im, spec):
        dists, wl, mu, n_nodes, greek_order, normalized, allow = spec
        d = dists.copy()
        n_th = {3: 3, 4: 1}.get(int(d["kind"][0]), 2) if d.size else 2
        d["param"][:, :n_th] = theta.detach().to("cpu", torch.float64).numpy()
        fr = fractions.detach().to("cpu", torch.float64).numpy()
        m = (m_re.detach().to("cpu", torch.float64).numpy()
             + 1j * m_im.detach().to("cpu", torch.float64).numpy())
        v, ph, g, dv, dph, dg = _native.ensemble_fixed_layered_d(d, wl, fr, m, mu, n_nodes,
                                                                 greek_order, normalized, allow)
        dev = theta.device
        ctx.n_dist, ctx.n_wl, ctx.n_th, ctx.n_layers = d.size, wl.size, n_th, m.shape[1]
        ctx.jac = [torch.from_numpy(a).to(dev) if a is not None else None for a in (dv, dph, dg)]
        empty = torch.zeros(0, dtype=torch.float64, device=dev)
        return tuple(torch.from_numpy(a).to(dev) if a is not None else empty for a in (v, ph, g))

    @staticmethod
    def backward(ctx, gv, gph, gg):
        total = None
        for grad, jac in zip((gv, gph, gg), ctx.jac):
            if jac is None or grad is None or grad.numel() == 0:
                continue
            g = grad.to(jac.dtype)
            dims = [k for k in range(g.dim()) if k != 1]
            contrib = (jac * g.unsqueeze(0)).sum(dim=[k + 1 for k in dims])
            total = contrib if total is None else total + contrib
        if total is None:
            return None, None, None, None, None
        n_th, L = ctx.n_th, ctx.n_layers
        per_unit = total.reshape(total.shape[0], ctx.n_dist, ctx.n_wl)
        g_theta = per_unit[:n_th].sum(dim=2).transpose(0, 1)          # (n_dist, n_th)
        g_re = per_unit[n_th:n_th + 2 * L:2].transpose(0, 1)           # (n_dist, L, n_wl)
        g_im = per_unit[n_th + 1:n_th + 2 * L:2].transpose(0, 1)
        g_fr = per_unit[n_th + 2 * L:].sum(dim=2).transpose(0, 1)      # (n_dist, L - 1)
        return g_theta, g_fr, g_re, g_im, None


def ensemble_fixed_layered(theta: torch.Tensor, fractions: torch.Tensor, m_re: torch.Tensor,
                           m_im: torch.Tensor, *, kind: str, ranges, wavelengths, mu=None,
                           n_nodes: int = 256, greek_order: int = -1, normalized: bool = True,
                           allow_unvalidated: bool = False):
    """Differentiable fixed-grid ensemble of layered spheres (at least two layers): ``theta``
    (n_dist, P) as in ensemble_fixed, ``fractions`` (n_dist, L - 1) the layers' outer radii over
    the particle's, ``m_re``, ``m_im`` (n_dist, L, n_wl) each layer's index per wavelength.
    Returns (values, phase, greek) as ensemble_fixed; gradients flow to theta, fractions, m_re
    and m_im (scatrs_ensemble_fixed_layered_d's forward-mode blocks contracted with the incoming
    gradients)."""
    if kind not in _native.KINDS:
        raise TypeError(f"unknown distribution kind {kind!r}")
    ranges = np.asarray(ranges, dtype=np.float64).reshape(-1, 2)
    d = np.zeros(ranges.shape[0], dtype=_native.DIST_DTYPE)
    d["kind"] = _native.KINDS[kind]
    d["r_lo"], d["r_hi"] = ranges[:, 0], ranges[:, 1]
    if kind == "power_law":
        d["param"][:, 1], d["param"][:, 2] = ranges[:, 0], ranges[:, 1]
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    spec = (d, wl, mu, int(n_nodes), int(greek_order), bool(normalized), bool(allow_unvalidated))
    return _LayeredEnsemble.apply(theta, fractions, m_re, m_im, spec)
