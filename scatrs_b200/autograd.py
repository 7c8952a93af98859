"""Gradients of the fixed-grid ensemble for torch: torch.autograd.Functions whose forward pass
is one scatrs_ensemble_fixed_d (or _layered_d) call -- values and their forward-mode
derivatives along the distribution parameters, the refractive indices and the radius
fractions, all on the GPU -- and whose backward pass contracts the incoming gradients with
those derivatives (J^T g) in torch, on the same device.

With CUDA tensors the inputs, outputs and Jacobians stay in device memory: the forward pass
calls the *_device entry points with the tensors' storage, and only the distribution
parameters, the radius fractions and the cosines (a few doubles each) reach the host to build
the size grid. CPU tensors take the host-buffer entry points (the computation is on the GPU
either way).

With at most a handful of directions per unit (3 distribution parameters, Re m, Im m per layer,
the fractions) the forward-mode blocks cost about one extra GEMM tile per block on the GPU, so
no separate adjoint pass is run; the reference returns the same forward-mode Jacobians from
`derivatives=` (scatrs/src/ensemble/mod.rs:515-521).

`refractive_index` makes m(lambda) from a refractive-index model on the device
(python/scatrs/refractive.py: Constant, Cauchy, Sellmeier, with their parameters
differentiable), so that gradients reach a model's parameters through m.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _native

# The rows of `values` (python/scatrs/ensemble.py:51-63).
SCALARS = ("c_ext", "c_sca", "c_abs", "c_back", "ssa", "g", "lidar_ratio", "depolarization",
           "effective_radius", "mean_area", "mean_volume")


def named(values: torch.Tensor) -> dict:
    """The rows of an ensemble's values (11, n) by the reference's names."""
    return {name: values[k] for k, name in enumerate(SCALARS)}


def _theta_count(dists) -> int:
    return {3: 3, 4: 1, _native.TABULATED: 0}.get(int(dists["kind"][0]), 2) if dists.size else 2


def _outputs(n, n_mu, L, P, dev):
    """values, phase, greek and their P derivative blocks, zero-sized where not requested."""
    f64 = dict(dtype=torch.float64, device=dev)
    v = torch.empty(11, n, **f64)
    ph = torch.empty(6, n, n_mu, **f64) if n_mu else torch.empty(0, **f64)
    g = torch.empty(6, n, L + 1, **f64) if L >= 0 else torch.empty(0, **f64)
    dv = torch.empty(P, 11, n, **f64)
    dph = torch.empty(P, 6, n, n_mu, **f64) if n_mu else None
    dg = torch.empty(P, 6, n, L + 1, **f64) if L >= 0 else None
    return v, ph, g, dv, dph, dg


def _ptr(t):
    return 0 if t is None or t.numel() == 0 else t.data_ptr()


def _contract(grads, jacs):
    """sum over every output of one unit of J^T g: (P, n_units)."""
    total = None
    for grad, jac in zip(grads, jacs):
        if jac is None or grad is None or grad.numel() == 0:
            continue
        g = grad.to(jac.dtype)
        dims = [k for k in range(g.dim()) if k != 1]
        contrib = (jac * g.unsqueeze(0)).sum(dim=[k + 1 for k in dims])
        total = contrib if total is None else total + contrib
    return total


class _FixedEnsemble(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, m_re, m_im, spec):
        dists, wl, mu, n_nodes, greek_order, normalized, allow = spec
        d = dists.copy()
        n_th = _theta_count(d)
        d["param"][:, :n_th] = theta.detach().to("cpu", torch.float64).numpy()
        dev = m_re.device
        P = n_th + 2
        n = d.size * wl.size
        if dev.type == "cuda":
            m = torch.complex(m_re.detach().to(torch.float64), m_im.detach().to(torch.float64))
            m = torch.view_as_real(m.contiguous()).contiguous()
            wl_d = torch.as_tensor(wl, dtype=torch.float64, device=dev)
            outs = _outputs(n, mu.size, greek_order, P, dev)
            stream = torch.cuda.current_stream(dev).cuda_stream
            _native.ensemble_fixed_d_device(d, wl_d.data_ptr(), wl.size, m.data_ptr(), mu,
                                            n_nodes, greek_order, normalized,
                                            [_ptr(t) for t in outs], stream, allow)
            v, ph, g, dv, dph, dg = outs
        else:
            m = (m_re.detach().to(torch.float64).numpy()
                 + 1j * m_im.detach().to(torch.float64).numpy())
            res = _native.ensemble_fixed_d(d, wl, m, mu, n_nodes, greek_order, normalized, allow)
            empty = torch.zeros(0, dtype=torch.float64)
            v, ph, g = (torch.from_numpy(a) if a is not None else empty for a in res[:3])
            dv, dph, dg = (torch.from_numpy(a) if a is not None else None for a in res[3:])
        ctx.n_dist, ctx.n_wl, ctx.n_th = d.size, wl.size, n_th
        ctx.jac = (dv, dph, dg)
        return v, ph, g

    @staticmethod
    def backward(ctx, gv, gph, gg):
        total = _contract((gv, gph, gg), ctx.jac)
        if total is None:
            return None, None, None, None
        n_th = ctx.n_th
        per_unit = total.reshape(total.shape[0], ctx.n_dist, ctx.n_wl)
        g_theta = per_unit[:n_th].sum(dim=2).transpose(0, 1)   # (n_dist, n_th)
        g_re, g_im = per_unit[n_th], per_unit[n_th + 1]         # (n_dist, n_wl)
        return g_theta, g_re, g_im, None


def _grid(kind, ranges):
    if kind not in _native.KINDS:
        raise TypeError(f"unknown distribution kind {kind!r}")
    ranges = np.asarray(ranges, dtype=np.float64).reshape(-1, 2)
    d = np.zeros(ranges.shape[0], dtype=_native.DIST_DTYPE)
    d["kind"] = _native.KINDS[kind]
    d["r_lo"], d["r_hi"] = ranges[:, 0], ranges[:, 1]
    if kind == "power_law":
        d["param"][:, 1], d["param"][:, 2] = ranges[:, 0], ranges[:, 1]
    return d


def ensemble_fixed(theta: torch.Tensor, m_re: torch.Tensor, m_im: torch.Tensor, *, kind: str,
                   ranges, wavelengths, mu=None, n_nodes: int = 256, greek_order: int = -1,
                   normalized: bool = True, allow_unvalidated: bool = False):
    """Differentiable fixed-grid ensemble of homogeneous spheres.

    ``theta`` (n_dist, P) holds each distribution's parameters in ensemble_parameters order
    (lognormal: median_radius, width; gamma: effective_radius, effective_variance; modified
    gamma: alpha, b, gamma; power law: exponent, with its range in ``ranges``), ``m_re``,
    ``m_im`` (n_dist, n_wl) the index per distribution and wavelength, ``ranges`` (n_dist, 2)
    the fixed grid [r_lo, r_hi] (for a power law also its [min_radius, max_radius]). Returns
    (values (11, n), phase (6, n, n_mu), greek (6, n, L + 1)) as float64 tensors on m_re's
    device (kept there, with the Jacobians, when it is a CUDA device), empty where not
    requested; gradients flow to theta, m_re and m_im."""
    d = _grid(kind, ranges)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    spec = (d, wl, mu, int(n_nodes), int(greek_order), bool(normalized), bool(allow_unvalidated))
    return _FixedEnsemble.apply(theta, m_re, m_im, spec)


class _SpheroidEnsemble(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, aspect_ratio, m_re, m_im, spec):
        dists, wl, mu, n_nodes, greek_order, normalized, rtol = spec
        d = dists.copy()
        n_th = _theta_count(d)
        d["param"][:, :n_th] = theta.detach().to("cpu", torch.float64).numpy()
        dev = m_re.device
        m = (m_re.detach().to("cpu", torch.float64).numpy()
             + 1j * m_im.detach().to("cpu", torch.float64).numpy())
        eps = aspect_ratio.detach().to("cpu", torch.float64).numpy()
        res = _native.ensemble_fixed_spheroid_d(d, wl, eps, m, mu, n_nodes, greek_order,
                                                normalized, rtol)
        empty = torch.zeros(0, dtype=torch.float64, device=dev)
        v, ph, g = (torch.from_numpy(a).to(dev) if a is not None else empty for a in res[:3])
        ctx.jac = tuple(torch.from_numpy(a).to(dev) if a is not None else None
                        for a in res[3:6])
        ctx.n_dist, ctx.n_wl, ctx.n_th = d.size, wl.size, n_th
        return v, ph, g

    @staticmethod
    def backward(ctx, gv, gph, gg):
        total = _contract((gv, gph, gg), ctx.jac)
        if total is None:
            return None, None, None, None, None
        n_th = ctx.n_th
        per_unit = total.reshape(total.shape[0], ctx.n_dist, ctx.n_wl)
        g_theta = per_unit[:n_th].sum(dim=2).transpose(0, 1)   # (n_dist, n_th)
        g_eps = per_unit[n_th].sum(dim=1)                      # (n_dist,)
        g_re, g_im = per_unit[n_th + 1], per_unit[n_th + 2]     # (n_dist, n_wl)
        return g_theta, g_eps, g_re, g_im, None


def ensemble_fixed_spheroid(theta: torch.Tensor, aspect_ratio: torch.Tensor, m_re: torch.Tensor,
                            m_im: torch.Tensor, *, kind: str, ranges, wavelengths, mu=None,
                            n_nodes: int = 64, greek_order: int = -1, normalized: bool = True,
                            tmatrix_rtol: float = 1e-8):
    """Differentiable fixed-grid ensemble of randomly oriented spheroids.

    ``theta`` (n_dist, P) the distributions' parameters (as ensemble_fixed's), ``aspect_ratio``
    (n_dist,) each distribution's spheroid aspect ratio, ``m_re``, ``m_im`` (n_dist, n_wl) the
    index, ``ranges`` (n_dist, 2) the fixed grid of volume-equivalent radii. Returns (values,
    phase, greek) as ensemble_fixed does; gradients flow to theta, aspect_ratio, m_re and m_im
    (scatrs_ensemble_fixed_spheroid_d: each node's solution differentiated at its converged N
    and n_theta, the averages and ratios in forward mode)."""
    d = _grid(kind, ranges)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    spec = (d, wl, mu, int(n_nodes), int(greek_order), bool(normalized), float(tmatrix_rtol))
    return _SpheroidEnsemble.apply(theta, aspect_ratio, m_re, m_im, spec)


class _LayeredEnsemble(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, fractions, m_re, m_im, spec):
        dists, wl, mu, n_nodes, greek_order, normalized, allow = spec
        d = dists.copy()
        n_th = _theta_count(d)
        d["param"][:, :n_th] = theta.detach().to("cpu", torch.float64).numpy()
        fr = fractions.detach().to("cpu", torch.float64).numpy()
        L = m_re.shape[1]
        P = n_th + 3 * L - 1
        n = d.size * wl.size
        dev = m_re.device
        if dev.type == "cuda":
            m = torch.complex(m_re.detach().to(torch.float64), m_im.detach().to(torch.float64))
            m = torch.view_as_real(m.contiguous()).contiguous()
            wl_d = torch.as_tensor(wl, dtype=torch.float64, device=dev)
            outs = _outputs(n, mu.size, greek_order, P, dev)
            stream = torch.cuda.current_stream(dev).cuda_stream
            _native.ensemble_fixed_layered_d_device(d, wl_d.data_ptr(), wl.size, fr, L,
                                                    m.data_ptr(), mu, n_nodes, greek_order,
                                                    normalized, [_ptr(t) for t in outs], stream,
                                                    allow)
            v, ph, g, dv, dph, dg = outs
        else:
            m = (m_re.detach().to(torch.float64).numpy()
                 + 1j * m_im.detach().to(torch.float64).numpy())
            res = _native.ensemble_fixed_layered_d(d, wl, fr, m, mu, n_nodes, greek_order,
                                                   normalized, allow)
            empty = torch.zeros(0, dtype=torch.float64)
            v, ph, g = (torch.from_numpy(a) if a is not None else empty for a in res[:3])
            dv, dph, dg = (torch.from_numpy(a) if a is not None else None for a in res[3:])
        ctx.n_dist, ctx.n_wl, ctx.n_th, ctx.n_layers = d.size, wl.size, n_th, L
        ctx.jac = (dv, dph, dg)
        return v, ph, g

    @staticmethod
    def backward(ctx, gv, gph, gg):
        total = _contract((gv, gph, gg), ctx.jac)
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
    d = _grid(kind, ranges)
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    spec = (d, wl, mu, int(n_nodes), int(greek_order), bool(normalized), bool(allow_unvalidated))
    return _LayeredEnsemble.apply(theta, fractions, m_re, m_im, spec)


class _RefractiveIndex(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, kind, wl_d, wl_host):
        dev = wl_d.device
        rows = params.detach().to("cpu", torch.float64).numpy()
        specs = [_model_spec(kind, row) for row in rows]
        P = params.shape[1]
        m = torch.empty(len(specs), wl_host.size, 2, dtype=torch.float64, device=dev)
        dm = torch.empty(len(specs), P, wl_host.size, 2, dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _native.refractive_index_device(specs, wl_d.data_ptr(), wl_host.size, m.data_ptr(),
                                        dm.data_ptr(), P, stream)
        ctx.save_for_backward(dm)
        return m[..., 0].contiguous(), m[..., 1].contiguous()

    @staticmethod
    def backward(ctx, g_re, g_im):
        (dm,) = ctx.saved_tensors
        grad = torch.zeros(dm.shape[:2], dtype=torch.float64, device=dm.device)
        if g_re is not None:
            grad = grad + (dm[..., 0] * g_re.unsqueeze(1)).sum(dim=2)
        if g_im is not None:
            grad = grad + (dm[..., 1] * g_im.unsqueeze(1)).sum(dim=2)
        return grad, None, None, None


def _model_spec(kind, row):
    if kind == "constant":
        return ("constant", complex(row[0], row[1]))
    if kind == "cauchy":
        return ("cauchy", row[0], row[1], row[2], row[3])
    if kind == "sellmeier":
        t = (row.size - 1) // 2
        return ("sellmeier", row[:t], row[t:2 * t], row[2 * t])
    raise TypeError(f"no differentiable refractive-index model {kind!r} (constant, cauchy, "
                    "sellmeier)")


def refractive_index(kind: str, params: torch.Tensor, wavelengths):
    """m(lambda) of n_models refractive-index models of one kind on the device, differentiable
    along their parameters: ``params`` (n_models, P) in the reference's `parameters` order
    (constant: n, k; cauchy: A, B, C, k; sellmeier: B_0.., C_0.., k; refractive.py:168-354).
    Returns (m_re, m_im), each (n_models, n_wl), on params' device (a CUDA device)."""
    wl = np.ascontiguousarray(wavelengths, dtype=np.float64).reshape(-1)
    wl_d = torch.as_tensor(wl, dtype=torch.float64, device=params.device)
    return _RefractiveIndex.apply(params, kind, wl_d, wl)
