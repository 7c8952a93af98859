"""The fixed-grid ensemble through the C ABI against the oracle's restatement of the reference's
pass 2, averages, band projection and assembly, on the same seeded inputs.

Tolerances: the Mie coefficients agree to rounding (test_gpu_mie); the sums over orders (the
angle GEMMs) and over nodes run in a different order from the oracle's, with FMA, so the
outputs agree to rounding of those sums: 1e-12 relative for the scalars, 1e-12 of max F11 for
the phase matrix (the reference pins its own band products to 1e-12 of the largest value,
scatrs/src/ensemble/fast.rs:342-350), and 1e-12 (alpha1_0 = 1) for the Greek coefficients.
"""

import numpy as np
import pytest

from oracle import oracle as O
from scatrs_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _oracle(w: W.Workload, mu=None, greek=None, normalized=True, threads=0):
    d = np.zeros(w.dists.size, dtype=O.DIST_DTYPE)
    d["kind"] = w.dists["kind"]
    d["p"] = w.dists["param"]
    d["r_lo"] = w.dists["r_lo"]
    d["r_hi"] = w.dists["r_hi"]
    return O.ensemble_fixed(d, w.wavelengths, w.m, w.n_nodes, w.mu if mu is None else mu,
                            w.greek_order if greek is None else greek, normalized,
                            threads=threads)


def _compare(got, ref, tol=TOL):
    v, ph, g = got
    # scalars: relative, c_back against max(c_back, c_sca) as the reference measures it
    rv = ref["values"]
    scale = np.abs(rv).copy()
    scale[3] = np.maximum(scale[3], np.abs(rv[1]))
    scale[6] = np.maximum(scale[6], 1e-300)
    err = np.abs(v - rv) / np.maximum(scale, 1e-300)
    err[7] = np.abs(v[7] - rv[7])
    assert err.max() <= tol, (np.unravel_index(err.argmax(), err.shape), err.max())
    if ph is not None:
        rp = ref["phase"]
        size = np.abs(rp[0]).max(axis=1, keepdims=True)
        e = np.abs(ph - rp) / size[None]
        assert e.max() <= tol, (np.unravel_index(e.argmax(), e.shape), e.max())
    if g is not None:
        rg = ref["greek"]
        size = np.abs(rg[0]).max(axis=1, keepdims=True)
        e = np.abs(g - rg) / size[None]
        assert e.max() <= tol, (np.unravel_index(e.argmax(), e.shape), e.max())


def test_small_spheres_matches_oracle(gpu):
    w = W.small_spheres()
    got = gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, w.greek_order)
    _compare(got, _oracle(w))
    v, ph, g = got
    assert np.all(g[0, :, 0] == 1.0)


def test_batched_shape_small_matches_oracle(gpu):
    w = W.batched_spheres(seed=3, scale=0.04)  # 3 distributions x 41 wavelengths, x up to ~1000
    w.mu = W.gauss_legendre(64)
    got = gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, w.greek_order)
    _compare(got, _oracle(w))


@pytest.mark.parametrize("n_nodes", [1, 7, 33, 100])
def test_ragged_chunks(gpu, n_nodes):
    w = W.small_spheres()
    w.n_nodes = n_nodes
    w.mu = np.array([1.0, 0.3, -0.3, 0.0, -1.0, 0.77])  # unpaired and paired cosines
    got = gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, 12)
    _compare(got, _oracle(w, greek=12))


def test_real_index_unnormalized_no_outputs(gpu):
    w = W.small_spheres()
    w.m = np.full_like(w.m, 1.5 + 0j)
    got = gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, None, w.n_nodes, -1, normalized=False)
    assert got[1] is None and got[2] is None
    ref = _oracle(w, mu=np.zeros(0), greek=-1, normalized=False)
    _compare(got, ref)
    assert np.all(got[0][2] == 0.0)  # c_abs exactly 0 for real m
    got = gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, 20, normalized=False)
    _compare(got, _oracle(w, greek=20, normalized=False))


def test_phase_normalization_and_greek_consistency(gpu):
    """Normalized: 1/2 sum w F11 = 1 on a Gauss grid that integrates exactly, and alpha1_1 = 3g."""
    w = W.small_spheres()
    mu, wt = gpu.gauss_legendre(200)
    v, ph, g = gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, mu, w.n_nodes, 32)
    norm = 0.5 * (ph[0] * wt[None]).sum(axis=1)
    assert np.allclose(norm, 1.0, rtol=1e-12, atol=0)
    assert np.allclose(g[0, :, 1], 3 * v[5], rtol=1e-11, atol=0)


def test_errors(gpu):
    from scatrs_b200.errors import InvalidInputError, OutsideValidatedDomainError

    w = W.small_spheres()
    with pytest.raises(OutsideValidatedDomainError, match="at wavelength"):
        gpu.ensemble_fixed(w.dists, w.wavelengths, np.full_like(w.m, 1.5 + 11j), w.mu,
                           w.n_nodes, 8)
    with pytest.raises(InvalidInputError):
        gpu.ensemble_fixed(w.dists, w.wavelengths, np.full_like(w.m, -1.5 + 0j), w.mu,
                           w.n_nodes, 8)
    with pytest.raises(InvalidInputError):
        gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, np.array([1.5]), w.n_nodes, 8)
    bad = w.dists.copy()
    bad["param"][0, 1] = 0.5
    with pytest.raises(InvalidInputError, match="width"):
        gpu.ensemble_fixed(bad, w.wavelengths, w.m, w.mu, w.n_nodes, 8)
    # allowed outside the domain
    v, _, _ = gpu.ensemble_fixed(w.dists, w.wavelengths, np.full_like(w.m, 1.5 + 11j), None,
                                 w.n_nodes, -1, allow_unvalidated=True)
    assert np.all(np.isfinite(v))


def test_deterministic_and_empty(gpu):
    w = W.batched_spheres(seed=1, scale=0.02)
    w.mu = W.gauss_legendre(32)
    a = gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, 16)
    b = gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, 16)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    v, p, g = gpu.ensemble_fixed(w.dists[:0], w.wavelengths, w.m[:0], w.mu, w.n_nodes, 16)
    assert v.shape == (11, 0) and p.shape == (6, 0, w.mu.size) and g.shape == (6, 0, 17)


def _oracle_layered(w, **kw):
    d = np.zeros(w.dists.size, dtype=O.DIST_DTYPE)
    d["kind"], d["p"] = w.dists["kind"], w.dists["param"]
    d["r_lo"], d["r_hi"] = w.dists["r_lo"], w.dists["r_hi"]
    return O.ensemble_fixed_layered(d, w.wavelengths, w.fractions, w.m_layers, w.n_nodes, w.mu,
                                    w.greek_order, **kw)


def test_layered_matches_oracle(gpu):
    w = W.layered_spheres(seed=2, scale=0.03)  # 8 distributions x 4 wavelengths of three-layer spheres
    got = gpu.ensemble_fixed_layered(w.dists, w.wavelengths, w.fractions, w.m_layers, w.mu,
                                     w.n_nodes, w.greek_order)
    _compare(got, _oracle_layered(w), tol=1e-11)


def test_layered_with_equal_indices_is_the_sphere(gpu):
    """One index in every layer: the sphere's results bit for bit (tests/ensemble_layered.rs:
    62-116 of the reference)."""
    w = W.small_spheres()
    ml = np.repeat(w.m[:, None, :], 3, axis=1)
    fr = np.array([[0.4, 0.8]])
    got = gpu.ensemble_fixed_layered(w.dists, w.wavelengths, fr, ml, w.mu, w.n_nodes, 16)
    ref = gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, 16)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


def test_pinned_outputs_are_copied_per_slab(gpu):
    """Pinned host outputs are copied slab by slab on a second stream beside the later slabs'
    kernels; the results are the same bits as the copies at the end (pageable outputs), on a
    workload of several slabs."""
    import ctypes

    import torch

    from scatrs_b200 import _native as N

    w = W.batched_spheres(scale=0.5)
    values, phase, greek = N.ensemble_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes,
                                            w.greek_order)
    n = w.n_units
    pv = torch.zeros(11 * n, dtype=torch.float64).pin_memory()
    pp = torch.zeros(6 * n * w.mu.size, dtype=torch.float64).pin_memory()
    pg = torch.zeros(6 * n * (w.greek_order + 1), dtype=torch.float64).pin_memory()
    dists = np.ascontiguousarray(w.dists, dtype=N.DIST_DTYPE)
    wl = np.ascontiguousarray(w.wavelengths, dtype=np.float64)
    m = np.ascontiguousarray(np.broadcast_to(w.m, (dists.size, wl.size)), dtype=np.complex128)
    mu = np.ascontiguousarray(w.mu, dtype=np.float64)
    opts = N.FixedOptions(w.n_nodes, w.greek_order, 1, 0)
    err = ctypes.create_string_buffer(1024)
    st = N.load().scatrs_ensemble_fixed(dists.ctypes.data, dists.size, N._p(wl), wl.size,
                                        N._p(m.view(np.float64)), N._p(mu), mu.size,
                                        ctypes.byref(opts), ctypes.cast(pv.data_ptr(), N._PD),
                                        ctypes.cast(pp.data_ptr(), N._PD),
                                        ctypes.cast(pg.data_ptr(), N._PD), err, 1024)
    assert st == 0, err.value
    assert np.array_equal(pv.numpy().reshape(values.shape), values)
    assert np.array_equal(pp.numpy().reshape(phase.shape), phase)
    assert np.array_equal(pg.numpy().reshape(greek.shape), greek)


def _sub(w, dist_idx, wl_idx):
    """The units (dist_idx x wl_idx) of a workload, at its own shape (nodes, cosines, order)."""
    dist_idx, wl_idx = np.atleast_1d(dist_idx), np.atleast_1d(wl_idx)
    return W.Workload(w.name + "[sub]", w.dists[dist_idx], w.wavelengths[wl_idx],
                      w.m[np.ix_(dist_idx, wl_idx)], w.mu, w.n_nodes, w.greek_order)


def test_batched_full_shape_largest_n_units(gpu):
    """The batched workload at its real shape (512 nodes, 360 Gauss cosines, order 64) on its
    units of largest N (the widest lognormal at the shortest wavelengths: N up to 2198) and on
    units of a middle and a small distribution."""
    w = W.batched_spheres(seed=0)
    assert w.mu.size == 360 and w.n_nodes == 512 and w.greek_order == 64
    top = int(np.argmax(w.dists["r_hi"]))
    sub = _sub(w, top, [0, 1, 2, 3, 700, 1023])
    x = 2 * np.pi * sub.dists["r_hi"][0] / sub.wavelengths[0]
    assert np.ceil(x + 6 * np.cbrt(x) + 3) >= 2190
    got = gpu.ensemble_fixed(sub.dists, sub.wavelengths, sub.m, sub.mu, sub.n_nodes,
                             sub.greek_order)
    _compare(got, _oracle(sub, threads=0))
    order = np.argsort(w.dists["r_hi"])
    sub = _sub(w, [int(order[0]), int(order[w.dists.size // 2])], [0, 333, 1023])
    got = gpu.ensemble_fixed(sub.dists, sub.wavelengths, sub.m, sub.mu, sub.n_nodes,
                             sub.greek_order)
    _compare(got, _oracle(sub, threads=0))


def test_layered_full_shape_units(gpu):
    """The layered workload at its real shape (three layers, 256 nodes, order 32) on full-size
    units: its two widest distributions at its shortest and longest wavelengths."""
    w = W.layered_spheres(seed=0)
    top = np.argsort(w.dists["r_hi"])[-2:]
    wl_idx = np.array([0, w.wavelengths.size - 1])
    sub = W.LayeredWorkload(w.name + "[sub]", w.dists[top], w.wavelengths[wl_idx],
                            w.fractions[top], w.m_layers[np.ix_(top, np.arange(3), wl_idx)],
                            w.mu, w.n_nodes, w.greek_order)
    got = gpu.ensemble_fixed_layered(sub.dists, sub.wavelengths, sub.fractions, sub.m_layers,
                                     sub.mu, sub.n_nodes, sub.greek_order)
    _compare(got, _oracle_layered(sub), tol=1e-11)
