"""The mixed form of the fixed-grid ensemble (scatrs_ensemble_fixed_mixed): the angle GEMMs of
the chunks with more than i8_above terms as exact int8 digit products on the tensor cores,
everything else FP64. Its stated tolerance is 1e-10 against the FP64 oracle: scalars relative,
the phase matrix relative to each unit's largest F11, the Greek coefficients relative to each
unit's largest alpha1 (= 1) -- the metrics of test_gpu_ensemble.py.

The scalars (cross sections, ratios) come from the Mie sums of K-a, which the mixed form keeps in
FP64, so they match the oracle to 1e-12 as in the plain form.
"""

import numpy as np
import pytest

from oracle import oracle as O
from scatrs_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _oracle(w, threads=0):
    d = np.zeros(w.dists.size, dtype=O.DIST_DTYPE)
    d["kind"], d["p"] = w.dists["kind"], w.dists["param"]
    d["r_lo"], d["r_hi"] = w.dists["r_lo"], w.dists["r_hi"]
    return O.ensemble_fixed(d, w.wavelengths, w.m, w.n_nodes, w.mu, w.greek_order, True,
                            threads=threads)


def _errors(got, ref):
    v, ph, g = got
    rv = ref["values"]
    scale = np.abs(rv).copy()
    scale[3] = np.maximum(scale[3], np.abs(rv[1]))
    ev = np.abs(v - rv) / np.maximum(scale, 1e-300)
    ev[7] = np.abs(v[7] - rv[7])
    out = {"values": float(ev.max())}
    if ph is not None:
        size = np.abs(ref["phase"][0]).max(axis=1, keepdims=True)
        out["phase"] = float((np.abs(ph - ref["phase"]) / size[None]).max())
    if g is not None:
        size = np.abs(ref["greek"][0]).max(axis=1, keepdims=True)
        out["greek"] = float((np.abs(g - ref["greek"]) / size[None]).max())
    return out


def _sub(w, dist_idx, wl_idx):
    dist_idx, wl_idx = np.atleast_1d(dist_idx), np.atleast_1d(wl_idx)
    return W.Workload(w.name + "[sub]", w.dists[dist_idx], w.wavelengths[wl_idx],
                      w.m[np.ix_(dist_idx, wl_idx)], w.mu, w.n_nodes, w.greek_order)


def _mixed(gpu, w, above, levels=0):
    return gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, w.greek_order,
                              i8_above=above, levels=levels)


@pytest.mark.parametrize("levels", [5, 6])
@pytest.mark.parametrize("above", [1, 8, 20])
def test_small_spheres_mixed_within_tolerance(gpu, above, levels):
    """Every chunk with more than `above` terms on the int8 path (1: all of them)."""
    w = W.small_spheres()
    e = _errors(_mixed(gpu, w, above, levels), _oracle(w))
    print(f"small spheres, above {above}, {levels} levels: {e}")
    assert e["values"] <= 1e-12, e
    assert max(e.values()) <= TOL, e


def test_batched_full_shape_largest_n_units_mixed(gpu):
    """The batched workload's real shape (512 nodes, 360 Gauss cosines, order 64) on its units
    of largest N (up to 2198) and on a middle and a small distribution's units."""
    w = W.batched_spheres(seed=0)
    top = int(np.argmax(w.dists["r_hi"]))
    sub = _sub(w, top, [0, 1, 2, 3, 700, 1023])
    ref = _oracle(sub)
    for levels in (5, 6):
        e = _errors(_mixed(gpu, sub, 64, levels), ref)
        print(f"largest-N units, {levels} levels: {e}")
    e = _errors(_mixed(gpu, sub, 64), ref)
    assert max(e.values()) <= TOL, e
    order = np.argsort(w.dists["r_hi"])
    sub = _sub(w, [int(order[0]), int(order[w.dists.size // 2])], [0, 333, 1023])
    e = _errors(_mixed(gpu, sub, 64), _oracle(sub))
    assert max(e.values()) <= TOL, e


def test_batched_shape_small_mixed(gpu):
    w = W.batched_spheres(seed=3, scale=0.04)
    w.mu = W.gauss_legendre(64)
    e = _errors(_mixed(gpu, w, 32), _oracle(w))
    assert max(e.values()) <= TOL, e


@pytest.mark.parametrize("n_nodes", [7, 33, 100])
def test_ragged_chunks_and_unpaired_cosines_mixed(gpu, n_nodes):
    w = W.batched_spheres(seed=4, scale=0.02)
    w.n_nodes = n_nodes
    w.mu = np.array([1.0, 0.3, -0.3, 0.0, -1.0, 0.77, -0.9, 0.123])  # paired and unpaired
    w.greek_order = 24
    e = _errors(_mixed(gpu, w, 16), _oracle(w))
    assert max(e.values()) <= TOL, e


def test_mixed_deterministic_and_plain_when_no_chunk_qualifies(gpu):
    w = W.batched_spheres(seed=1, scale=0.03)
    w.mu = W.gauss_legendre(48)
    a = _mixed(gpu, w, 40)
    b = _mixed(gpu, w, 40)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    plain = gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, w.greek_order)
    none = _mixed(gpu, w, 100000)  # no chunk above: the plain path, bit for bit
    for x, y in zip(plain, none):
        assert np.array_equal(x, y)
    e = _errors(a, {"values": plain[0], "phase": plain[1], "greek": plain[2]})
    assert max(e.values()) <= TOL, e


def test_mixed_device_entry_matches_host_entry(gpu):
    import torch

    from scatrs_b200 import _native as N

    w = W.batched_spheres(seed=2, scale=0.03)
    w.mu = W.gauss_legendre(40)
    ref = _mixed(gpu, w, 24)
    dev = torch.device("cuda", 0)
    n = w.n_units
    wl = torch.tensor(w.wavelengths, dtype=torch.float64, device=dev)
    m = torch.tensor(w.m.view(np.float64).reshape(-1), dtype=torch.float64, device=dev)
    v = torch.empty(11 * n, dtype=torch.float64, device=dev)
    p = torch.empty(6 * n * w.mu.size, dtype=torch.float64, device=dev)
    g = torch.empty(6 * n * (w.greek_order + 1), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    N.ensemble_fixed_device(w.dists, wl.data_ptr(), w.wavelengths.size, m.data_ptr(), w.mu,
                            w.n_nodes, w.greek_order, True, v.data_ptr(), p.data_ptr(),
                            g.data_ptr(), stream, i8_above=24)
    N.check_errors(stream)
    assert np.array_equal(v.cpu().numpy().reshape(ref[0].shape), ref[0])
    assert np.array_equal(p.cpu().numpy().reshape(ref[1].shape), ref[1])
    assert np.array_equal(g.cpu().numpy().reshape(ref[2].shape), ref[2])
