"""Host logic without a GPU: the binding surface's parameter names and specs, the seeded
workloads, and ensemble identities of the reference's tests (scatrs/tests/ensemble.rs) on the
oracle's fixed-grid restatement."""

import ctypes
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from scatrs_b200 import _native, _scatrs, workloads as W
from scatrs_b200.errors import InvalidInputError


def test_parameter_names_follow_the_reference():
    m = np.array([1.5 + 0j])
    assert _scatrs.ensemble_parameters([(("lognormal", 0.1, 1.5), ("sphere", m), 1.0)], False) \
        == ["median_radius", "width", "m_real", "m_imag"]
    names = _scatrs.ensemble_parameters(
        [(("gamma", 1.0, 0.1), ("sphere", m), 1.0),
         (("multimodal", [(1.0, ("lognormal", 0.1, 1.5)), (2.0, ("lognormal", 1.0, 2.0))]),
          ("layered", np.array([0.5]), np.ones((2, 1), complex)), 2.0)], True)
    assert names == ["c0.effective_radius", "c0.effective_variance", "c0.m_real", "c0.m_imag",
                     "c0.weight", "c1.mode0.median_radius", "c1.mode0.width", "c1.mode0.weight",
                     "c1.mode1.median_radius", "c1.mode1.width", "c1.mode1.weight",
                     "c1.layer0.m_real", "c1.layer0.m_imag", "c1.layer1.m_real",
                     "c1.layer1.m_imag", "c1.layer0.radius_fraction", "c1.weight"]
    with pytest.raises(InvalidInputError):
        _scatrs.ensemble_parameters([(("lognormal", 0.1, 1.5), ("sphere", m), 1.0)] * 2, False)
    with pytest.raises(TypeError):
        _scatrs.ensemble_parameters([(("weibull", 1.0), ("sphere", m), 1.0)], False)


def test_parameter_records_carry_each_name_to_its_kind():
    """Every name of ensemble_parameters has a (component, mode, kind, index) record in the same
    order (EnsembleParam, ensemble/mod.rs:180-215): a spheroid's Re m, Im m and aspect ratio, a
    layered sphere's LayerRefrReal(l), LayerRefrImag(l) per layer then RadiusFraction(l), a
    multimodal component's modes and mode weights."""
    m = np.array([1.5 + 0j])
    items = [(("lognormal", 0.1, 1.5), ("spheroid", 2.0, m), 1.0),
             (("multimodal", [(1.0, ("lognormal", 0.1, 1.5)), (2.0, ("gamma", 1.0, 0.1))]),
              ("layered", np.array([0.3, 0.6]), np.ones((3, 1), complex)), 2.0)]
    names = _scatrs.ensemble_parameters(items, True)
    records = _scatrs._parameter_records(items, True)
    assert len(records) == len(names)
    kind = {_native.PARAM_DISTRIBUTION: "d", _native.PARAM_REFR_REAL: "m_real",
            _native.PARAM_REFR_IMAG: "m_imag", _native.PARAM_WEIGHT: "weight",
            _native.PARAM_ASPECT_RATIO: "aspect_ratio",
            _native.PARAM_LAYER_REFR_REAL: "layer{}.m_real",
            _native.PARAM_LAYER_REFR_IMAG: "layer{}.m_imag",
            _native.PARAM_RADIUS_FRACTION: "layer{}.radius_fraction"}
    for name, (comp, mode, k, index) in zip(names, records):
        assert name.startswith(f"c{comp}.")
        if mode >= 0:
            assert f".mode{mode}." in name
        if k != _native.PARAM_DISTRIBUTION:
            assert name.endswith("." + kind[k].format(index)), (name, k, index)
    assert [r[2] for r in records[:6]] == [0, 0, 1, 2, 4, 3]
    assert records[-4:-1] == [(1, -1, _native.PARAM_LAYER_REFR_IMAG, 2),
                              (1, -1, _native.PARAM_RADIUS_FRACTION, 0),
                              (1, -1, _native.PARAM_RADIUS_FRACTION, 1)]


def test_distribution_specs_and_ranges():
    d = _scatrs._dist_array([("lognormal", 0.2, 1.5), ("power_law", 3.0, 0.1, 2.0)], 4.0)
    assert d["kind"].tolist() == [1, 4]
    assert np.isclose(d["r_lo"][0], 0.2 * 1.5 ** -4) and np.isclose(d["r_hi"][0], 0.2 * 1.5 ** 4)
    assert (d["r_lo"][1], d["r_hi"][1]) == (0.1, 2.0)
    with pytest.raises(InvalidInputError):
        _scatrs._dist_array([("gamma", 1.0, 0.1)], 4.0)
    with pytest.raises(TypeError):
        _scatrs._dist_array([("bogus", 1.0)], 4.0)


def test_tabulated_specs_point_at_their_tables():
    """("tabulated", radii, densities) (scatrs-py/src/ensemble.rs:58-61): kind 6, the table as
    radii then densities, kept alive by the records; the grid spans the table."""
    d = _scatrs._adaptive_dists([("lognormal", 0.2, 1.5), ("tabulated", [0.1, 0.3, 0.9],
                                                            [0.0, 2.0, 1.0])])
    assert d["kind"].tolist() == [1, _native.TABULATED] and d["table_len"].tolist() == [0, 3]
    tab = np.ctypeslib.as_array(
        ctypes.cast(int(d["table"][1]), ctypes.POINTER(ctypes.c_double)), shape=(6,))
    assert tab.tolist() == [0.1, 0.3, 0.9, 0.0, 2.0, 1.0]
    assert len(d.tables) == 1 and d.tables[0].ctypes.data == int(d["table"][1])
    f = _scatrs._dist_array([("tabulated", [0.1, 0.9], [1.0, 1.0])], 4.0)
    assert (f["r_lo"][0], f["r_hi"][0]) == (0.1, 0.9)
    with pytest.raises(InvalidInputError, match="at least 2 points"):
        _scatrs._adaptive_dists([("tabulated", [0.1, 0.2, 0.3], [1.0, 1.0])])


def test_distribution_records_match_the_c_struct(tmp_path):
    """The numpy record is scatrs_distribution byte for byte (size and field offsets)."""
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stddef.h>\n#include <stdio.h>\n#include "scatrs_b200.h"\n'
        "int main(void) { printf(\"%zu %zu %zu %zu %zu %zu %zu\", sizeof(scatrs_distribution), "
        "offsetof(scatrs_distribution, param), offsetof(scatrs_distribution, r_lo), "
        "offsetof(scatrs_distribution, r_hi), offsetof(scatrs_distribution, table), "
        "offsetof(scatrs_distribution, table_len), offsetof(scatrs_distribution, kind)); "
        "return 0; }\n")
    exe = tmp_path / "layout"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run(["gcc", "-I", inc, str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    t = _native.DIST_DTYPE
    want = [t.itemsize] + [t.fields[k][1] for k in ("param", "r_lo", "r_hi", "table",
                                                     "table_len", "kind")]
    assert got == want


def test_workloads_are_seeded_and_shaped():
    a, b = W.batched_spheres(seed=5), W.batched_spheres(seed=5)
    assert np.array_equal(a.m, b.m) and np.array_equal(a.dists, b.dists)
    assert a.n_nodes_total == 33554432 and a.mu.size == 360 and a.greek_order == 64
    assert not np.array_equal(W.batched_spheres(seed=6).m, a.m)
    assert 1.33 <= a.m.real.min() and a.m.real.max() <= 1.60
    assert 1e-8 <= a.m.imag.min() and a.m.imag.max() <= 1e-1
    c = W.small_spheres()
    assert c.n_nodes_total == 768 and c.greek_order == 32


def test_bands_follow_the_reference_sequence():
    seq = [O.bucket(n) for n in range(1, 40)]
    assert seq[:12] == [1, 2, 3, 4, 5, 7, 7, 9, 9, 12, 12, 12]
    assert O.bucket(2198) == 2712 and O.bucket(2169) == 2169


def _fixed(w, **kw):
    d = np.zeros(w.dists.size, dtype=O.DIST_DTYPE)
    d["kind"], d["p"] = w.dists["kind"], w.dists["param"]
    d["r_lo"], d["r_hi"] = w.dists["r_lo"], w.dists["r_hi"]
    return O.ensemble_fixed(d, w.wavelengths, w.m, w.n_nodes, w.mu, w.greek_order, **kw)


def test_narrow_distribution_is_the_single_sphere():
    """A lognormal narrow enough is one sphere: the averages are its cross sections
    (scatrs/tests/ensemble.rs:61-112, monodisperse = single sphere)."""
    r0, lam, m = 0.3, 0.55, 1.5 + 0.01j
    w = W.Workload("narrow", W.lognormals(r0, 1.0 + 1e-9, 1.0), np.array([lam]),
                   np.full((1, 1), m), np.array([1.0, 0.5, -0.2, -1.0]), 64, 8)
    out = _fixed(w)
    s = O.mie(2 * np.pi * r0 / lam, m)
    area = np.pi * r0 * r0
    assert np.isclose(out["values"][0, 0], area * s["q_ext"], rtol=1e-7)
    assert np.isclose(out["values"][5, 0], s["g"], rtol=1e-7)
    g = O.mie_greek(2 * np.pi * r0 / lam, m, 8)
    assert np.allclose(out["greek"][:, 0, :], g, rtol=1e-6, atol=1e-9)


def test_normalized_phase_integrates_to_one_and_alpha1_is_3g():
    w = W.small_spheres()
    mu, wt = O.gauss_legendre(200)
    w.mu = mu
    out = _fixed(w)
    norm = 0.5 * (out["phase"][0] * wt[None]).sum(axis=1)
    assert np.allclose(norm, 1.0, rtol=1e-12)
    assert np.allclose(out["greek"][0, :, 1], 3 * out["values"][5], rtol=1e-11)
    assert np.all(out["greek"][0, :, 0] == 1.0)


def test_rayleigh_limit():
    """Small spheres: Q_sca ~ (8/3) x^4 |(m^2-1)/(m^2+2)|^2 (scatrs/tests/ensemble.rs:158-174)."""
    r, lam, m = 1e-3, 1.0, 1.5 + 0j
    x = 2 * np.pi * r / lam
    s = O.mie(x, m)
    k = abs((m * m - 1) / (m * m + 2)) ** 2
    assert np.isclose(s["q_sca"], 8.0 / 3.0 * x ** 4 * k, rtol=1e-4)


def test_errors_are_the_reference_classes():
    w = W.small_spheres()
    w.m = np.full_like(w.m, 1.5 + 11j)
    with pytest.raises(O.OracleError) as e:
        _fixed(w)
    assert e.value.status == 3 and "at wavelength" in str(e.value)


def test_autograd_backward_contracts_the_jacobian(monkeypatch):
    """The torch wrapper's backward pass is J^T g over every output of each unit, summed over
    the wavelengths for the distribution parameters (a fake forward with a known Jacobian)."""
    import torch

    from scatrs_b200 import _native, autograd

    rng = np.random.default_rng(3)
    n_dist, n_wl, n_mu, L = 2, 3, 4, 5
    n = n_dist * n_wl
    P = 4
    jv, jp, jg = (rng.normal(size=s) for s in ((P, 11, n), (P, 6, n, n_mu), (P, 6, n, L + 1)))

    def fake(dists, wl, m, mu, n_nodes, greek_order, normalized, allow):
        th = dists["param"][:, :2]
        x = np.concatenate([np.repeat(th, n_wl, axis=0).T, m.real.reshape(1, -1),
                            m.imag.reshape(1, -1)])  # (P, n)
        v = np.einsum("pkn,pn->kn", jv, x)
        ph = np.einsum("pknj,pn->knj", jp, x)
        g = np.einsum("pknj,pn->knj", jg, x)
        return v, ph, g, jv, jp, jg

    monkeypatch.setattr(_native, "ensemble_fixed_d", fake)
    theta = torch.tensor(rng.uniform(0.1, 2, (n_dist, 2)), requires_grad=True)
    m_re = torch.tensor(rng.uniform(1.3, 1.6, (n_dist, n_wl)), requires_grad=True)
    m_im = torch.tensor(rng.uniform(0, 0.1, (n_dist, n_wl)), requires_grad=True)
    v, ph, g = autograd.ensemble_fixed(theta, m_re, m_im, kind="lognormal",
                                       ranges=[[0.01, 1.0]] * n_dist, wavelengths=[0.4, 0.5, 0.6],
                                       mu=np.zeros(n_mu), greek_order=L)
    wv, wp, wg = (torch.tensor(rng.normal(size=t.shape)) for t in (v, ph, g))
    ((v * wv).sum() + (ph * wp).sum() + (g * wg).sum()).backward()
    tot = (np.einsum("pkn,kn->pn", jv, wv.numpy()) + np.einsum("pknj,knj->pn", jp, wp.numpy())
           + np.einsum("pknj,knj->pn", jg, wg.numpy())).reshape(P, n_dist, n_wl)
    assert np.allclose(theta.grad.numpy(), tot[:2].sum(axis=2).T)
    assert np.allclose(m_re.grad.numpy(), tot[2])
    assert np.allclose(m_im.grad.numpy(), tot[3])
