"""Failures made on the host while the GPU path runs (no GPU fault): a device allocation that
fails as an out-of-memory cudaMalloc would, and node errors merged into the device's error word
as the kernels merge theirs. Both must reach Python as the reference's classes, with the first
error in (wavelength, distribution, radius) order (scatrs/src/ensemble/engine.rs:588-606) named
by its wavelength and radius (engine.rs:124-131), and leave the library usable."""

import numpy as np
import pytest

from scatrs_b200 import workloads as W
from scatrs_b200.errors import DeviceError, InvalidInputError, OutsideValidatedDomainError

pytestmark = pytest.mark.gpu


def _radii(w, d):
    xi = W.gauss_legendre(w.n_nodes)
    a, b = np.log(w.dists["r_lo"][d]), np.log(w.dists["r_hi"][d])
    return np.exp(0.5 * (a + b) + 0.5 * (b - a) * xi)


def _small():
    w = W.batched_spheres(seed=5, scale=0.01)  # 1 distribution x 10 wavelengths
    w.n_nodes = 64
    w.mu = W.gauss_legendre(16)
    w.greek_order = 8
    return w


def test_allocation_failure_is_a_device_error_and_the_library_recovers(gpu):
    w = _small()
    lib = gpu.load()
    ref = gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, w.greek_order)
    for k in (1, 3):
        lib.scatrs_release()  # every buffer grows again on the next call
        lib.scatrs_testing_fail_allocation(k)
        with pytest.raises(DeviceError, match="out of memory"):
            gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, w.greek_order)
        lib.scatrs_testing_fail_allocation(0)
        got = gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, w.greek_order)
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)


def test_forced_node_error_names_its_wavelength_and_radius(gpu):
    w = _small()
    lib = gpu.load()
    n_dist = w.dists.size
    r = _radii(w, 0)
    i, j = 3, 17
    lib.scatrs_testing_force_node_error((i * n_dist + 0) * w.n_nodes + j, 3)
    with pytest.raises(OutsideValidatedDomainError) as info:
        gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, w.greek_order)
    msg = str(info.value)
    assert f"{w.wavelengths[i]:e}" in msg and f"{r[j]:e}" in msg, msg
    # one-shot: the next call succeeds
    gpu.ensemble_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, w.greek_order)


def test_first_error_in_order_wins(gpu):
    w = _small()
    lib = gpu.load()
    n_dist = w.dists.size
    r = _radii(w, 0)
    bad = w.m.copy()
    bad[0, 5] = -1.5 + 0j  # a real invalid input at wavelength 5, every node
    # a forced error later in order than the real one: the real one is reported
    lib.scatrs_testing_force_node_error((7 * n_dist + 0) * w.n_nodes + 2, 3)
    with pytest.raises(InvalidInputError) as info:
        gpu.ensemble_fixed(w.dists, w.wavelengths, bad, w.mu, w.n_nodes, w.greek_order)
    assert f"{w.wavelengths[5]:e}" in str(info.value) and f"{r[0]:e}" in str(info.value)
    # a forced error earlier in order: it is reported
    lib.scatrs_testing_force_node_error((2 * n_dist + 0) * w.n_nodes + 9, 3)
    with pytest.raises(OutsideValidatedDomainError) as info:
        gpu.ensemble_fixed(w.dists, w.wavelengths, bad, w.mu, w.n_nodes, w.greek_order)
    assert f"{w.wavelengths[2]:e}" in str(info.value) and f"{r[9]:e}" in str(info.value)
