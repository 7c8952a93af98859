"""The Greek projection of phase tables at Gauss cosines (scatrs_project_greek_device): the
FP64 form against the band projection of the same ensemble (both exact for these tables, so
they agree to rounding: 1e-10 of alpha1_0 = 1), and the 3xTF32 tensor-core form against the
FP64 form (TF32 heads and tails with FP32 accumulation: within 2e-5 of the largest
coefficient of each table)."""

import numpy as np
import pytest
import torch

from scatrs_b200 import _native
from scatrs_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _ensemble_on_device(w, mu, L):
    n = w.n_units
    dev = torch.device("cuda")
    wl = torch.tensor(w.wavelengths, device=dev)
    m = torch.tensor(np.ascontiguousarray(w.m).view(np.float64).reshape(-1), device=dev)
    values = torch.zeros(11 * n, dtype=torch.float64, device=dev)
    phase = torch.zeros(6 * n * mu.size, dtype=torch.float64, device=dev)
    greek = torch.zeros(6 * n * (L + 1), dtype=torch.float64, device=dev)
    _native.ensemble_fixed_device(w.dists, wl.data_ptr(), w.wavelengths.size, m.data_ptr(), mu,
                                  w.n_nodes, L, True, values.data_ptr(), phase.data_ptr(),
                                  greek.data_ptr())
    _native.check_errors()
    return phase, greek.reshape(6, n, L + 1).cpu().numpy()


def _project(phase, n, n_q, L, precision):
    out = torch.zeros(6 * n * (L + 1), dtype=torch.float64, device="cuda")
    _native.project_greek_device(phase.data_ptr(), n, n_q, L, precision, out.data_ptr())
    torch.cuda.synchronize()
    return out.reshape(6, n, L + 1).cpu().numpy()


@pytest.mark.parametrize("n_q,L", [(512, 200), (301, 77)])
def test_fp64_projection_matches_the_bands(gpu, n_q, L):
    w = W.Workload("gammas", W.gammas([1.0, 1.8], [0.1, 0.15]), np.array([0.5, 0.9, 1.5]),
                   np.full((2, 3), 1.33 + 1e-6j), W.gauss_legendre(n_q), 128, L)
    phase, band = _ensemble_on_device(w, w.mu, L)
    got = _project(phase, w.n_units, n_q, L, 0)
    assert np.abs(got - band).max() <= 1e-10, np.abs(got - band).max()
    assert np.allclose(got[0, :, 0], 1.0, rtol=0, atol=1e-12)


def test_tensor_core_projection_matches_fp64(gpu):
    w = W.large_droplets(seed=1, scale=0.02, n_q=1024)  # 3 distributions x 5 wavelengths
    w.wavelengths = w.wavelengths * 4.0            # smaller size parameters: N < 1024 - L / 2
    L = 300
    phase, _ = _ensemble_on_device(w, w.mu, -1)
    ref = _project(phase, w.n_units, w.mu.size, L, 0)
    tc = _project(phase, w.n_units, w.mu.size, L, 1)
    size = np.abs(ref).max(axis=(0, 2), keepdims=True)
    err = np.abs(tc - ref) / size
    assert err.max() <= 2e-5, err.max()
    assert err.max() > 0.0  # the tensor-core form ran (it differs from FP64 by rounding)


def test_tensor_core_projection_at_the_large_droplet_shape(gpu):
    """The large-droplet configuration's own shape: 4096 Gauss cosines, order 1024, on the
    ensemble's own phase tables (gamma distributions of effective radius 5-20 um, x up to about
    300), the 3xTF32 form against the FP64 form. The stated tolerance is 2e-5 of each table's
    largest coefficient (TF32 heads and tails, the tensor cores' FP32 accumulation over 4096
    cosines)."""
    w = W.large_droplets(seed=0, scale=0.02, n_q=4096)  # 3 distributions x 5 wavelengths
    L = 1024
    phase, _ = _ensemble_on_device(w, w.mu, -1)
    ref = _project(phase, w.n_units, w.mu.size, L, 0)
    tc = _project(phase, w.n_units, w.mu.size, L, 1)
    size = np.abs(ref).max(axis=(0, 2), keepdims=True)
    err = np.abs(tc - ref) / size
    print(f"3xTF32 at n_q = 4096, L = 1024: max error {err.max():.3e} of the largest "
          "coefficient")
    assert err.max() <= 2e-5, err.max()
