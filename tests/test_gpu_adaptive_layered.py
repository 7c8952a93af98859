"""The adaptive ensemble of layered spheres on the GPU (scatrs_ensemble_adaptive_layered: the
layered branch of the pass-1 kernel and the layered K-a on the final panels) against the
oracle's adaptive engine with its layered node solve (layered/kernel.rs): the same panels and
convergence flags, values within 1e-11 (the layered recursion's rounding, as the fixed grid's
layered check), error estimates as the sphere path's; one layer equals the sphere path."""

import numpy as np
import pytest

from oracle import oracle as O
from test_gpu_adaptive import MU, _compare, _dists, _odist

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("batch", [False, True])
def test_matches_the_oracle(gpu, batch):
    d = _dists((1, 0.2, 1.5), (2, 0.3, 0.12), (5, 0.4))
    wl = np.array([0.45, 0.8])
    fr = np.array([[0.6, 0.9], [0.5, 0.95], [0.7, 0.8]])
    ml = np.array([[[1.8 + 0.05j, 1.7 + 0.04j], [1.5 + 0.001j, 1.5 + 0.0j],
                    [1.33 + 0j, 1.33 + 1e-5j]],
                   [[2.0 + 0.3j, 1.9 + 0.2j], [1.6 + 0.01j, 1.55 + 0.01j], [1.4 + 0j, 1.4 + 0j]],
                   [[1.5 + 0.1j, 1.5 + 0.1j], [1.45 + 0j, 1.45 + 0j], [1.6 + 0.02j, 1.6 + 0.02j]]])
    if batch:  # a batch has one particle
        fr = np.broadcast_to(fr[0], fr.shape).copy()
        ml = np.broadcast_to(ml[0], ml.shape).copy()
    got = gpu.ensemble_adaptive_layered(d, wl, fr, ml, MU, 12, batch=batch)
    ref = O.ensemble_adaptive_layered(_odist(d), wl, fr, ml, MU, 12, batch=batch)
    _compare(got, ref, tol=1e-11)


def test_one_layer_is_the_sphere_path(gpu):
    d = _dists((1, 0.1, 1.7), (2, 0.4, 0.1))
    wl = np.array([0.5, 0.9])
    m = np.array([1.45 + 0.002j, 1.44 + 0.001j])
    one = gpu.ensemble_adaptive_layered(d, wl, np.zeros((2, 0)),
                                        np.broadcast_to(m, (2, 1, 2)), MU, 8)
    sph = gpu.ensemble_adaptive(d, wl, m, MU, 8)
    for k in ("values", "errors", "phase", "greek", "panels", "converged"):
        assert np.array_equal(one[k], sph[k]), k
