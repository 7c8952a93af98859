"""The spheroid T-matrix's regularized y-part (tmatrix.cu: tm_series_kernel, tm_surface_kernel;
the reference's tmatrix/regular.rs and kernel.rs:468-490) on the GPU.

- Exactness: the three forms of each element of Q (plain, minus the y-part's Laurent terms of
  power < 0, minus those of power <= 0) are the same integral; forcing each form on every element
  where it applies (SCATRS_TMATRIX_FORM) gives the T-matrix of the chosen forms within 1e-11 of
  its largest element at sizes where the plain form is still accurate in double-double.
- The workload's corners inside the validated domain converge to rtol 1e-8: aspect ratio 3 at
  x = 25 and aspect ratio 0.4 at x = 21 (|m| x_max = 60 is the domain's edge), for the
  workload's smallest and largest Im m.
- Lossless spheroids there conserve energy: |Q_abs| <= 1e-9 Q_ext, and the converged mode-0
  T-matrix is unitary (T + T^H = -2 T^H T) to 1e-8 of its largest element.
- Outside the validated domain (tmatrix/domain.rs:45-79) a spheroid is refused with
  OutsideValidatedDomainError unless allow_unvalidated; x = 25 at aspect ratio 0.4 (|m| x_max =
  70) then converges for Im m = 0.1.
"""

import numpy as np
import pytest

from scatrs_b200 import _native
from scatrs_b200.errors import OutsideValidatedDomainError

pytestmark = pytest.mark.gpu


def _unitarity(t):
    a = t + t.conj().T
    b = 2.0 * t.conj().T @ t
    return min(np.abs(a + b).max(), np.abs(a - b).max()) / np.abs(t).max()


FORMS = [(6.0, 2.0, 1.5 + 0.01j, 24, 60), (12.0, 3.0, 1.53 + 0.01j, 36, 90),
         (8.0, 0.4, 1.53 + 1e-3j, 30, 80), (10.0, 0.5, 1.33 + 0.0j, 30, 80)]


@pytest.mark.parametrize("x,eps,m,N,nth", FORMS)
def test_every_form_gives_the_same_tmatrix(gpu, monkeypatch, x, eps, m, N, nth):
    for mode in (0, 3):
        monkeypatch.delenv("SCATRS_TMATRIX_FORM", raising=False)
        ref = _native.spheroid_tmatrix(x, eps, m, mode, N, nth)
        for form in ("0", "1", "2"):
            monkeypatch.setenv("SCATRS_TMATRIX_FORM", form)
            t = _native.spheroid_tmatrix(x, eps, m, mode, N, nth)
            err = np.abs(t - ref).max() / np.abs(ref).max()
            assert err <= 1e-11, (mode, form, err)


CORNERS = [(25.0, 3.0), (21.0, 0.4)]


@pytest.mark.parametrize("x,eps", CORNERS)
@pytest.mark.parametrize("k", [1e-4, 1e-1])
def test_the_workload_corners_converge(gpu, x, eps, k):
    r = _native.spheroid_compute(np.array([x]), eps, 1.53 + 1j * k, rtol=1e-8)
    q_ext, q_sca, q_abs = r["efficiencies"][0][:3]
    assert np.isfinite(r["efficiencies"][0][:3]).all()
    assert q_ext > q_sca > 0.0 and q_abs > 0.0
    assert r["n_terms"][0] >= 50
    assert r["error_estimate"][0] < 1e-12


@pytest.mark.parametrize("x,eps", CORNERS)
def test_lossless_corners_conserve_energy(gpu, x, eps):
    r = _native.spheroid_compute(np.array([x]), eps, 1.53 + 0j, rtol=1e-8)
    q_ext, q_sca, q_abs = r["efficiencies"][0][:3]
    assert abs(q_abs) <= 1e-9 * q_ext, (q_ext, q_sca)
    t = _native.spheroid_tmatrix(x, eps, 1.53 + 0j, 0, int(r["n_terms"][0]),
                                 int(r["n_theta"][0]))
    assert _unitarity(t) <= 1e-8


def test_outside_the_validated_domain(gpu):
    with pytest.raises(OutsideValidatedDomainError):
        _native.spheroid_compute(np.array([25.0]), 0.4, 1.53 + 1e-4j, rtol=1e-8)
    with pytest.raises(OutsideValidatedDomainError):
        _native.spheroid_compute(np.array([2.0]), 2.0, 1.2 + 0.01j, rtol=1e-8)
    with pytest.raises(OutsideValidatedDomainError):
        _native.spheroid_compute(np.array([2.0]), 6.0, 1.5 + 0.01j, rtol=1e-8)
    r = _native.spheroid_compute(np.array([25.0]), 0.4, 1.53 + 0.1j, rtol=1e-8,
                                 allow_unvalidated=True)
    q_ext, q_sca, q_abs = r["efficiencies"][0][:3]
    assert q_ext > q_sca > 0.0 and q_abs > 0.0
