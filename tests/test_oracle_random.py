"""The oracle's orientation average of a spheroid's phase matrix (oracle/oracle_random.cpp, the
rank decomposition of random.rs:85-335) against the reference's own checks of it
(random.rs:338-411): the brute-force average of research/tmatrix/ranks.py at one angle, a
sphere giving Mie's phase matrix, and the phase function integrating to the scattering cross
section; and its Greek coefficients (greek_raw, random.rs:283-292): alpha1_0 = C_sca / (4 pi),
and the expansion reproducing the elements."""

import numpy as np
import pytest

from oracle import oracle as O


def test_matches_the_brute_force_average():
    """random.rs:343-355: x = 2, eps = 1.8, s = 1.5 + 0.02i, N = 6, 15 nodes in 0 < theta <
    pi/2, Theta = 0.4: the six elements of the brute-force average to 2e-6."""
    modes = O.tmatrix_modes(2.0, 1.8, 1.5 + 0.02j, 6, 15)
    f = O.random_orientation(modes, [np.cos(0.4)])[:, 0]
    want = [6.980506, -0.33857, 6.912394, 6.902738, 0.118319, 6.84077]
    assert np.abs(f - want).max() < 2e-6


def test_a_sphere_gives_the_mie_phase_matrix():
    """random.rs:357-395: (4/x^2) <Z> = Mie's unnormalized phase matrix, F22 = F11, F44 = F33."""
    x, m, n = 3.0, 1.5 + 0.01j, 14
    modes = O.tmatrix_modes(x, 1.0, m, n, 30)
    mu = np.array([-0.95 + 0.3 * k for k in range(7)])
    f = O.random_orientation(modes, mu) * (4.0 / x ** 2)
    s1, s2 = O.amplitudes(x, m, mu, n_max=n)
    k = 4.0 / x ** 2
    f11 = k * (abs(s1) ** 2 + abs(s2) ** 2) / 2
    f12 = k * (abs(s2) ** 2 - abs(s1) ** 2) / 2
    f33 = k * (s2 * np.conj(s1)).real
    f34 = k * (s2 * np.conj(s1)).imag
    for got, want in [(f[0], f11), (f[2], f11), (f[1], f12), (f[3], f33), (f[5], f33),
                      (f[4], f34)]:
        assert np.all(np.abs(got - want) <= 1e-12 * np.abs(f11))


def _c_sca(x, eps, s, n, nt):
    return O.spheroid_q(x, eps, s, n, nt)[1] * np.pi * x * x


def test_the_phase_function_integrates_to_the_scattering_cross_section():
    """random.rs:397-410: 2 pi int F11 dmu = <C_sca> (Gauss-Legendre, exact for the degree-2N
    polynomial)."""
    n = 10
    modes = O.tmatrix_modes(3.0, 0.5, 1.5 + 0.02j, n, 30)
    mu, w = O.gauss_legendre(2 * n + 2)
    f = O.random_orientation(modes, mu)
    integral = 2 * np.pi * np.dot(w, f[0])
    sca = _c_sca(3.0, 0.5, 1.5 + 0.02j, n, 30)
    assert abs(integral - sca) < 1e-12 * sca


@pytest.mark.parametrize("x,eps,s,n,nt", [(2.0, 1.8, 1.5 + 0.02j, 8, 20),
                                          (1.5, 0.6, 1.33 + 0.0j, 7, 16)])
def test_greek_coefficients(x, eps, s, n, nt):
    """alpha1_0 = C_sca / (4 pi) (random.rs:283-287), the order capped at 2N, and the Greek
    expansion sum_l alpha1_l P_l(mu) reproducing F11 at other cosines."""
    modes = O.tmatrix_modes(x, eps, s, n, nt)
    g = O.random_greek(modes, 100)
    assert g.shape == (6, 2 * n + 1)
    sca = _c_sca(x, eps, s, n, nt)
    assert abs(g[0, 0] - sca / (4 * np.pi)) < 1e-12 * g[0, 0]
    mu = np.array([-0.7, 0.1, 0.55, 0.93])
    f = O.random_orientation(modes, mu)
    for j, u in enumerate(mu):
        p = np.polynomial.legendre.legval(u, g[0])
        assert abs(p - f[0, j]) < 1e-12 * abs(f[0]).max()
