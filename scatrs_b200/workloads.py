"""Seeded synthetic inputs of the benchmark configurations (no dataset is involved: every
input is drawn from numpy's default_rng with a recorded seed).

* ``small_spheres``: spheres m = 1.43 + 1e-8 i; lognormal r_g = 0.08, sigma_g = 1.6; wavelengths
  0.35, 0.55, 1.0; 256 Gauss nodes in ln r over r_g sigma_g^(+-5); 180 Gauss cosines; L = 32.
* ``batched_spheres``: 1024 wavelengths log-spaced over 0.3-2.5; 64 lognormals (median log-uniform
  0.05-5, width uniform 1.2-2.2); m per (distribution, wavelength) with Re uniform 1.33-1.60 and
  Im log-uniform 1e-8-1e-1; 512 Gauss nodes over median width^(+-4); 360 Gauss cosines; L = 64.
  ``scale`` keeps the first fraction of the wavelengths and distributions for smaller cases of
  the same shape.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from ._native import DIST_DTYPE, KINDS


@dataclass
class LayeredWorkload:
    name: str
    dists: np.ndarray
    wavelengths: np.ndarray
    fractions: np.ndarray  # (n_dist, L - 1)
    m_layers: np.ndarray   # complex (n_dist, L, n_wl)
    mu: np.ndarray
    n_nodes: int
    greek_order: int

    @property
    def n_units(self) -> int:
        return self.dists.size * self.wavelengths.size


@dataclass
class Workload:
    name: str
    dists: np.ndarray       # DIST_DTYPE, (n_dist,)
    wavelengths: np.ndarray  # (n_wl,)
    m: np.ndarray            # complex128 (n_dist, n_wl)
    mu: np.ndarray           # cosines
    n_nodes: int
    greek_order: int

    @property
    def n_units(self) -> int:
        return self.dists.size * self.wavelengths.size

    @property
    def n_nodes_total(self) -> int:
        return self.n_units * self.n_nodes


def gauss_legendre(n: int) -> np.ndarray:
    """Gauss-Legendre cosines from the library's own rule (the same on every machine)."""
    from ._native import gauss_legendre as gl

    return gl(n)[0]


def lognormals(median, width, spread) -> np.ndarray:
    median = np.atleast_1d(np.asarray(median, dtype=np.float64))
    width = np.broadcast_to(np.asarray(width, dtype=np.float64), median.shape)
    d = np.zeros(median.size, dtype=DIST_DTYPE)
    d["kind"] = KINDS["lognormal"]
    d["param"][:, 0] = median
    d["param"][:, 1] = width
    d["r_lo"] = median * width ** (-float(spread))
    d["r_hi"] = median * width ** float(spread)
    return d


def small_spheres(mu: np.ndarray | None = None) -> Workload:
    wl = np.array([0.35, 0.55, 1.0])
    d = lognormals(0.08, 1.6, 5)
    m = np.full((1, wl.size), 1.43 + 1e-8j)
    mu = gauss_legendre(180) if mu is None else mu
    return Workload("small_spheres", d, wl, m, mu, 256, 32)


def batched_spheres(seed: int = 0, scale: float = 1.0, mu: np.ndarray | None = None) -> Workload:
    rng = np.random.default_rng(seed)
    n_dist, n_wl = 64, 1024
    wl = np.geomspace(0.3, 2.5, n_wl)
    med = np.exp(rng.uniform(np.log(0.05), np.log(5.0), n_dist))
    wid = rng.uniform(1.2, 2.2, n_dist)
    m_re = rng.uniform(1.33, 1.60, (n_dist, n_wl))
    m_im = np.exp(rng.uniform(np.log(1e-8), np.log(1e-1), (n_dist, n_wl)))
    m = m_re + 1j * m_im
    if scale < 1.0:
        kd = max(1, int(round(n_dist * scale)))
        kw = max(1, int(round(n_wl * scale)))
        med, wid, m = med[:kd], wid[:kd], m[:kd, :kw]
        wl = wl[:kw]
    mu = gauss_legendre(360) if mu is None else mu
    return Workload(f"batched_spheres(seed={seed},scale={scale})", lognormals(med, wid, 4), wl, m, mu,
                    512, 64)


def gammas(r_eff, v_eff) -> np.ndarray:
    """Gamma distributions on grids wide enough for their tails: [max(0.01, 1 - 8 sqrt(b)) a,
    (1 + 12 sqrt(b)) a] for effective radius a and variance b."""
    a = np.atleast_1d(np.asarray(r_eff, dtype=np.float64))
    b = np.broadcast_to(np.asarray(v_eff, dtype=np.float64), a.shape)
    d = np.zeros(a.size, dtype=DIST_DTYPE)
    d["kind"] = KINDS["gamma"]
    d["param"][:, 0] = a
    d["param"][:, 1] = b
    d["r_lo"] = a * np.maximum(0.01, 1.0 - 8.0 * np.sqrt(b))
    d["r_hi"] = a * (1.0 + 12.0 * np.sqrt(b))
    return d


def large_droplets(seed: int = 0, scale: float = 1.0, n_q: int = 4096) -> Workload:
    """Large droplets: 128 gamma distributions (effective radius uniform 5-20, effective
    variance uniform 0.05-0.2) x 256 wavelengths log-spaced over 0.4-2.2, m = 1.33 + k i with k
    log-uniform 1e-9-1e-3 per (distribution, wavelength), 256 nodes in ln r, the phase matrix at
    n_q = 4096 Gauss cosines, Greek order 1024 (projected from those tables). ``scale`` keeps the
    first fraction of the distributions and wavelengths."""
    rng = np.random.default_rng(seed)
    n_dist, n_wl = 128, 256
    wl = np.geomspace(0.4, 2.2, n_wl)
    a = rng.uniform(5.0, 20.0, n_dist)
    b = rng.uniform(0.05, 0.2, n_dist)
    k = np.exp(rng.uniform(np.log(1e-9), np.log(1e-3), (n_dist, n_wl)))
    m = 1.33 + 1j * k
    if scale < 1.0:
        kd = max(1, int(round(n_dist * scale)))
        kw = max(1, int(round(n_wl * scale)))
        a, b, m, wl = a[:kd], b[:kd], m[:kd, :kw], wl[:kw]
    return Workload(f"large_droplets(seed={seed},scale={scale})", gammas(a, b), wl, m,
                    gauss_legendre(n_q), 256, 1024)


def layered_spheres(seed: int = 0, scale: float = 1.0, mu: np.ndarray | None = None) -> LayeredWorkload:
    """Three-layer spheres (a core and two shells): core fraction uniform 0.3-0.9, inner shell
    boundary uniform 0.9-0.99; each layer's index Re uniform 1.3-2.0, Im log-uniform 1e-6-0.5
    (per distribution and layer, the same at every wavelength); lognormal median uniform
    0.05-1, width uniform 1.3-2.0; 256 distributions x 128 wavelengths log-spaced over 0.3-1.6;
    256 Gauss nodes in ln r over median width^(+-4); Greek order 32."""
    rng = np.random.default_rng(seed)
    n_dist, n_wl = 256, 128
    wl = np.geomspace(0.3, 1.6, n_wl)
    med = rng.uniform(0.05, 1.0, n_dist)
    wid = rng.uniform(1.3, 2.0, n_dist)
    f = np.stack([rng.uniform(0.3, 0.9, n_dist), rng.uniform(0.9, 0.99, n_dist)], axis=1)
    m_re = rng.uniform(1.3, 2.0, (n_dist, 3))
    m_im = np.exp(rng.uniform(np.log(1e-6), np.log(0.5), (n_dist, 3)))
    ml = np.repeat((m_re + 1j * m_im)[:, :, None], n_wl, axis=2)
    if scale < 1.0:
        kd = max(1, int(round(n_dist * scale)))
        kw = max(1, int(round(n_wl * scale)))
        med, wid, f, ml, wl = med[:kd], wid[:kd], f[:kd], ml[:kd, :, :kw], wl[:kw]
    mu = gauss_legendre(180) if mu is None else mu
    return LayeredWorkload(f"layered_spheres(seed={seed},scale={scale})", lognormals(med, wid, 4), wl, f,
                           ml, mu, 256, 32)


@dataclass
class SpheroidWorkload:
    name: str
    dists: np.ndarray       # DIST_DTYPE, (n_dist,)
    wavelengths: np.ndarray
    aspect_ratio: np.ndarray  # (n_dist,)
    m: np.ndarray             # complex128 (n_dist, n_wl)
    mu: np.ndarray
    n_nodes: int
    greek_order: int

    @property
    def n_units(self) -> int:
        return self.dists.size * self.wavelengths.size

    @property
    def n_nodes_total(self) -> int:
        return self.n_units * self.n_nodes


def spheroids(seed: int = 0, scale: float = 1.0, per_ratio: int = 2, x_max: float = 25.0,
              mu: np.ndarray | None = None) -> SpheroidWorkload:
    """Randomly oriented spheroids: 16 aspect ratios log-spaced over 0.4-3.0, `per_ratio`
    lognormal volume-equivalent size distributions each (median uniform 0.2-1.5, width uniform
    1.5-2.0), m = 1.53 + k i with k log-uniform 1e-4-1e-1 per distribution, 32 wavelengths
    log-spaced over 0.35-1.0, 64 Gauss nodes in ln r over median width^(+-2) with the upper end
    capped where the size parameter at the shortest wavelength reaches `x_max` (the workload's
    sizes reach about 25); Greek order 64, 180 Gauss cosines."""
    rng = np.random.default_rng(seed)
    eps = np.repeat(np.geomspace(0.4, 3.0, 16), per_ratio)
    n_dist, n_wl = eps.size, 32
    wl = np.geomspace(0.35, 1.0, n_wl)
    med = rng.uniform(0.2, 1.5, n_dist)
    wid = rng.uniform(1.5, 2.0, n_dist)
    k = np.exp(rng.uniform(np.log(1e-4), np.log(1e-1), n_dist))
    m = np.repeat((1.53 + 1j * k)[:, None], n_wl, axis=1)
    d = np.zeros(n_dist, dtype=DIST_DTYPE)
    d["kind"] = KINDS["lognormal"]
    d["param"][:, 0] = med
    d["param"][:, 1] = wid
    r_cap = x_max * wl.min() / (2 * np.pi)
    d["r_hi"] = np.minimum(med * wid ** 2, r_cap)
    d["r_lo"] = np.minimum(med * wid ** -2, d["r_hi"] / 4)
    if scale < 1.0:
        kw = max(1, int(round(n_wl * scale)))
        wl, m = wl[:kw], m[:, :kw]
    mu = gauss_legendre(180) if mu is None else mu
    return SpheroidWorkload(f"spheroids(seed={seed},scale={scale},x_max={x_max})", d, wl, eps, m,
                            mu, 64, 64)
