"""Tabulated size distributions in the oracle (n(r) linear between the table's points, 0
outside; scatrs/src/ensemble/distribution.rs:55-62, 149-172, 458-468) against the reference's
own checks: a uniform table is a flat power law (scatrs/tests/ensemble.rs:718-734), a spike
table with fewer panels allowed than intervals stays finite (ensemble.rs:890-897), invalid
tables are rejected (distribution.rs:624-633), the error estimates of the reference's table
case bound the true errors (ensemble.rs:501-507 on the grid of 469-647); and the moments
against the closed form of a piecewise-linear density."""

import math

import numpy as np
import pytest

from oracle import oracle as O

REF_TABLE = ([0.05, 0.1, 0.4, 1.0], [0.0, 3.0, 1.0, 0.2])


def _linear_moment(radii, dens, k):
    """The exact integral of r^k n(r) over a piecewise-linear n."""
    total = 0.0
    for a, b, na, nb in zip(radii[:-1], radii[1:], dens[:-1], dens[1:]):
        s = (nb - na) / (b - a)
        total += (na - s * a) * (b ** (k + 1) - a ** (k + 1)) / (k + 1)
        total += s * (b ** (k + 2) - a ** (k + 2)) / (k + 2)
    return total


def test_a_uniform_table_is_a_flat_power_law():
    table = O.table_dist([0.1, 0.5], [1.0, 1.0])
    flat = O.dist(4, 0.0, 0.1, 0.5)
    a = O.ensemble_adaptive(table, [0.5], 1.5 + 0j, rtol=1e-9)
    b = O.ensemble_adaptive(flat, [0.5], 1.5 + 0j, rtol=1e-9)
    assert abs(a["values"][0, 0] / b["values"][0, 0] - 1) < 1e-8


def test_moments_match_the_piecewise_linear_closed_form():
    r, n = REF_TABLE
    e = O.ensemble_adaptive(O.table_dist(r, n), [0.5], 1.45 + 0.001j, rtol=1e-9)
    v = e["values"][:, 0]
    z, m2, m3 = (_linear_moment(r, n, k) for k in (0, 2, 3))
    assert abs(v[9] - math.pi * m2 / z) <= 1e-9 * math.pi * m2 / z
    assert abs(v[10] - 4 * math.pi / 3 * m3 / z) <= 1e-9 * 4 * math.pi / 3 * m3 / z
    assert abs(v[8] - m3 / m2) <= 1e-9 * m3 / m2
    assert e["converged"][0]


def test_a_spike_with_one_panel_stays_finite():
    spike = O.table_dist([0.1, 0.2, 0.2001, 0.2002, 0.5], [0.0, 0.0, 1.0, 0.0, 0.0])
    e = O.ensemble_adaptive(spike, [0.5], 1.5 + 0j, max_panels=1)
    assert np.all(np.isfinite(e["values"])) and e["values"][0, 0] > 0.0


@pytest.mark.parametrize("radii,dens,msg", [
    ([1.0, 1.0], [1.0, 1.0], "increase"),
    ([1.0, 2.0], [0.0, 0.0], "all be 0"),
    ([1.0, 2.0], [1.0, -1.0], "finite and >= 0"),
    ([float("nan"), 2.0], [1.0, 1.0], "radius"),
    ([1.0], [1.0], "at least 2"),
])
def test_invalid_tables_are_rejected(radii, dens, msg):
    with pytest.raises(O.OracleError, match=msg):
        O.ensemble_adaptive(O.table_dist(radii, dens), [0.5], 1.5 + 0j)
    with pytest.raises(O.OracleError, match=msg):
        O.ensemble_fixed(O.table_dist(radii, dens), [0.5], 1.5 + 0j, 32)


def test_error_estimates_bound_the_true_errors():
    mu = np.array([1.0, 0.5, -0.2, -1.0])
    d = O.table_dist(*REF_TABLE)
    a = O.ensemble_adaptive(d, [0.4], 2.0 + 0.5j, mu=mu, greek_order=12, rtol=1e-6)
    b = O.ensemble_adaptive(d, [0.4], 2.0 + 0.5j, mu=mu, greek_order=12, rtol=1e-11,
                            max_panels=50_000)
    assert a["converged"][0] and b["converged"][0]
    true = np.abs(a["values"] - b["values"])
    assert np.all(true <= a["errors"] + 1e-14 * np.abs(b["values"]))
    for key in ("phase", "greek"):
        t = np.abs(a[key] - b[key])
        assert np.all(t <= 2.0 * a[key + "_err"] + 1e-13 * np.abs(b[key]).max())
    rel = lambda k: abs(a["values"][k, 0] / b["values"][k, 0] - 1)  # noqa: E731
    assert rel(0) <= 1e-6 and rel(1) <= 1e-6


def test_table_radii_are_panel_edges_of_a_batch():
    """A table batched with a lognormal: the table's kinks split the shared panels, so the
    batch matches each distribution alone within the error estimates."""
    d = O.join(O.table_dist(*REF_TABLE), O.dist(1, 0.2, 1.5))
    wl, m = [0.45, 0.8], [1.5 + 0.01j, 1.45 + 1e-4j]
    single = O.ensemble_adaptive(d, wl, m, greek_order=8)
    batch = O.ensemble_adaptive(d, wl, m, greek_order=8, batch=True)
    err = single["errors"] + batch["errors"]
    assert np.all(np.abs(single["values"] - batch["values"]) <= err + 1e-15)
