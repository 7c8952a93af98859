"""The non-allocating batched Mie entry point (scatrs_mie_static) against the allocating one
(scatrs_mie), through the C ABI.

Callers that cannot allocate device memory (a plugin whose host process owns every device
allocation through its own pool, or a loop that must not allocate) pass device buffers for the
inputs and outputs; the scratch of the recurrences is a fixed array inside the library. The test
allocates its own device buffers (with torch) and calls the entry point twice in a row: both
calls must reproduce the allocating entry point's coefficients and efficiencies. This file runs
last (pytest collects it last), and passes alone in a fresh process as well.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12  # as tests/test_gpu_mie.py (the two entry points run the same arithmetic)


SENTINEL = 12345.678  # fills the padding around the coefficient buffer


def _call_static(lib, x, m, allow_unvalidated=0, total=None, off=None, pad=0):
    """One call with device buffers from torch; the coefficient buffer has `pad` terms of
    SENTINEL on both sides of the caller's [0, total) terms. Returns the status, the message,
    the term counts, the offsets, the coefficients (padding included) and the efficiencies."""
    import torch

    n = x.size
    nt = np.ceil(x + 6.0 * np.cbrt(x) + 3.0).astype(np.int64)
    if off is None:
        off = np.zeros(n, dtype=np.int64)
        off[1:] = np.cumsum(nt)[:-1]
    total = int(nt.sum()) if total is None else total
    dev = torch.device("cuda", 0)
    x_d = torch.tensor(x, dtype=torch.float64, device=dev)
    m_d = torch.tensor(m.view(np.float64), dtype=torch.float64, device=dev)
    off_d = torch.tensor(off, dtype=torch.int64, device=dev)
    nt_d = torch.zeros(n, dtype=torch.int64, device=dev)
    co_d = torch.full((4 * (max(total, 1) + 2 * pad),), SENTINEL, dtype=torch.float64,
                      device=dev)
    co_d[4 * pad:4 * (pad + total)] = 0.0
    eff_d = torch.zeros(5 * n, dtype=torch.float64, device=dev)
    err = ctypes.create_string_buffer(512)
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = lib.scatrs_mie_static(x_d.data_ptr(), m_d.data_ptr(), n, allow_unvalidated, total,
                               nt_d.data_ptr(), off_d.data_ptr(), co_d[4 * pad:].data_ptr(),
                               eff_d.data_ptr(), stream or None, err, 512)
    return st, err.value.decode(), nt_d.cpu().numpy(), off, co_d.cpu().numpy(), \
        eff_d.cpu().numpy().reshape(n, 5)


def test_static_entry_matches_allocating_entry_twice(gpu):
    rng = np.random.default_rng(11)
    x = np.concatenate([np.exp(rng.uniform(np.log(1e-3), np.log(400.0), 300)), [1500.0, 0.5]])
    m = (rng.uniform(1.33, 1.7, x.size) + 1j * np.exp(rng.uniform(np.log(1e-8), np.log(0.3),
                                                                    x.size)))
    ref_coeffs, ref_eff = gpu.mie(x, m)
    lib = gpu.load()
    for _ in range(2):
        st, msg, nt, off, co, eff = _call_static(lib, x, m)
        assert st == 0, msg
        c = co.view(np.complex128)
        for k in range(x.size):
            a = c[2 * off[k]:2 * off[k] + nt[k]]
            b = c[2 * off[k] + nt[k]:2 * off[k] + 2 * nt[k]]
            ra, rb = ref_coeffs[k]
            assert nt[k] == ra.size  # the allocating entry point's number of terms
            assert a.size == ra.size
            assert np.abs(a - ra).max() <= TOL * np.abs(ra).max()
            assert np.abs(b - rb).max() <= TOL * np.abs(rb).max()
        assert np.all(np.abs(eff - ref_eff) <= TOL * np.maximum(np.abs(ref_eff), 1e-300))


def test_static_entry_rejects_too_many_terms(gpu):
    lib = gpu.load()
    x = np.full(3, 5.0)
    m = np.full(3, 1.5 + 0.01j)
    st, msg, *_ = _call_static(lib, x, m, total=1 << 20)
    assert st == 1 and "static array" in msg
    from scatrs_b200.errors import OutsideValidatedDomainError  # noqa: F401

    st, msg, *_ = _call_static(lib, np.array([1.0]), np.array([1.5 + 20j]))
    assert st == 3, msg


@pytest.mark.parametrize("case", ["short_middle", "short_total", "negative"])
def test_static_entry_rejects_a_layout_that_does_not_hold_the_terms(gpu, case):
    """Offsets one term short for one sphere (or a total one term short, or a negative offset)
    must come back as SCATRS_INVALID_INPUT without a write outside the caller's buffer."""
    lib = gpu.load()
    x = np.array([3.0, 40.0, 7.5, 120.0])
    m = np.full(x.size, 1.45 + 0.003j)
    nt = np.ceil(x + 6.0 * np.cbrt(x) + 3.0).astype(np.int64)
    off = np.zeros(x.size, dtype=np.int64)
    off[1:] = np.cumsum(nt)[:-1]
    total = int(nt.sum())
    if case == "short_middle":
        off[2:] -= 1  # sphere 1's terms reach sphere 2's first one
        total -= 1
    elif case == "short_total":
        total -= 1  # the last sphere's terms pass the end
    else:
        off[0] = -1
    pad = 8
    st, msg, _, _, co, _ = _call_static(lib, x, m, total=total, off=off, pad=pad)
    assert st == 1, msg
    assert "layout" in msg
    assert np.all(co[:4 * pad] == SENTINEL)
    assert np.all(co[4 * (pad + total):] == SENTINEL)
