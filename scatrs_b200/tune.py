"""Autotuner of the fixed-grid ensemble's work division and of the mixed form's threshold.

The fixed-grid entries cut each call into slabs (an arena of coefficient rows) and each unit's
table-row tiles into work items (scatrs_set_tuning: ``arena_rows``, ``split``); neither changes a
result, only how the work lands on the SMs. The mixed form's ``i8_above`` decides which chunks
run as int8 digit products: it changes the outputs within the mixed form's tolerance. The right
values depend on the workload's spread of sizes (chunks with few terms favour the FP64 path) and
on the device, so they are measured: ``autotune_fixed`` times candidate settings on a sample of
the caller's own workload (a strided subset of its wavelengths, every distribution), keeps the
fastest split and arena whose outputs equal the default settings' bit for bit, then the fastest
threshold whose outputs stay within ``tol`` of the FP64 form's, applies them and returns them. A
JSON cache keyed by the device and the workload's shape makes later calls free.

The reference has no counterpart (its batch runs on host threads with fixed band widths); the
band widths themselves are part of its numerics (the projection's quadrature per band,
scatrs/src/engine.rs:951-1017) and are not tuned.
"""

from __future__ import annotations

import json
import os
from dataclasses import dataclass, field

import numpy as np

from . import _native

DEFAULT_SPLITS = (2, 4, 8, 16)
# A sample of a workload usually fits one slab, where the arena size changes nothing; the
# default searches only the split, and callers with many slabs may pass arenas to search.
DEFAULT_ARENAS = (1 << 22,)
DEFAULT_THRESHOLDS = (0, 16, 24, 32, 48, 64, 96)


@dataclass
class Tuned:
    split: int
    arena_rows: int
    i8_above: int
    ms: dict = field(default_factory=dict)  # candidate -> milliseconds per call on the sample
    errors: dict = field(default_factory=dict)  # threshold -> worst error vs the FP64 form
    sample_units: int = 0

    def as_dict(self) -> dict:
        return {"split": self.split, "arena_rows": self.arena_rows, "i8_above": self.i8_above,
                "ms": self.ms, "errors": self.errors, "sample_units": self.sample_units}


def output_errors(ref: tuple, got: tuple, n_units: int, n_mu: int, order: int) -> float:
    """The worst error of one form's outputs against another's, in the measures of the parity
    tests: the scalars relative to themselves, the phase matrix relative to each unit's largest
    F11, the Greek coefficients relative to each unit's alpha_1 at order 0."""
    rv, rp, rg = ref
    gv, gp, gg = got
    worst = float(np.max(np.abs(gv - rv) / np.maximum(np.abs(rv), 1e-300)))
    if n_mu > 0:
        rp = rp.reshape(6, n_units, n_mu)
        gp = gp.reshape(6, n_units, n_mu)
        scale = np.maximum(np.abs(rp[0]).max(axis=1), 1e-300)[None, :, None]
        worst = max(worst, float(np.max(np.abs(gp - rp) / scale)))
    if order >= 0:
        rg = rg.reshape(6, n_units, order + 1)
        gg = gg.reshape(6, n_units, order + 1)
        scale = np.maximum(np.abs(rg[0, :, 0]), 1e-300)[None, :, None]
        worst = max(worst, float(np.max(np.abs(gg - rg) / scale)))
    return worst


def choose(ms: dict, identical: dict, default):
    """The fastest candidate whose outputs equal the default's (work-division settings)."""
    ok = [c for c in ms if identical.get(c, False) or c == default]
    return min(ok, key=lambda c: (ms[c], c != default))


def choose_threshold(ms: dict, errors: dict, tol: float) -> int:
    """The fastest threshold whose outputs are within tol of the FP64 form's (0 = FP64 always
    qualifies)."""
    ok = [t for t in ms if t == 0 or errors.get(t, np.inf) <= tol]
    return min(ok, key=lambda t: (ms[t], t))


def sample_wavelengths(n_wl: int, target: int) -> np.ndarray:
    """A strided subset of about `target` wavelength indices (all when n_wl <= target), so that
    the sample spans the whole range of sizes x = 2 pi r / lambda."""
    if n_wl <= target:
        return np.arange(n_wl)
    return np.unique(np.linspace(0, n_wl - 1, target).round().astype(np.int64))


def _signature(dists, wavelengths, n_nodes, n_mu, order) -> str:
    r_lo = float(np.min(dists["r_lo"])) if dists.size else 0.0
    r_hi = float(np.max(dists["r_hi"])) if dists.size else 0.0
    return (f"n_dist={dists.size},n_wl={len(wavelengths)},n_nodes={n_nodes},n_mu={n_mu},"
            f"L={order},x=[{2 * np.pi * r_lo / max(wavelengths):.3g},"
            f"{2 * np.pi * r_hi / min(wavelengths):.3g}]")


def autotune_fixed(dists, wavelengths, m, mu, n_nodes: int, greek_order: int, *,
                   sample_wl: int = 64, splits=DEFAULT_SPLITS, arenas=DEFAULT_ARENAS,
                   thresholds=DEFAULT_THRESHOLDS, levels: int = 0, tol: float = 1e-10,
                   repeats: int = 2, cache: str | None = None, apply: bool = True) -> Tuned:
    """Times the fixed-grid ensemble (normalized outputs) on a sample of this workload for the
    candidate settings and returns (and, with apply, sets) the fastest admissible ones."""
    import torch

    _native.require_device()
    dists = np.ascontiguousarray(dists, dtype=_native.DIST_DTYPE)
    wavelengths = np.ascontiguousarray(wavelengths, dtype=np.float64)
    m = np.ascontiguousarray(m, dtype=np.complex128).reshape(dists.size, wavelengths.size)
    mu = np.zeros(0) if mu is None else np.ascontiguousarray(mu, dtype=np.float64)
    dev_name = torch.cuda.get_device_name()
    key = dev_name + "|" + _signature(dists, wavelengths, n_nodes, mu.size, greek_order)
    if cache and os.path.exists(cache):
        with open(cache) as f:
            stored = json.load(f).get(key)
        if stored is not None:
            t = Tuned(stored["split"], stored["arena_rows"], stored["i8_above"], stored["ms"],
                      stored["errors"], stored["sample_units"])
            if apply:
                _native.set_tuning(t.split, t.arena_rows)
            return t

    idx = sample_wavelengths(wavelengths.size, sample_wl)
    wl_s = wavelengths[idx]
    m_s = np.ascontiguousarray(m[:, idx])
    n_units = dists.size * wl_s.size
    dev = torch.device("cuda")
    wl_d = torch.from_numpy(wl_s).to(dev)
    m_d = torch.from_numpy(m_s.view(np.float64).reshape(-1).copy()).to(dev)
    v_d = torch.empty(11 * n_units, dtype=torch.float64, device=dev)
    p_d = torch.empty(max(1, 6 * n_units * mu.size), dtype=torch.float64, device=dev)
    g_d = torch.empty(max(1, 6 * n_units * (greek_order + 1)), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()

    def run(i8_above: int) -> tuple[float, tuple]:
        def call():
            _native.ensemble_fixed_device(dists, wl_d.data_ptr(), wl_s.size, m_d.data_ptr(), mu,
                                          n_nodes, greek_order, True, v_d.data_ptr(),
                                          p_d.data_ptr() if mu.size else 0,
                                          g_d.data_ptr() if greek_order >= 0 else 0,
                                          stream.cuda_stream, i8_above=i8_above, levels=levels)
        call()  # warm-up (tables, buffers)
        _native.check_errors(stream.cuda_stream)
        best = np.inf
        for _ in range(repeats):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            call()
            e.record(stream)
            e.synchronize()
            best = min(best, s.elapsed_time(e))
        _native.check_errors(stream.cuda_stream)
        out = (v_d.cpu().numpy().copy(), p_d.cpu().numpy().copy() if mu.size else None,
               g_d.cpu().numpy().copy() if greek_order >= 0 else None)
        return best, out

    before = _native.get_tuning()
    ms: dict = {}
    try:
        # 1. Work division on the FP64 form: results must not change (bit for bit).
        _native.set_tuning(0, 0)
        _, ref = run(0)
        identical = {}
        for sp in splits:
            for ar in arenas:
                _native.set_tuning(sp, ar)
                t, out = run(0)
                ms[f"split={sp},arena={ar}"] = t
                identical[(sp, ar)] = all(
                    (a is None and b is None) or np.array_equal(a, b) for a, b in zip(ref, out))
        times = {(sp, ar): ms[f"split={sp},arena={ar}"] for sp in splits for ar in arenas}
        split, arena = choose(times, identical, (4, 1 << 22) if (4, 1 << 22) in times else None)
        _native.set_tuning(split, arena)
        # 2. The mixed form's threshold, against the FP64 outputs of the same settings.
        tms, errs = {}, {}
        for th in thresholds:
            t, out = run(th)
            tms[th] = t
            errs[th] = 0.0 if th == 0 else output_errors(ref, out, n_units, mu.size, greek_order)
            ms[f"i8_above={th}"] = t
        i8_above = choose_threshold(tms, errs, tol)
    finally:
        if not apply:
            _native.set_tuning(before["split"], before["arena_rows"])
    tuned = Tuned(int(split), int(arena), int(i8_above), ms, {str(k): v for k, v in errs.items()},
                  n_units)
    if apply:
        _native.set_tuning(tuned.split, tuned.arena_rows)
    if cache:
        stored = {}
        if os.path.exists(cache):
            with open(cache) as f:
                stored = json.load(f)
        stored[key] = tuned.as_dict()
        with open(cache, "w") as f:
            json.dump(stored, f, indent=1)
    return tuned
