"""The autotuner on a GPU: the work-division settings it may pick leave every output bit for bit
unchanged, the threshold it picks keeps the mixed form within its tolerance of the FP64 form, and
the settings are applied and cached."""

import json

import numpy as np
import pytest

from scatrs_b200 import _native, tune
from scatrs_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _run(w, i8_above=0):
    import torch

    dev = torch.device("cuda")
    n = w.dists.size * w.wavelengths.size
    wl = torch.from_numpy(w.wavelengths).to(dev)
    m = torch.from_numpy(np.ascontiguousarray(w.m).view(np.float64).reshape(-1).copy()).to(dev)
    v = torch.empty(11 * n, dtype=torch.float64, device=dev)
    p = torch.empty(6 * n * w.mu.size, dtype=torch.float64, device=dev)
    g = torch.empty(6 * n * (w.greek_order + 1), dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream()
    _native.ensemble_fixed_device(w.dists, wl.data_ptr(), w.wavelengths.size, m.data_ptr(), w.mu,
                                  w.n_nodes, w.greek_order, True, v.data_ptr(), p.data_ptr(),
                                  g.data_ptr(), s.cuda_stream, i8_above=i8_above)
    _native.check_errors(s.cuda_stream)
    return v.cpu().numpy(), p.cpu().numpy(), g.cpu().numpy()


def test_work_division_leaves_results_unchanged(gpu):
    w = W.batched_spheres(seed=3, scale=0.03)
    before = _native.get_tuning()
    try:
        outs = []
        for split, arena in ((1, 1 << 16), (4, 1 << 22), (16, 1 << 18), (64, 1 << 20)):
            _native.set_tuning(split, arena)
            outs.append(_run(w))
        for o in outs[1:]:
            for a, b in zip(outs[0], o):
                assert np.array_equal(a, b)
    finally:
        _native.set_tuning(before["split"], before["arena_rows"])


def test_autotune_picks_admissible_settings(gpu, tmp_path):
    w = W.batched_spheres(seed=4, scale=0.04)
    before = _native.get_tuning()
    cache = str(tmp_path / "tuning.json")
    try:
        t = tune.autotune_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, w.greek_order,
                                sample_wl=16, splits=(2, 4, 8), thresholds=(0, 32, 64),
                                repeats=1, cache=cache)
        assert t.split in (2, 4, 8) and t.i8_above in (0, 32, 64)
        assert _native.get_tuning() == {"split": t.split, "arena_rows": t.arena_rows}
        assert all(float(e) <= 1e-10 for k, e in t.errors.items() if int(k) == t.i8_above)
        # the chosen threshold on the whole workload: within the tolerance of the FP64 form
        ref, got = _run(w), _run(w, t.i8_above)
        n = w.dists.size * w.wavelengths.size
        assert tune.output_errors(ref, got, n, w.mu.size, w.greek_order) <= 1e-10
        # cached: a second call reads the stored settings
        with open(cache) as f:
            assert len(json.load(f)) == 1
        t2 = tune.autotune_fixed(w.dists, w.wavelengths, w.m, w.mu, w.n_nodes, w.greek_order,
                                 cache=cache)
        assert (t2.split, t2.arena_rows, t2.i8_above) == (t.split, t.arena_rows, t.i8_above)
    finally:
        _native.set_tuning(before["split"], before["arena_rows"])
