"""Writes the golden fixtures of this directory from the reference's Arb data.

The reference (usask-arg/scatrs) ships certified or high-precision values computed with Arb
ball arithmetic in ``reference/data/*.jsonl`` (each value as hi + lo + lo2 plus an error bound).
This script keeps the records on the ensemble path (homogeneous spheres, their Greek
coefficients, the derivatives of their coefficients and efficiencies, Gauss-Legendre rules, the
Wigner d functions the projection uses, layered spheres and their derivatives, spheroids'
T-matrices) as hi + lo pairs in compact JSON, so that the tests run without the reference tree.

The refractive-index fixture (refractive.json) is the reference package's own models
(python/scatrs/refractive.py: Constant, Table linear and log_k, Cauchy, Sellmeier) evaluated here
with their derivatives at wavelengths on, between and at the ends of their nodes; the package is
imported with a stand-in for its compiled extension that holds only the constants it reads at
import (scatrs-py/src/lib.rs:17-50), since the models themselves are pure Python.

Run from the repository root:  python tests/golden/make_fixtures.py path/to/reference
"""

from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def pairs(o):
    """hi + lo of every value of one output (lo2 is below double-double precision)."""
    return [[h, l] for h, l in zip(o["hi"], o["lo"])]


def load(ref, name):
    with open(os.path.join(ref, "reference", "data", name)) as f:
        return [json.loads(line) for line in f]


def main(ref: str) -> None:
    out = {}
    mie = load(ref, "mie.jsonl")
    out["mie_coefficients"] = [
        {"case": r["case"], "x": r["inputs"]["x"], "m": [r["inputs"]["m_re"], r["inputs"]["m_im"]],
         "orders": r["inputs"]["orders"],
         **{k: pairs(r["outputs"][k]) for k in ("a_re", "a_im", "b_re", "b_im")}}
        for r in mie if r["case"].endswith(",coefficients")
    ]
    out["mie_series"] = [
        {"case": r["case"], "x": r["inputs"]["x"], "m": [r["inputs"]["m_re"], r["inputs"]["m_im"]],
         "mu": r["inputs"]["mu"],
         **{k: pairs(r["outputs"][k]) for k in
            ("q_ext", "q_sca", "q_abs", "q_back", "g", "s1_re", "s1_im", "s2_re", "s2_im")}}
        for r in mie if r["case"].endswith(",series")
    ]
    greek = load(ref, "mie_greek.jsonl")
    out["mie_greek"] = [
        {"case": r["case"], "x": r["inputs"]["x"], "m": [r["inputs"]["m_re"], r["inputs"]["m_im"]],
         "order": r["inputs"]["order"],
         **{k: pairs(r["outputs"][k]) for k in
            ("alpha1", "alpha2", "alpha3", "alpha4", "beta1", "beta2")}}
        for r in greek if r["case"].endswith(",greek")
    ]
    out["mie_phase"] = [
        {"case": r["case"], "x": r["inputs"]["x"], "m": [r["inputs"]["m_re"], r["inputs"]["m_im"]],
         "mu": r["inputs"]["mu"],
         **{k: pairs(r["outputs"][k]) for k in ("f11", "f12", "f33", "f34")}}
        for r in greek if r["case"].endswith(",phase")
    ]
    gl = load(ref, "gauss_legendre.jsonl")
    out["gauss_legendre"] = [
        {"n": r["inputs"]["n"], "nodes": pairs(r["outputs"]["nodes"]),
         "weights": pairs(r["outputs"]["weights"])}
        for r in gl if r["case"] == f"n={r['inputs']['n']}"
    ]
    wd = load(ref, "wigner_d.jsonl")
    out["wigner_d"] = [
        {"m": r["inputs"]["m"], "n": r["inputs"]["n"], "x": r["inputs"]["x"],
         "l_max": r["inputs"]["l_max"], "d": pairs(r["outputs"]["d"])}
        for r in wd
        if max(abs(r["inputs"]["m"]), abs(r["inputs"]["n"])) <= 2 and "l_max" in r["inputs"]
        and len(r["outputs"]["d"]["hi"]) == r["inputs"]["l_max"] + 1
    ]
    layered = load(ref, "layered.jsonl")
    out["layered_coefficients"] = [
        {"case": r["case"], "x": r["inputs"]["x"], "m_re": r["inputs"]["m_re"],
         "m_im": r["inputs"]["m_im"], "orders": r["inputs"]["orders"],
         **{k: pairs(r["outputs"][k]) for k in ("a_re", "a_im", "b_re", "b_im")}}
        for r in layered if r["case"].endswith(",coefficients")
    ]
    out["layered_series"] = [
        {"case": r["case"], "x": r["inputs"]["x"], "m_re": r["inputs"]["m_re"],
         "m_im": r["inputs"]["m_im"],
         **{k: pairs(r["outputs"][k]) for k in r["outputs"] if k.startswith("q_") or k == "g"}}
        for r in layered if r["case"].endswith(",series")
    ]
    md = load(ref, "mie_derivatives.jsonl")
    out["mie_coefficient_derivatives"] = [
        {"case": r["case"], "x": r["inputs"]["x"], "m": [r["inputs"]["m_re"], r["inputs"]["m_im"]],
         "orders": r["inputs"]["orders"], **{k: pairs(v) for k, v in r["outputs"].items()}}
        for r in md if r["case"].endswith(",coefficients")
    ]
    out["mie_jacobian"] = [
        {"case": r["case"], "x": r["inputs"]["x"], "m": [r["inputs"]["m_re"], r["inputs"]["m_im"]],
         **{k: pairs(v) for k, v in r["outputs"].items() if k.startswith(("q_", "g_"))}}
        for r in md if r["case"].endswith(",series")
    ]
    ld = load(ref, "layered_derivatives.jsonl")
    out["layered_derivatives"] = [
        {"case": r["case"], "x": r["inputs"]["x"], "m_re": r["inputs"]["m_re"],
         "m_im": r["inputs"]["m_im"], "orders": r["inputs"]["orders"],
         **{k: pairs(v) for k, v in r["outputs"].items()}}
        for r in ld
    ]
    sph = load(ref, "spheroid.jsonl")
    out["spheroid"] = [
        {"case": r["case"], "x": r["inputs"]["x"], "eps": r["inputs"]["aspect_ratio"],
         "m": [r["inputs"]["m_re"], r["inputs"]["m_im"]],
         "n_terms": r["inputs"].get("n_terms"), "n_theta": r["inputs"].get("n_theta"),
         **{k: pairs(v) for k, v in r["outputs"].items()}}
        for r in sph
    ]
    out["refractive"] = refractive_records(ref)
    for name, recs in out.items():
        with open(os.path.join(HERE, f"{name}.json"), "w") as f:
            json.dump(recs, f, separators=(",", ":"))
        print(name, len(recs))


def refractive_records(ref):
    """The reference's refractive-index models at test wavelengths: m and derivatives()."""
    import types

    import numpy as np

    ext = types.ModuleType("scatrs._scatrs")
    ext.__version__ = "0.3.0"
    for name, value in (("MAX_GAUSS_LEGENDRE_POINTS", 1 << 17), ("MAX_WIGNER_D_VALUES", 1 << 28),
                        ("MAX_MIE_ORDER", 1 << 20), ("MAX_MIE_VALUES", 1 << 27),
                        ("MAX_GREEK_ORDER", 1 << 21), ("MAX_LAYERS", 1 << 10),
                        ("MAX_TMATRIX_ORDER", 500)):
        setattr(ext, name, value)
    sys.modules["scatrs._scatrs"] = ext
    sys.path.insert(0, os.path.join(ref, "python"))
    from scatrs import refractive as R

    wl_nodes = [0.3, 0.45, 0.6, 1.1, 2.5]
    m_nodes = [1.52 + 1e-3j, 1.5 + 2e-4j, 1.49 + 5e-6j, 1.47 + 1e-7j, 1.44 + 4e-4j]
    lam = np.array([0.3, 0.31, 0.45, 0.5, 0.577, 0.6, 0.9, 1.1, 1.7, 2.49, 2.5])
    models = [
        (("constant", 1.53 + 0.008j), R.Constant(1.53 + 0.008j)),
        (("table", wl_nodes, m_nodes), R.Table(wl_nodes, m_nodes)),
        (("table_log_k", wl_nodes, m_nodes), R.Table(wl_nodes, m_nodes, interpolation="log_k")),
        (("cauchy", 1.458, 3.54e-3, 2.1e-5, 1e-6), R.Cauchy(1.458, 3.54e-3, 2.1e-5, 1e-6)),
        (("sellmeier", [0.6961663, 0.4079426, 0.8974794], [0.0684043 ** 2, 0.1162414 ** 2,
                                                           9.896161 ** 2], 2e-7),
         R.Sellmeier([0.6961663, 0.4079426, 0.8974794],
                     [0.0684043 ** 2, 0.1162414 ** 2, 9.896161 ** 2], 2e-7)),
    ]
    recs = []
    for spec, model in models:
        m = model.evaluate(lam)
        dm = model.derivatives(lam)
        recs.append({"spec": [spec[0]] + [
            [[float(z.real), float(z.imag)] for z in v] if spec[0].startswith("table") and i == 1
            else ([float(u) for u in v] if isinstance(v, list) else
                  ([float(v.real), float(v.imag)] if isinstance(v, complex) else float(v)))
            for i, v in enumerate(spec[1:])],
            "parameters": list(model.parameters), "wavelength": lam.tolist(),
            "m": m.view(np.float64).tolist(), "dm": dm.view(np.float64).tolist()})
    return recs


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py path/to/reference")
    main(sys.argv[1])
