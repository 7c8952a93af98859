"""Writes the golden fixtures of this directory from the reference's Arb data.

The reference (usask-arg/scatrs) ships certified or high-precision values computed with Arb
ball arithmetic in ``reference/data/*.jsonl`` (each value as hi + lo + lo2 plus an error bound).
This script keeps the records on the ensemble path (homogeneous spheres, their Greek
coefficients, the derivatives of their coefficients and efficiencies, Gauss-Legendre rules, the
Wigner d functions the projection uses, layered spheres and their derivatives, spheroids'
T-matrices) as hi + lo pairs in compact JSON, so that the tests run without the reference tree.

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
    for name, recs in out.items():
        with open(os.path.join(HERE, f"{name}.json"), "w") as f:
            json.dump(recs, f, separators=(",", ":"))
        print(name, len(recs))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py path/to/reference")
    main(sys.argv[1])
