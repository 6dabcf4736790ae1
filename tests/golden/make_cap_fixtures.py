"""Writes cap_justrelax.json: the pinned JustRelax tensile-cap return-map rows of the
reference's test/test_drucker_prager_cap.jl ("Pinned JustRelax cap fixtures"), read from
that file's text. Run where a FEMTools.jl checkout is present, naming its root:

    python tests/golden/make_cap_fixtures.py path/to/FEMTools.jl

Each row: (ψ in degrees, η_reg, s_trial, p_trial, τII, P, λ, θdot) for C = η = G = Δt = 1,
K = 4, ϕ = 30°, pT = −0.5 and ηve = 0.5 (the reference calls
cap_return_map(s_trial, p_trial, 0.5, 4.0, sinpi(1/6), sind(ψ), cospi(1/6), −0.5, η_reg)).
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    text = open(os.path.join(ref_root, "test", "test_drucker_prager_cap.jl")).read()
    block = text[text.index('@testset "Pinned JustRelax cap fixtures"'):]
    block = block[block.index("fixtures = ("):block.index("\n    )\n")]
    rows = [tuple(float(x) for x in m.split(","))
            for m in re.findall(r"\(([-0-9.e, ]+)\)", block)]
    assert len(rows) == 16 and all(len(r) == 8 for r in rows), rows
    out = {"source": "test/test_drucker_prager_cap.jl, testset \"Pinned JustRelax cap fixtures\"",
           "columns": ["psi_deg", "eta_reg", "s_trial", "p_trial", "tau_II", "P", "lambda", "theta_dot"],
           "eta_ve": 0.5, "K_dt": 4.0, "phi_deg": 30.0, "pT": -0.5, "rtol": 1e-12, "atol": 1e-14,
           "rows": rows}
    rows_txt = ",\n  ".join(json.dumps(r) for r in rows)
    head = json.dumps({k: v for k, v in out.items() if k != "rows"})[:-1]
    with open(os.path.join(HERE, "cap_justrelax.json"), "w") as f:
        f.write(head + ',\n "rows": [\n  ' + rows_txt + "\n ]\n}\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_cap_fixtures.py path/to/FEMTools.jl")
    main(sys.argv[1])
