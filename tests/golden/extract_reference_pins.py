"""Extract the golden values of MarineHydro.jl's own tests and of its
published sensitivity data into ``reference_pins.json``.

Run where a checkout of the reference exists (the tests only read the JSON);
the checkout's path is a required argument:

    python tests/golden/extract_reference_pins.py <path-to-MarineHydro.jl>

The values are parsed from the reference's files as text; nothing of the
reference is executed (Julia is not available).  Pins:

* test/greens_function.jl:81   Delhommeau dimensionless term and dG/dr at (r, z) = (1, -1)
* test/greens_function.jl:88-89  k*G and its gradient for e1 = (0,0,-1), e2 = (1,1,-2), k = 1
* test/consistency_with_analytical_solutions.jl:14-18  Hulme's hemisphere heave table
* paper/Plots/11_heuristics_dx_DELhommeau.csv, 11_heuristics_dr_DELhommeau.csv:
  the reference's Zygote gradients dA11/d(dx), dB11/d(dx) and dA11/dr,
  dB11/dr of two heaving 6 x 6 hemispheres (radius r = 1, body 2 centred at
  x = r + dx), omega = 1.03, Rankine + reflected + Wu, direct
  (paper/ArraySensitivities.jl:16-68, meshes from paper/meshGradients_pair.jl:7-15)
* paper/Plots/added_mass_data_dimensionless.csv, damping_data_dimensionless.csv:
  dA21/dr and dB21/dr (the force on body 2 from body 1's heave) on the grid
  dx/r in 1.5:0.5:8, kr in 0.5:1:9.5 with omega = sqrt(kr 9.8 / r), r = 1
  (the commented-out loops of paper/ArraySensitivities.jl:71-97)
"""
from __future__ import annotations

import csv
import json
import pathlib
import re
import sys


def _floats(s: str):
    return [float(x) for x in re.findall(r"[-+]?\d+\.\d+(?:[eE][-+]?\d+)?", s)]


def _csv(path: pathlib.Path) -> dict:
    with path.open() as f:
        rows = list(csv.reader(f))
    head, body = rows[0], [r for r in rows[1:] if r]
    return {h: [float(r[i]) for r in body] for i, h in enumerate(head)}


def extract(ref: pathlib.Path) -> dict:
    gf = (ref / "test" / "greens_function.jl").read_text()
    capy_ref = _floats(re.search(r"capy_ref\s*=\s*\[([^\]]*)\]", gf).group(1))
    g_line = re.search(r"capy_g\s*=\s*([^\n]*)", gf).group(1)
    g_vals = _floats(g_line)
    grad_line = re.search(r"capy_gradg\s*=\s*\[([^\]]*)\]", gf).group(1)
    grad_vals = _floats(grad_line)
    an = (ref / "test" / "consistency_with_analytical_solutions.jl").read_text()
    K = _floats(re.search(r"K_heave\s*=\s*\[([^\]]*)\]", an).group(1))
    A = _floats(re.search(r"A_heave\s*=\s*\[([^\]]*)\]", an).group(1))
    B = _floats(re.search(r"B_heave\s*=\s*\[([^\]]*)\]", an).group(1))
    plots = ref / "paper" / "Plots"
    dx = _csv(plots / "11_heuristics_dx_DELhommeau.csv")
    dr = _csv(plots / "11_heuristics_dr_DELhommeau.csv")
    am = _csv(plots / "added_mass_data_dimensionless.csv")
    dm = _csv(plots / "damping_data_dimensionless.csv")
    pair = {"radius": 1.0, "resolution": [6, 6], "omega": 1.03, "g_wavenumber": 9.81,
            "rho": 1000.0, "green_functions": "Rankine+RankineReflected+GFWu", "direct": True,
            "body2_center_x": "radius + dx"}
    return {
        "source": "MarineHydro.jl test suite and paper data (parsed as text)",
        "delhommeau_dimless_r1_zm1": {
            "cite": "test/greens_function.jl:81-83", "atol": 1e-4,
            "G": [capy_ref[0], capy_ref[1]], "dG_dr": [capy_ref[2], capy_ref[3]]},
        "delhommeau_greens_k1": {
            "cite": "test/greens_function.jl:88-92", "atol": 1e-4,
            "e1_center": [0.0, 0.0, -1.0], "e2_center": [1.0, 1.0, -2.0], "wavenumber": 1.0,
            "G": g_vals[:2],
            "grad_first_variable": [grad_vals[0:2], grad_vals[2:4], grad_vals[4:6]]},
        "hulme_heave": {
            "cite": "test/consistency_with_analytical_solutions.jl:14-18", "rtol": 0.1,
            "K": K, "A": A, "B": B},
        "pair_sensitivity_dx": dict(pair, cite="paper/Plots/11_heuristics_dx_DELhommeau.csv "
                                    "(paper/ArraySensitivities.jl:52-68)",
                                    dx=dx["dx"], dA11=dx["A11_grad_r"], dB11=dx["B11_grad_r"]),
        "pair_sensitivity_dr": dict(pair, cite="paper/Plots/11_heuristics_dr_DELhommeau.csv",
                                    dx=dr["dx"], dA11=dr["A11_grad_r"], dB11=dr["B11_grad_r"]),
        "pair_sensitivity_dimensionless": dict(
            pair, cite="paper/Plots/added_mass_data_dimensionless.csv, damping_data_dimensionless.csv "
            "(paper/ArraySensitivities.jl:71-97)", omega="sqrt(kr * 9.8 / radius)",
            dx_r_ratio=am["dx_r_ratio"], kr=am["kr"], dA21_dr=am["grad_r"], dB21_dr=dm["grad_r"]),
    }


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: extract_reference_pins.py <path-to-MarineHydro.jl>")
    out = pathlib.Path(__file__).resolve().parent / "reference_pins.json"
    out.write_text(json.dumps(extract(pathlib.Path(sys.argv[1])), indent=1) + "\n")
    print(out)
