"""Extract the golden values of MarineHydro.jl's own tests into
``reference_pins.json``.

Run (only where the reference checkout exists; the tests read the JSON):

    python tests/golden/extract_reference_pins.py /root/reference

The values are parsed from the reference test sources as text; nothing of the
reference is executed (Julia is not available).  Pins:

* test/greens_function.jl:81   Delhommeau dimensionless term and dG/dr at (r, z) = (1, -1)
* test/greens_function.jl:88-89  k*G and its gradient for e1 = (0,0,-1), e2 = (1,1,-2), k = 1
* test/consistency_with_analytical_solutions.jl:14-18  Hulme's hemisphere heave table
"""
from __future__ import annotations

import json
import pathlib
import re
import sys


def _floats(s: str):
    return [float(x) for x in re.findall(r"[-+]?\d+\.\d+(?:[eE][-+]?\d+)?", s)]


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
    return {
        "source": "MarineHydro.jl test suite (parsed as text)",
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
    }


if __name__ == "__main__":
    ref = pathlib.Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    out = pathlib.Path(__file__).resolve().parent / "reference_pins.json"
    out.write_text(json.dumps(extract(ref), indent=1) + "\n")
    print(out)
