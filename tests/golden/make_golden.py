"""Generate the known-answer fixtures of the reference's unit tests.

The reference pins its reconstruction and EOS with these cases
(src/physics/hydro/tests/test_reconstruction.cpp:13-194,
src/physics/material_properties/eos/tests/test_eos.cpp:55-85):

* cell averages of the polynomial c = (10, 3, 1, 0.5) about x_c = 20, of order
  1 (PLM), 2 (PPM) and 3 (WENO-Z); the reconstructed face values must equal
  the polynomial's point values at -1/2 and +1/2 to 5e-6 relative;
* a steep tanh profile (steepness 10, 100-sample midpoint averages, offset
  0.25/100) whose reversed stencil must swap the two face values to 4 ulp;
* the ideal gas with gamma 1.4, Abar 1 at rho = P = 1: e_int = 1/0.4 to 1e-14,
  and the ener-mode call returns P = 1 exactly.

This script writes those inputs and exact answers to reconstruction_kat.json
and eos_kat.json.  Run: python tests/golden/make_golden.py
"""
import json
import math
from pathlib import Path

HERE = Path(__file__).resolve().parent
COEFFS = [10.0, 3.0, 1.0, 0.5, 0.0]
XC = 20.0
CASES = [("plm", "minmod", 1), ("plm", "mc", 1), ("plm", "van_leer", 1), ("ppm", "minmod", 2),
         ("ppm", "mc", 2), ("ppm", "van_leer", 2), ("wenoz", "van_leer", 3)]


def poly_avg(order: int, idx: int) -> float:
    v = COEFFS[0]
    for i in range(1, order + 1):
        v += COEFFS[i] / (i + 1) * ((idx + 0.5 - XC) ** (i + 1) - (idx - 0.5 - XC) ** (i + 1))
    return v


def poly(order: int, x: float) -> float:
    v = COEFFS[0]
    for i in range(1, order + 1):
        v += COEFFS[i] * (x - XC) ** i
    return v


def tanh_avg(idx: int, steep: float = 10.0) -> float:
    n = 100
    dx = 1.0 / n
    x0 = 0.25 * dx
    s = 0.0
    for i in range(n):
        x = idx - 0.5 + (i + 0.5) * dx
        s += math.tanh(steep * (x - x0))
    return s * dx


def main():
    recon = []
    for rc, lim, order in CASES:
        recon.append({
            "reconstruction": rc, "slope_limiter": lim, "order": order,
            "stencil": [poly_avg(order, i) for i in range(-2, 3)],
            "exact_minus": poly(order, -0.5), "exact_plus": poly(order, 0.5),
            "rel_tol": 5e-6,
            "tanh_stencil": [tanh_avg(i) for i in range(-2, 3)],
            "symmetry_ulps": 4,
        })
    (HERE / "reconstruction_kat.json").write_text(json.dumps(recon, indent=1))
    eos = {"gamma": 1.4, "Abar": 1.0, "rho": 1.0, "pres": 1.0, "eint": 1.0 / 0.4, "eint_tol": 1e-14,
           "pres_back_exact": 1.0}
    (HERE / "eos_kat.json").write_text(json.dumps(eos, indent=1))


if __name__ == "__main__":
    main()
