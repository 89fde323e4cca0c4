"""Writes the seeded synthetic benchmark solutes as reference-format control
files (tests/golden/cfg*.inp), so the reference executable, the oracle and
the product all read identical inputs, and the workloads' solvent table
tip3p_cfg_vv.xvk: rigid 3-site water (O q -0.834, sigma 3.1507 A, eps 0.1521
kcal/mol; H q +0.417, sigma 0.4 A, eps 0.046 kcal/mol; OH 0.9572 A, HOH
104.52 deg) at 298.15 K and 0.03334 molecules/A^3, chi_vv(k) from the
library's own 1D XRISM-KH solve (4096 points, dr 0.05 A).

    python tests/golden/make_configs.py
"""
import math
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "3d-rism-cuda_b200"))
from rism3d_b200 import synth  # noqa: E402

KCAL = 4184.0
AVOGADRO = 6.02214076e23
SOLVENT = "tip3p_cfg_vv.xvk"


def water_sites():
    rho_m = 0.03334 / (AVOGADRO * 1e-27)          # molecules/A^3 -> mol/L
    l, half = 0.9572, math.radians(104.52) / 2
    hy, hz = l * math.sin(half), l * math.cos(half)
    return [("O", 1, 1, 3.1507, 0.1521 * KCAL, -0.834, 0.0, 0.0, 0.0, rho_m),
            ("H", 1, 2, 0.4, 0.046 * KCAL, 0.417, 0.0, hy, hz, rho_m),
            ("H", 1, -2, 0.4, 0.046 * KCAL, 0.417, 0.0, -hy, hz, rho_m)]


def write_solvent():
    from rism3d_b200 import xrism1d as X
    rows = water_sites()
    xvv, xt, it = X.solve(rows, 298.15, 4096, 0.05, convergence=1e-12)
    X.write_xvk(os.path.join(HERE, SOLVENT), rows, 298.15, xvv, xt, 4096, 0.05)
    print("%s: %d steps, chi_T %.8e 1/Pa" % (SOLVENT, it, xt))


def main():
    write_solvent()
    synth.small_chain().write_inp(os.path.join(HERE, "cfg0_chain12.inp"), xvk=SOLVENT)
    synth.globule().write_inp(os.path.join(HERE, "cfg1_globule300.inp"), xvk=SOLVENT)
    p = synth.protein_like()
    p.write_inp(os.path.join(HERE, "cfg2_protein846_kh.inp"), xvk=SOLVENT)
    p.write_inp(os.path.join(HERE, "cfg2_protein846_hnc.inp"), closure="HNC", maxstep=3000,
                xvk=SOLVENT)


if __name__ == "__main__":
    main()
