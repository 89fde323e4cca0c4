"""Writes the seeded synthetic benchmark solutes as reference-format control
files (tests/golden/cfg*.inp), so the reference executable, the oracle and
the product all read identical inputs.  Solvent: h2o_vv.xvk (the reference's
own TIP3P-like water table) until the project's 1D XRISM tables replace it.
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "3d-rism-cuda_b200"))
from rism3d_b200 import synth  # noqa: E402


def main():
    synth.small_chain().write_inp(os.path.join(HERE, "cfg0_chain12.inp"))
    synth.globule().write_inp(os.path.join(HERE, "cfg1_globule300.inp"))
    p = synth.protein_like()
    p.write_inp(os.path.join(HERE, "cfg2_protein846_kh.inp"))
    p.write_inp(os.path.join(HERE, "cfg2_protein846_hnc.inp"), closure="HNC", maxstep=3000)


if __name__ == "__main__":
    main()
