"""Copies the reference's own example inputs and golden outputs into
tests/golden/ (run once in the build container, where the reference tree is
mounted; the GPU box only sees the committed copies).

Inputs: example/test{1..4}.inp (+ the _c/_s split form of test1),
example/h2o_vv.xvk.  Goldens: example/test{1..4}.xmu (written by an older
reference build; see the tolerance notes in tests/test_oracle_golden.py).
Also writes tight-convergence variants (``*_tight.inp``, conv 1e-9) used to
compare solutions at the fixed point rather than at the 1e-6 stopping point.
"""
import os
import shutil
import sys

# The reference checkout: $RISM3D_REFERENCE, by default where the build
# container mounts it.
REFERENCE = os.environ.get("RISM3D_REFERENCE", "/root/reference")
SRC = os.path.join(REFERENCE, "example")
DST = os.path.dirname(os.path.abspath(__file__))

FILES = ["test1.inp", "test2.inp", "test3.inp", "test4.inp", "test1_c", "test1_s",
         "h2o_vv.xvk", "test1.xmu", "test2.xmu", "test3.xmu", "test4.xmu"]


def tighten(src, dst, conv="1.0e-9"):
    tok_lines = open(src).read().split("\n")
    # line 4 (index 3) holds "convergence maxstep" (read_input.cu:46)
    parts = tok_lines[3].split()
    tok_lines[3] = " %s   %s" % (conv, parts[1])
    open(dst, "w").write("\n".join(tok_lines))


def subsample_xvk(src, dst, step=4):
    """Keep every `step`-th chi row (rows step-1, 2 step-1, ...): with the same
    dr and ntab/step rows, k_i = (i+1) pi / (dr ntab) lands on the kept rows."""
    lines = open(src).read().split("\n")
    h = lines[1].split()
    num, natv, ntab, dr = int(h[1]), int(h[2]), int(h[3]), float(h[4])
    head = lines[:num + 5]
    nnew = ntab // step
    head[1] = "##  %8d%8d%8d  %14.8f  %14.8f" % (num, natv, nnew, dr, 3.141592653589793 / (dr * nnew))
    data = " ".join(lines[num + 5:]).split()
    per = natv * natv
    rows = []
    for i in range(nnew):
        k = step * i + step - 1
        rows.append(" ".join(data[k * per:(k + 1) * per]))
    open(dst, "w").write("\n".join(head + rows) + "\n")


RMDFT_SRC = os.path.join(REFERENCE, "example_rmdft")


def rmdft_inputs():
    """RMDFT example (example_rmdft: benzene in water, hard-sphere table
    287.xsv), with the benzene atoms inline, on the example's own cell
    (64 A, 256^3) and on a 64^3 cell of 32 A for the CPU oracle.  The tables
    are copied whole: the reference leaves the hard-sphere rows of sites >= 1
    uninitialised (solvent_read.cc:124-127 allocates them with new[]), and
    only allocations as large as the example's 16384 rows came back zeroed
    in its runs; smaller tables gave it heap garbage."""
    for src, dst in (("h2o_vv.xvk", "rmdft_h2o_vv.xvk"), ("h2o_vv.cvk", "rmdft_h2o_vv.cvk"),
                     ("287.xsv", "rmdft_287.xsv")):
        shutil.copyfile(os.path.join(RMDFT_SRC, src), os.path.join(DST, dst))
    atoms = open(os.path.join(RMDFT_SRC, "benzene")).read().strip().split("\n")
    for name, box, grid in (("rmdft_benzene", 64, 256), ("rmdft_benzene64", 32, 64)):
        head = [" m    0  20220301", " KH", " rmdft_h2o_vv.xvk", " 1.0e-6   10000", " 2   0.6   0.2",
                "  %d  %d  %d" % (box, box, box), "  %d  %d  %d" % (grid, grid, grid)]
        open(os.path.join(DST, name + ".inp"), "w").write("\n".join(head + atoms) + "\n")


def main():
    if not os.path.isdir(SRC):
        sys.exit("reference examples not mounted")
    for f in FILES:
        shutil.copyfile(os.path.join(SRC, f), os.path.join(DST, f))
    subsample_xvk(os.path.join(SRC, "naclaq_vv.xvk"), os.path.join(DST, "naclaq_sub4_vv.xvk"))
    for name in ("test1", "test2"):
        tighten(os.path.join(DST, name + ".inp"), os.path.join(DST, name + "_tight.inp"))
    rmdft_inputs()


if __name__ == "__main__":
    main()
