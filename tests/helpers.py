"""Shared test helpers: build a case once, feed identical arrays to the
oracle (CPU FP64 restatement) and to the product (C ABI)."""
import os

import numpy as np

from conftest import GOLDEN
from oracle import formats as F
from oracle import oracle as O

KCAL = 4184.0
MU_TOL = 0.01 * KCAL          # 0.01 kcal/mol in J/mol (the parity target)


def load_case(name, **over):
    """Case from a control file in tests/golden (centred like the reference)."""
    case, ctrl, sol = O.case_from_inp(os.path.join(GOLDEN, name + ".inp"))
    for k, v in over.items():
        setattr(case, k, v)
    return case, ctrl, sol


# the -e (ESP cube) case: control file it reuses
ESP_CASES = {"cfg0_esp": "cfg0_chain12"}


def esp_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_esp", os.path.join(GOLDEN, "make_esp.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def load_esp_case(name="cfg0_esp", cube=None):
    """The control file of ESP_CASES[name], uncentred (-e implies -f,
    main.cu:37-41), with the ESP cube of tests/golden/make_esp.py; `cube`
    (a path) writes the cube file too and reads the values back from it."""
    inp = os.path.join(GOLDEN, ESP_CASES[name] + ".inp")
    case, ctrl, sol = O.case_from_inp(inp, centering=False)
    mod = esp_module()
    if cube is None:
        _, _, case.esp = mod.esp_values(inp)
    else:
        mod.write_cube(inp, cube)
        case.esp = F.read_esp_cube(cube, case.grid)
    return case, ctrl, sol


def load_rmdft_case(name="rmdft_benzene64"):
    """An RMDFT control file with its .cvk (beside the .xvk) and the
    hard-sphere table rmdft_287.xsv (the -r input)."""
    case, ctrl, sol = O.case_from_inp(os.path.join(GOLDEN, name + ".inp"))
    case.cvv = F.read_cvk(os.path.join(GOLDEN, ctrl.fsolvent))
    case.hs = F.read_hard_sphere(os.path.join(GOLDEN, "rmdft_287.xsv"))
    return case, ctrl, sol


def product_solver(case, precision=0, **kw):
    import rism3d_b200 as R
    s = R.Solver(case.grid, case.box, closure=case.closure, convergence=case.conv,
                 maxstep=case.maxstep, an2=(case.count, case.m, case.mp),
                 precision=precision, **kw)
    s.set_solvent_obj(case.sv)
    if getattr(case, "cvv", None) is not None and getattr(case, "hs", None) is not None:
        hs = case.hs
        s.set_rmdft(case.cvv, hs.k, hs.chs, hs.w, hs.pfhs, hs.wfk0)
    if getattr(case, "esp", None) is not None:
        s.set_esp(case.esp)
    s.set_solute(case.sig, case.eps, case.q, case.xyz)
    return s


def ref_xmu(name):
    return F.parse_xmu(os.path.join(GOLDEN, "ref_b200", name + ".xmu"))


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
