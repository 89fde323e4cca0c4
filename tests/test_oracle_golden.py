"""Pins the CPU FP64 oracle before it is trusted as the checker.

1. Against the reference executable itself, built from its own sources for
   sm_100a and run on a B200 (tests/golden/ref_b200, written by
   tests/golden/run_reference.py): the oracle reproduces the printed .xmu
   values (5 decimals) and the iteration counts.
2. Against the example goldens shipped with the reference
   (example/test*.xmu).  Those were written by an older reference build
   (different header, no SE lines), so they pin only to ~1e-3 relative.
"""
import json
import os

import numpy as np
import pytest

from helpers import load_case, ref_xmu
from oracle import formats as F
from oracle import oracle as O

KEYS = ["SFE_SC", "SFE_SC_HNC", "SFE_GF", "SE", "SE_LJ", "SE_ES", "PMV",
        "Pressure", "Correction_Term"]


def oracle_xmu(res, tmp_path, closure, natv):
    p = tmp_path / "o.xmu"
    O.write_xmu(res, str(p), closure, natv)
    return F.parse_xmu(str(p))


@pytest.mark.parametrize("name", ["test1", "test2", "cfg0_chain12"])
def test_oracle_reproduces_reference_binary(name, tmp_path, golden):
    case, _, _ = load_case(name)
    res = O.solve(case)
    summary = json.load(open(os.path.join(golden, "ref_b200", "summary.json")))
    assert res["iterations"] == summary[name]["iterations"]
    got = oracle_xmu(res, tmp_path, case.closure, case.sv.natv)
    ref = ref_xmu(name)
    for k in KEYS:
        # printed with 5 decimals; last-digit rounding plus FP64 summation order (~1e-10 relative on SE)
        assert abs(got[k] - ref[k]) <= 2e-5 + 2e-9 * abs(ref[k]), (k, got[k], ref[k])
    for i in range(case.sv.natv):
        k = "SFEC_SC(%d)" % i
        assert abs(got[k] - ref[k]) <= 2e-5 + 2e-9 * abs(ref[k])


@pytest.mark.parametrize("name", ["test1", "test2"])
def test_oracle_near_old_example_goldens(name, golden):
    case, _, _ = load_case(name)
    res = O.solve(case)
    old = F.parse_xmu(os.path.join(golden, name + ".xmu"))
    ib = res["ibeta"]
    assert abs(ib * res["xmu_sc"].sum() - old["SFE_SC"]) < 1e-3 * abs(old["SFE_SC"])
    assert abs(ib * res["xmu_gf"].sum() - old["SFE_GF"]) < 1e-3 * abs(old["SFE_GF"])
    assert abs(res["pmv"] * 1000 - old["PMV"]) < 1e-4
    assert abs(res["correction"] - old["Correction_Term"]) < 1e-3 * abs(old["Correction_Term"])


def test_tight_convergence_pins(golden):
    """conv 1e-9: the fixed point itself, independent of the stopping step."""
    case, _, _ = load_case("test1_tight")
    res = O.solve(case)
    ref = ref_xmu("test1_tight")
    summary = json.load(open(os.path.join(golden, "ref_b200", "summary.json")))
    # at 1e-9 the last step can land on either side of the threshold
    # (oracle 9.95e-10 at step 75, reference 1.0048e-9 then 2.8e-10 at 76)
    assert abs(res["iterations"] - summary["test1_tight"]["iterations"]) <= 1
    assert abs(res["ibeta"] * res["xmu_sc"].sum() - ref["SFE_SC"]) < 1e-3
