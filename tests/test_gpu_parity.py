"""GPU parity: the CUDA solve path (through the C ABI) against the CPU FP64
oracle on identical inputs, and against the reference executable's own
outputs recorded on a B200 (tests/golden/ref_b200).

Tolerances: mu_ex within 0.01 kcal/mol (41.84 J/mol) and g(r) within 1e-4
relative, as the solve path requires; tighter informative bounds where
both sides run the same FP64 algorithm."""
import numpy as np
import pytest

from helpers import MU_TOL, load_case, product_solver, ref_xmu, rel_err
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def test1_oracle():
    case, _, _ = load_case("test1")
    return case, O.solve(case, want_grids=True)


def test_potential_grids_match_oracle():
    case, _, _ = load_case("cfg0_chain12")
    u, e, fr, fk = O.potentials(case)
    s = product_solver(case)
    import rism3d_b200 as R
    assert rel_err(s.grid_array(R.GRID_U), u) < 1e-11
    assert rel_err(s.grid_array(R.GRID_FR)[0], fr) < 1e-11
    assert rel_err(s.grid_array(R.GRID_E)[0], e) < 1e-11
    s.close()


def test_fp64_solve_test1_matches_oracle_and_reference(test1_oracle):
    case, o = test1_oracle
    s = product_solver(case)
    r = s.solve()
    ref = ref_xmu("test1")
    # same algorithm, same stopping rule: identical iteration count
    assert abs(r["iterations"] - o["iterations"]) <= 1
    assert abs(r["sfe_sc"] - o["sfe_sc"]) < 1.0
    assert abs(r["sfe_gf"] - o["sfe_gf"]) < 1.0
    assert abs(r["sfe_sc"] - ref["SFE_SC"]) < MU_TOL
    assert abs(r["sfe_sc_hnc"] - ref["SFE_SC_HNC"]) < MU_TOL
    assert abs(r["sfe_gf"] - ref["SFE_GF"]) < MU_TOL
    assert abs(r["pmv"] - ref["PMV"]) < 1e-4
    assert abs(r["se"] - ref["SE"]) < 1.0
    import rism3d_b200 as R
    g = s.grid_array(R.GRID_G)
    assert rel_err(g, o["g"]) < 1e-4
    h = s.grid_array(R.GRID_H)
    assert rel_err(h, o["h"]) < 1e-4
    s.close()


def test_fp64_solve_test2_matches_reference():
    case, _, _ = load_case("test2")
    s = product_solver(case)
    r = s.solve()
    ref = ref_xmu("test2")
    assert abs(r["sfe_sc"] - ref["SFE_SC"]) < MU_TOL
    assert abs(r["sfe_gf"] - ref["SFE_GF"]) < MU_TOL
    assert abs(r["pmv"] - ref["PMV"]) < 1e-4
    assert abs(r["correction"] - ref["Correction_Term"]) < 1.0
    s.close()


def test_mixed_precision_within_target(test1_oracle):
    case, o = test1_oracle
    import rism3d_b200 as R
    s = product_solver(case, precision=R.MIXED)
    r = s.solve()
    assert r["iterations_fp32"] > 0
    # FP64 work: the refinement base cycle and the confirming final cycle
    assert r["iterations"] - r["iterations_fp32"] <= 3
    assert abs(r["sfe_sc"] - o["sfe_sc"]) < MU_TOL
    assert rel_err(s.grid_array(R.GRID_G), o["g"]) < 1e-4
    s.close()


def test_forces_match_oracle(test1_oracle):
    case, o = test1_oracle
    s = product_solver(case)
    s.solve()
    dulj, due = s.forces()
    dv = case.box[0] * case.box[1] * case.box[2] / case.n
    assert np.allclose(dulj, o["dulj"] * dv, rtol=1e-6, atol=1e-6)
    assert np.allclose(due, o["due"] * dv, rtol=1e-6, atol=1e-6)
    s.close()


@pytest.mark.parametrize("name", ["cfg0_chain12", "cfg2_protein846_kh"])
def test_fused_axis_passes_match_the_cufft_path(name):
    """The FP32 phases of a mixed solve with the x and y axes of the
    transforms folded into the passes (RISM3D_XFFT=1: cuFFT along z only;
    64^3 and 256^3 cells) against the same solve through 3D cuFFT
    transforms: mu_ex and PMV within rounding of FP32 transforms.  The step
    counts agree to 10 %: the FP32 rounding of the bulk (and the order of
    its FP64 partial sums) moves where the bulk hands over to the
    refinement, and the AN2 trajectory after that point by tens of steps
    at 256^3, while the converged fixed point stays the same."""
    import os
    import rism3d_b200 as R
    case, _, _ = load_case(name)
    s0 = product_solver(case, precision=R.MIXED)
    r0 = s0.solve()
    s0.close()
    os.environ["RISM3D_XFFT"] = "1"
    try:
        s1 = product_solver(case, precision=R.MIXED)
    finally:
        del os.environ["RISM3D_XFFT"]
    r1 = s1.solve()
    s1.close()
    assert abs(r1["sfe_sc"] - r0["sfe_sc"]) < 0.1 * MU_TOL
    assert abs(r1["pmv"] - r0["pmv"]) < 1e-4
    assert abs(r1["iterations"] - r0["iterations"]) <= max(10, 0.1 * r0["iterations"]), \
        (r1["iterations"], r0["iterations"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pass_r_forms_agree(precision):
    """Pass R (residual, rms and the AN2 Gram sums) in its three forms on the
    same 64^3 solve: the plain grid-stride kernel (RISM3D_NO_PIPE_R=1), the
    cp.async pipeline (RISM3D_BULK_R=0) and the bulk-copy stream
    (RISM3D_BULK_R=1).  Only the order of the FP64 partial sums differs, so
    FP64 solves take the same steps to the same mu_ex (1e-6 J/mol); the
    mixed solves agree within the FP32 rounding of the bulk."""
    import os
    import rism3d_b200 as R
    case, _, _ = load_case("cfg0_chain12")
    prec = R.FP64 if precision == "fp64" else R.MIXED
    out = []
    for env in ({"RISM3D_NO_PIPE_R": "1"}, {"RISM3D_BULK_R": "0"}, {"RISM3D_BULK_R": "1"}):
        old = {k: os.environ.get(k) for k in env}
        os.environ.update(env)
        try:
            s = product_solver(case, precision=prec)
        finally:
            for k, v in old.items():
                if v is None:
                    del os.environ[k]
                else:
                    os.environ[k] = v
        out.append(s.solve())
        s.close()
    for r in out[1:]:
        if precision == "fp64":
            assert r["iterations"] == out[0]["iterations"]
            assert abs(r["sfe_sc"] - out[0]["sfe_sc"]) < 1e-6
        else:
            assert abs(r["sfe_sc"] - out[0]["sfe_sc"]) < 0.1 * MU_TOL
            assert abs(r["iterations"] - out[0]["iterations"]) <= max(10, 0.1 * out[0]["iterations"])


@pytest.mark.parametrize("name", ["cfg0_chain12", "cfg2_protein846_kh"])
def test_depth_m_anderson_bulk(name):
    """The opt-in depth-M Anderson accelerator of the FP32 bulk
    (RISM3D_MDIIS=M).  With M = 2 it is AN2's own update, so the mixed solve
    takes the AN2 form's steps (within the rounding of the FP64 Gram sums,
    which the two passes add in different orders) to the same mu_ex; with
    M = 5 it converges to the same fixed point (mu_ex within the FP32 bulk's
    reach of the AN2 result, the FP64 cycles gate both)."""
    import os
    import rism3d_b200 as R
    case, _, _ = load_case(name)
    s = product_solver(case, precision=R.MIXED)
    r_an2 = s.solve()
    s.close()
    out = {}
    for M in (2, 5):
        os.environ["RISM3D_MDIIS"] = str(M)
        try:
            s = product_solver(case, precision=R.MIXED)
        finally:
            del os.environ["RISM3D_MDIIS"]
        out[M] = s.solve()
        s.close()
    assert abs(out[2]["iterations"] - r_an2["iterations"]) <= max(3, 0.05 * r_an2["iterations"]), \
        (out[2]["iterations"], r_an2["iterations"])
    for M in (2, 5):
        assert abs(out[M]["sfe_sc"] - r_an2["sfe_sc"]) < 0.1 * MU_TOL, (M, out[M]["sfe_sc"], r_an2["sfe_sc"])
        assert abs(out[M]["pmv"] - r_an2["pmv"]) < 1e-4
