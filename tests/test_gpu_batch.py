"""Batched solves of many small solutes (rism3d_solve_batch): every solute
of a mixed-size batch gets the result of its own single solve, and the
single solves agree with the oracle."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from helpers import MU_TOL
from oracle import formats as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _mols():
    import rism3d_b200.synth as S
    out = []
    for k, (g, L) in enumerate([(32, 16.0), (48, 24.0), (32, 16.0), (64, 32.0), (48, 24.0),
                                (64, 32.0), (32, 16.0)]):
        m = S.small_chain(seed=100 + k, natom=8 + 4 * k, grid=(g, g, g), box=(L, L, L))
        F.centre(m.xyz)
        out.append((m.sig, m.eps, m.q, m.xyz, g, L))
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_matches_single_solves(precision):
    import rism3d_b200 as R
    sv = F.read_xvk(os.path.join(GOLDEN, "h2o_vv.xvk"))
    mols = _mols()
    parent = R.Solver((32, 32, 32), (16.0, 16.0, 16.0), precision=precision)
    parent.set_solvent_obj(sv)
    res = parent.solve_batch(mols)
    res2 = parent.solve_batch(mols)               # cached children, same answers
    for i, (sig, eps, q, xyz, g, L) in enumerate(mols):
        s = R.Solver((g, g, g), (L, L, L), precision=precision)
        s.set_solvent_obj(sv)
        s.set_solute(sig, eps, q, xyz)
        r = s.solve()
        s.close()
        assert res[i]["status"] == 0
        assert abs(res[i]["sfe_sc"] - r["sfe_sc"]) < MU_TOL, i
        assert abs(res[i]["sfe_gf"] - r["sfe_gf"]) < MU_TOL, i
        assert abs(res[i]["pmv"] - r["pmv"]) < 1e-4, i
        assert abs(res[i]["se"] - r["se"]) < 1e-4 * abs(r["se"]) + 1e-3, i
        assert res2[i]["sfe_sc"] == res[i]["sfe_sc"]
    parent.close()


def test_sub_batches_give_the_same_results():
    """A cell's solutes split into sub-batches (batch_chunk_points = 2 x 32^3:
    the three 32^3 solutes run as sub-batches of two and one, the two 48^3
    and the two 64^3 ones one by one), each on its own child context and
    stream: the same results as one batch per cell."""
    import rism3d_b200 as R
    sv = F.read_xvk(os.path.join(GOLDEN, "h2o_vv.xvk"))
    mols = _mols()
    whole = R.Solver((32, 32, 32), (16.0, 16.0, 16.0))
    whole.set_solvent_obj(sv)
    ref = whole.solve_batch(mols)
    whole.close()
    split = R.Solver((32, 32, 32), (16.0, 16.0, 16.0), batch_chunk_points=2 * 32 ** 3)
    split.set_solvent_obj(sv)
    res = split.solve_batch(mols)
    split.close()
    for i in range(len(mols)):
        assert res[i]["status"] == 0
        assert abs(res[i]["sfe_sc"] - ref[i]["sfe_sc"]) < 1e-6 * abs(ref[i]["sfe_sc"]) + 1e-6, i
        assert abs(res[i]["iterations"] - ref[i]["iterations"]) <= 1, i


def test_batch_member_matches_oracle():
    import rism3d_b200 as R
    sv = F.read_xvk(os.path.join(GOLDEN, "h2o_vv.xvk"))
    mols = _mols()
    parent = R.Solver((32, 32, 32), (16.0, 16.0, 16.0))
    parent.set_solvent_obj(sv)
    res = parent.solve_batch(mols)
    parent.close()
    sig, eps, q, xyz, g, L = mols[1]
    o = O.solve(O.Case((g, g, g), (L, L, L), sv, sig, eps, q, xyz))
    assert abs(res[1]["sfe_sc"] - o["sfe_sc"]) < MU_TOL
    assert abs(res[1]["pmv"] - o["pmv"] * 1000) < 1e-4


def test_batch_config3_shapes_match_oracle():
    """Config-3 shapes: one batch of three molecules from the seeded
    256-molecule generator, one per grid class (48^3, 64^3 and 96^3 at
    0.5 A), in the 4-site water + 0.1 M NaCl table, FP32 bulk + FP64 polish.
    Every member, the 96^3 one included (outside the reference executable's
    valid sizes: its block reductions need power-of-two rows), matches the
    CPU FP64 oracle."""
    import rism3d_b200 as R
    import rism3d_b200.synth as S
    sv = F.read_xvk(os.path.join(GOLDEN, "naclaq_sub4_vv.xvk"))
    pick = {}
    for m in S.small_batch(seed=3, nmol=256):
        if m.grid[0] not in pick and m.natom <= 24:
            pick[m.grid[0]] = m
    mols = []
    for g in (48, 64, 96):
        m = pick[g]
        F.centre(m.xyz)
        mols.append((m.sig, m.eps, m.q, m.xyz, g, m.box[0]))
    parent = R.Solver((48, 48, 48), (24.0, 24.0, 24.0), precision=R.MIXED)
    parent.set_solvent_obj(sv)
    res = parent.solve_batch(mols)
    parent.close()
    for i, (sig, eps, q, xyz, g, L) in enumerate(mols):
        o = O.solve(O.Case((g, g, g), (L, L, L), sv, sig, eps, q, xyz))
        assert res[i]["status"] == 0, g
        assert abs(res[i]["sfe_sc"] - o["sfe_sc"]) < MU_TOL, (g, res[i]["sfe_sc"], o["sfe_sc"])
        assert abs(res[i]["sfe_gf"] - o["sfe_gf"]) < MU_TOL, g
        assert abs(res[i]["pmv"] - o["pmv"] * 1000) < 1e-4, g


def test_batch_child_cache_stays_within_its_budget():
    """Batch calls whose composition changes every call (as in a training
    loop with random batches) each need new sub-batch contexts; the idle
    ones are freed least recently used first once they hold more than
    RISM3D_BATCH_CACHE_BYTES, so device memory stops growing, and results
    stay those of fresh contexts."""
    import torch
    import rism3d_b200 as R
    sv = F.read_xvk(os.path.join(GOLDEN, "h2o_vv.xvk"))
    mols = _mols()
    small = [m for m in mols if m[4] == 32]
    os.environ["RISM3D_BATCH_CACHE_BYTES"] = str(64 << 20)
    try:
        parent = R.Solver((32, 32, 32), (16.0, 16.0, 16.0), batch_chunk_points=1 << 30)
        parent.set_solvent_obj(sv)
        ref = parent.solve_batch(small[:1])
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        used = []
        for k in range(1, 25):
            # k copies of the 32^3 solutes: a new composition every call
            batch = (small * k)[:k + 1]
            res = parent.solve_batch(batch)
            assert abs(res[0]["sfe_sc"] - ref[0]["sfe_sc"]) < 1e-6 * abs(ref[0]["sfe_sc"]) + 1e-6
            torch.cuda.synchronize()
            used.append(free0 - torch.cuda.mem_get_info()[0])
        parent.close()
    finally:
        del os.environ["RISM3D_BATCH_CACHE_BYTES"]
    # the last calls hold their own child plus at most the budget of idle ones
    per_solute = used[0] / 2.0
    assert used[-1] <= (64 << 20) + 30 * per_solute + (256 << 20), (used[-1], per_solute)
