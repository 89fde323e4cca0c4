"""Multi-rank plumbing of the replica / batch-partition path on CPU: two
gloo ranks (127.0.0.1), the same calls bench.py makes under torchrun."""
import os
import socket

import pytest

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, costs, q):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "3d-rism-cuda_b200"))
    import torch.distributed as D
    from rism3d_b200 import replicas as RP
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    D.init_process_group("gloo", rank=rank, world_size=world)
    try:
        parts = RP.partition_by_cost(costs, world)
        mine = parts[rank]
        gathered = [None] * world
        D.all_gather_object(gathered, mine)
        t = 1.0 + rank                                 # a slower second rank
        q.put((rank, gathered, RP.max_over_ranks(t), RP.sum_over_ranks(len(mine)),
               RP.job_rate(len(mine), t)))
    finally:
        D.barrier()
        D.destroy_process_group()


def test_partition_covers_every_unit_once_and_balances():
    from rism3d_b200 import replicas as RP
    costs = [RP.solve_cost(g ** 3, a) for g, a in
             [(48, 10), (64, 20), (96, 40), (48, 8), (96, 33), (64, 12), (96, 15)] * 9]
    for world in (1, 2, 3, 8):
        parts = RP.partition_by_cost(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - sum(loads) / world <= max(costs)


@pytest.mark.timeout(120)
def test_two_gloo_ranks_agree_on_partition_time_and_rate():
    import torch.multiprocessing as mp
    from rism3d_b200 import replicas as RP
    costs = [RP.solve_cost(g ** 3, 10) for g in (48, 64, 96) * 20]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=90) for _ in procs]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, gathered, tmax, units, rate in out:
        assert sorted(i for part in gathered for i in part) == list(range(len(costs)))
        assert tmax == 2.0                      # the slower rank sets the time
        assert units == len(costs)
        assert abs(rate - len(costs) / 2.0) < 1e-12


def _fake_solve(i):
    """Stand-in for one solute's result dict (deterministic in i)."""
    return {"sfe_sc": 1000.0 + i, "sfe_sc_hnc": -2.0 * i, "sfe_gf": 0.5 * i, "pmv": 1e-4 * i,
            "pressure": 7.0, "correction": -i, "se": 3.0 * i, "se_lj": i, "se_es": 2.0 * i,
            "rms": 1e-7 * (i + 1), "iterations": 100 + i, "iterations_fp32": 90 + i,
            "status": i % 3}


def _gather_rank(rank, world, port, costs, q):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "3d-rism-cuda_b200"))
    import torch.distributed as D
    from rism3d_b200 import replicas as RP
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    D.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = RP.partition_by_cost(costs, world)[rank]
        res = [_fake_solve(i) for i in mine]      # this rank's "solves"
        q.put((rank, RP.gather_results(res, mine, len(costs))))
    finally:
        D.barrier()
        D.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_gather_per_solute_results_in_input_order():
    import torch.multiprocessing as mp
    from rism3d_b200 import replicas as RP
    # uneven parts: 61 solutes of mixed cost
    costs = [RP.solve_cost(g ** 3, 10) for g in (48, 64, 96) * 20] + [RP.solve_cost(96 ** 3, 40)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_rank, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=90) for _ in procs]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    want = [_fake_solve(i) for i in range(len(costs))]
    for rank, got in out:
        assert got == want


def test_gather_without_process_group_reorders_and_checks():
    from rism3d_b200 import replicas as RP
    idx = [3, 0, 2, 1]
    got = RP.gather_results([_fake_solve(i) for i in idx], idx, 4)
    assert got == [_fake_solve(i) for i in range(4)]
    with pytest.raises(ValueError):
        RP.gather_results([_fake_solve(0)], [0], 2)          # solute 1 missing
