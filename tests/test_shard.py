"""Solute-parallel batches over ranks (bgy3d_b200.shard): the cost partition,
and the shard / solve / gather protocol on two gloo ranks on the CPU (the
local solve replaced by a stand-in: solves never communicate, so the host
protocol is the whole multi-rank path)."""
import os
import socket

import pytest

from bgy3d_b200.shard import hnc3d_run_batch_sharded, shard, solve_cost


def test_shard_covers_and_balances():
    grids = [64, 72, 96, 108, 128, 144, 162, 192] * 8
    costs = [solve_cost({"N": n}) for n in grids]
    for world in (1, 2, 3, 4, 8):
        parts = shard(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)  # LPT bound
    assert shard([1.0, 1.0], 4)[2:] == [[], []]
    with pytest.raises(ValueError):
        shard([1.0], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import json

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    solutes = [[{"name": "X", "x": (float(i), 0.0, 0.0), "sigma": 3.0, "epsilon": 0.1, "charge": 0.0}]
               for i in range(7)]
    sets = [{"N": n} for n in (64, 192, 96, 128, 64, 144, 72)]
    seen = []

    def fake(sol, solvent, st, chi):
        seen.extend(int(s[0]["x"][0]) for s in sol)
        return [{"free-energy": -s[0]["x"][0], "N": t["N"], "rank": rank} for s, t in zip(sol, st)]

    res = hnc3d_run_batch_sharded(solutes, [], sets, None, solve=fake)
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump({"res": res, "seen": seen}, f)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_gather_every_solute(tmp_path):
    import json

    import torch.multiprocessing as mp
    mp.start_processes(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, start_method="spawn")
    outs = [json.load(open(tmp_path / f"r{r}.json")) for r in range(2)]
    assert outs[0]["res"] == outs[1]["res"]  # every rank holds the whole batch
    res = outs[0]["res"]
    assert [r["free-energy"] for r in res] == [-float(i) for i in range(7)]
    assert [r["N"] for r in res] == [64, 192, 96, 128, 64, 144, 72]
    assert sorted(outs[0]["seen"] + outs[1]["seen"]) == list(range(7))  # each solute solved once
    assert set(outs[0]["seen"]).isdisjoint(outs[1]["seen"])
    for i, r in enumerate(res):
        assert i in outs[r["rank"]]["seen"]
