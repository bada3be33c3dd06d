"""Member sharding of ensembles over ranks (ins2d_b200/ensembles.py) on the
CPU: the longest-first partition, and the world-size-2 gather of per-member
statistics over torch.distributed with the gloo backend (the multi-GPU path
shards members with no data-path collective; only statistics are gathered)."""
import os
import socket
import tempfile

import pytest

from ins2d_b200 import ensembles


def test_lpt_partition_covers_and_balances():
    members = ensembles.random_members(40, seed=9)
    costs = [ensembles.member_cost(kw) for kw in members]
    for nr in (1, 2, 3, 8):
        parts = ensembles.lpt_partition(costs, nr)
        flat = sorted(m for p in parts for m in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[m] for m in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)  # LPT bound
        assert parts == ensembles.lpt_partition(costs, nr)  # deterministic


def test_random_members_config():
    members = ensembles.random_members(16, seed=4)
    for m, kw in enumerate(members):
        nx, ny = len(kw["x"]) - 1, len(kw["y"]) - 1
        assert nx in (64, 96, 128, 192, 256) and ny in (64, 96, 128, 192, 256)
        assert 100.0 <= kw["Re"] <= 5000.0
        assert kw["BC"]["u"]["right"] == ("dir" if m % 2 == 0 else "pres")
        assert kw["CG_acc"] == 1e-10


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import json
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    members = ensembles.random_members(11, seed=3)
    costs = [ensembles.member_cost(kw) for kw in members]
    mine = ensembles.lpt_partition(costs, world)[rank]
    local = [dict(member=m, rank=rank, iters_total=7 * m) for m in mine]
    allst = ensembles.gather_stats(local, mine, len(members))
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as fh:
        json.dump(dict(mine=mine, all=allst), fh)
    dist.barrier()
    dist.destroy_process_group()


def test_gather_stats_two_ranks_gloo():
    import json
    import torch.multiprocessing as mp
    port = _free_port()
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(2, port, d), nprocs=2, join=True, start_method="spawn")
        res = [json.load(open(os.path.join(d, f"rank{r}.json"))) for r in range(2)]
    assert sorted(res[0]["mine"] + res[1]["mine"]) == list(range(11))
    assert not set(res[0]["mine"]) & set(res[1]["mine"])
    for r in range(2):
        allst = res[r]["all"]
        assert [s["member"] for s in allst] == list(range(11))
        assert all(s["iters_total"] == 7 * s["member"] for s in allst)
        assert all(s["rank"] == (0 if s["member"] in res[0]["mine"] else 1) for s in allst)
