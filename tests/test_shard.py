"""Multi-rank host logic of the sharded k-point / cell solves (qumasun_b200/shard.py),
run as world_size-2 gloo process groups on the CPU: the longest-processing-time
assignment, and that every unit is solved exactly once with its result gathered on
rank 0 and no other collective."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from qumasun_b200.shard import lpt_assign, run_sharded, unit_cost


def test_lpt_assignment_covers_every_unit_once_and_balances():
    costs = [unit_cost(40 ** 3, 16, 8, complex_states=True)] * 64 + [unit_cost(80 ** 3, 128, 64)] * 3
    parts, loads = lpt_assign(costs, 4)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(costs)))
    assert max(loads) <= min(loads) + max(costs)  # LPT bound
    # deterministic: the same costs give the same assignment on every rank
    assert lpt_assign(costs, 4)[0] == parts


def test_lpt_single_rank_runs_largest_first():
    parts, loads = lpt_assign([1.0, 5.0, 3.0], 1)
    assert parts == [[1, 2, 0]] and loads == [9.0]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, costs, out_dir):
    import json
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    solved = []

    def solve(i):
        solved.append(i)
        return {"unit": i, "rank": rank, "value": i * i}

    res = run_sharded(costs, solve)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"solved": solved, "result": res}, f)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_ranks_gloo_solve_each_unit_once(tmp_path):
    import json
    costs = [float(c) for c in (5, 1, 4, 4, 2, 9, 3, 3, 7)]
    mp.spawn(_worker, args=(2, _free_port(), costs, str(tmp_path)), nprocs=2, join=True)
    r0 = json.load(open(tmp_path / "rank0.json"))
    r1 = json.load(open(tmp_path / "rank1.json"))
    assert r1["result"] is None
    assert sorted(r0["solved"] + r1["solved"]) == list(range(len(costs)))
    res = {int(k): v for k, v in r0["result"].items()}
    assert sorted(res) == list(range(len(costs)))
    parts, _ = lpt_assign(costs, 2)
    for rank, part in enumerate(parts):
        for i in part:
            assert res[i] == {"unit": i, "rank": rank, "value": i * i}
