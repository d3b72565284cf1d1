"""The N > 1 replica path of bench.py on CPU: two ranks over gloo.

bench.py under torchrun runs one replica per GPU; its only collectives are
barriers and the reductions of hlld_ai_b200.replicas (the slowest rank's
time, the job's total work).  The same helpers run here on a gloo process
group of two CPU ranks, so the host-side logic is covered without a GPU:
the reductions, the whole-job rate of weak scaling, the per-rank seeds, and
a rank that fails before a collective ending its peer's wait with an error
rather than a hang.
"""
import json
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))


def _worker(rank, world, port, out_dir):
    _env(rank, world, port)
    from hlld_ai_b200 import replicas

    rp = replicas.from_env("cpu")
    replicas.init(rp, timeout_s=60)
    res = {
        "world": rp.world, "rank": rp.rank,
        "max": replicas.max_over_ranks(rp, rank + 1.0, -float(rank)),
        "sum": replicas.sum_over_ranks(rp, rank + 1.0, 10.0),
        # equal replicas, rank r took 10 (r + 1) ms for 100 units
        "rate": replicas.job_rate(rp, 100.0, 10.0 * (rank + 1)),
        "seed": replicas.replica_seed(20261203, rp),
    }
    replicas.barrier(rp)
    replicas.finish(rp)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as fh:
        json.dump(res, fh)


def _failing_worker(rank, world, port, out_dir):
    _env(rank, world, port)
    from hlld_ai_b200 import replicas

    rp = replicas.from_env("cpu")
    replicas.init(rp, timeout_s=20)
    if rank == 1:
        raise SystemExit(3)  # leaves before the collective, with none in flight
    try:
        replicas.max_over_ranks(rp, 1.0)
        outcome = "completed"
    except Exception as exc:  # the peer is gone: an error, not a hang
        outcome = "error: " + type(exc).__name__
    with open(os.path.join(out_dir, "rank0.json"), "w") as fh:
        json.dump({"outcome": outcome}, fh)


def test_two_gloo_ranks_reduce_like_the_bench(tmp_path):
    world, port = 2, _free_port()
    mp.start_processes(_worker, args=(world, port, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r, x in enumerate(res):
        assert x["world"] == 2 and x["rank"] == r
        assert x["max"] == [2.0, 0.0]
        assert x["sum"] == [3.0, 20.0]
        rate, ms = x["rate"]
        assert ms == 20.0  # the slowest rank's time
        assert rate == pytest.approx(2 * 100.0 / 20e-3)  # all ranks' units over it
    assert res[0]["seed"] != res[1]["seed"]


def test_a_rank_that_leaves_ends_its_peers_collective_with_an_error(tmp_path):
    world, port = 2, _free_port()
    with pytest.raises(Exception):
        mp.start_processes(_failing_worker, args=(world, port, str(tmp_path)), nprocs=world,
                           join=True, start_method="spawn")
    out = json.load(open(tmp_path / "rank0.json"))
    assert out["outcome"].startswith("error"), out
