"""The multi-GPU plumbing (replicas only) as two gloo ranks on CPU: the
process group aligns the ranks, the timed maximum is the maximum over ranks,
each replica gets its own seed and a disjoint round-robin share of the
requests, and a rank that never joins ends the others' wait with an error
instead of a hang."""
import json
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from weighted_bte_b200 import replicas

    r = replicas.init("gloo", timeout_s=60)
    r.barrier()
    result = {"max": r.max(10.0 * rank + 1.5), "seed": r.seed(1), "share": r.share(list(range(7))),
              "leader": r.leader}
    r.close()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(result, f)


def test_two_gloo_replicas(tmp_path):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    assert [x["max"] for x in res] == [11.5, 11.5]
    assert res[0]["seed"] != res[1]["seed"]
    assert res[0]["share"] == [0, 2, 4, 6] and res[1]["share"] == [1, 3, 5]
    assert [x["leader"] for x in res] == [True, False]


def _lonely_rank(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from weighted_bte_b200 import replicas

    try:
        replicas.init("gloo", timeout_s=5)
        outcome = "joined"
    except Exception as exc:  # noqa: BLE001 -- the missing peer must surface as an error
        outcome = type(exc).__name__
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(outcome, f)


def test_missing_replica_times_out(tmp_path):
    """Only rank 0 of two starts: its rendezvous ends with an error."""
    mp.spawn(_lonely_rank, args=(2, _free_port(), str(tmp_path)), nprocs=1, join=True)
    assert json.load(open(tmp_path / "rank0.json")) != "joined"


def test_single_replica_needs_no_process_group():
    from weighted_bte_b200 import replicas

    env = {k: os.environ.pop(k) for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK") if k in os.environ}
    try:
        r = replicas.init("gloo")
        assert (r.rank, r.world, r.leader) == (0, 1, True)
        assert r.max(3.0) == 3.0 and r.share([1, 2, 3]) == [1, 2, 3]
        r.barrier()
        r.close()
    finally:
        os.environ.update(env)
