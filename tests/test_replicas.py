"""Replica plumbing on CPU: two gloo ranks (the N > 1 path of bench.py and of
the learned-correction training, without a GPU)."""
import json
import os
import socket

import torch
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from pmpp_b200 import replicas
    r, w, _ = replicas.setup("gloo", timeout_s=60)
    replicas.barrier(w)
    g = torch.tensor([float(r), 2.0 * r + 1.0])
    replicas.average_gradient(g, w)
    res = {"rank": r, "world": w, "max": replicas.max_over_ranks(10.0 * (r + 1), w),
           "sum": replicas.sum_over_ranks(r + 1, w), "avg": g.tolist(), "seed": replicas.replica_seed(1, r)}
    with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
        json.dump(res, f)
    replicas.teardown(w)


def test_two_gloo_ranks(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r, d in enumerate(res):
        assert d["rank"] == r and d["world"] == world
        assert d["max"] == 20.0 and d["sum"] == 3.0
        assert d["avg"] == [0.5, 2.0]
    assert res[0]["seed"] != res[1]["seed"]


def test_single_process_is_identity():
    from pmpp_b200 import replicas
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        os.environ.pop(k, None)
    r, w, _ = replicas.setup()
    assert (r, w) == (0, 1)
    g = torch.tensor([3.0])
    assert replicas.average_gradient(g, w).item() == 3.0
    assert replicas.max_over_ranks(2.5, w) == 2.5
