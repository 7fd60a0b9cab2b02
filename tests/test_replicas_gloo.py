"""Multi-rank host logic on CPU: two gloo ranks agree on the slowest time and the whole-job rate,
get distinct replica seeds, and split tenants so every tenant has exactly one owner."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from gpusketch_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        r, w, lr = replicas.env_rank()
        replicas.barrier(dist)
        ms = 100.0 + 50.0 * r                  # rank 1 is the slow one
        ms_max = replicas.max_over_ranks(ms, dist)
        units = replicas.sum_over_ranks(1000.0 * (r + 1), dist)
        out.put({"rank": r, "world": w, "local": lr, "ms_max": ms_max, "units": units,
                 "rate": replicas.whole_job_rate(units, ms_max), "seed": replicas.replica_seed(0x5EED0002, r),
                 "tenants": replicas.tenant_shard(7, r, w)})
        replicas.barrier(dist)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in range(world)), key=lambda d: d["rank"])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [d["rank"] for d in res] == [0, 1] and all(d["world"] == 2 for d in res)
    assert all(d["ms_max"] == 150.0 for d in res)            # max over ranks, seen by every rank
    assert all(d["units"] == 3000.0 for d in res)
    assert all(d["rate"] == pytest.approx(3000.0 / 0.150) for d in res)
    assert res[0]["seed"] != res[1]["seed"]
    owned = sorted(res[0]["tenants"] + res[1]["tenants"])
    assert owned == list(range(7)) and not set(res[0]["tenants"]) & set(res[1]["tenants"])


def test_single_process_defaults(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert replicas.env_rank() == (0, 1, 0)
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.whole_job_rate(1e9, 500.0) == 2e9
