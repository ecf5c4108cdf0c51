"""The multi-GPU form of the batch and serving paths is a partition of
independent solves over ranks with no data-path collective; only results
are gathered on the host.  Two gloo ranks on the CPU check that every rank
computes the same partition, that it covers each request exactly once and
balances the device bytes, and that the gathered results are complete."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import importlib
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    eng = importlib.import_module("1_b200")
    reqs = eng.serve_stream(64, seed=5)
    part = eng.partition_requests(reqs, world)
    mine = [r["index"] for r, k in zip(reqs, part) if k == rank]
    load = sum(eng.footprint(eng.mmx_params(**reqs[i]["cfg"])) * (1 if reqs[i]["fields"] is None
                                                                   else len(reqs[i]["fields"])) for i in mine)
    parts = [None] * world
    dist.all_gather_object(parts, part)
    got = [None] * world
    dist.gather_object((mine, load), got if rank == 0 else None, dst=0)
    if rank == 0:
        q.put((parts, got))
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_rank_partition_and_gather():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    parts, got = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert parts[0] == parts[1]
    ids = sorted(i for mine, _ in got for i in mine)
    assert ids == list(range(64))
    loads = [ld for _, ld in got]
    assert max(loads) <= 1.5 * min(loads)
