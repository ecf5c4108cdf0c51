"""The multi-GPU form of the batch and serving paths is a partition of
independent solves over ranks with no data-path collective; only results
are gathered on the host.  Two gloo ranks on the CPU check that every rank
computes the same partition, that it covers each request exactly once and
balances the device bytes, and that the gathered results are complete."""
import os
import socket

import numpy as np
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


class OracleServer:
    """A serving loop over the FP64 oracle, for the multi-rank plumbing on
    the CPU: each pump advances every resident request by check_every RK4
    steps and finishes a relaxation when the last step's maximum torque is
    below the threshold (the same stop rule as the GPU server)."""

    def __init__(self, check_every=20):
        import oracle as O
        self.O, self.k, self.reqs, self.t0, self.next = O, check_every, {}, 0.0, 0

    def clock(self):
        import time
        return time.monotonic()

    def submit(self, params, m0, fields, max_torque, max_steps):
        raise NotImplementedError  # replaced per request below

    def pump(self):
        active = 0
        for rid, r in self.reqs.items():
            if r["done"]:
                continue
            r["sim"].steps(self.k)
            r["steps"] += self.k
            if r["sim"].torque() < r["max_torque"] or (r["max_steps"] and r["steps"] >= r["max_steps"]):
                r["done"] = True
                r["t_done"] = self.clock()
            else:
                active += 1
        return active, 0

    def result(self, rid):
        r = self.reqs[rid]
        return dict(state="done" if r["done"] else "active", converged=r["sim"].torque() < r["max_torque"],
                    steps=r["steps"], points_done=1, t_submit=0.0, t_admit=0.0, t_done=r["t_done"],
                    footprint=0, avg_m=r["sim"].avg_m()[None, :], point_steps=np.array([r["steps"]]))


def _tiny_stream():
    reqs = []
    for i, (nx, ny, b) in enumerate([(8, 8, 0.02), (16, 8, 0.05), (8, 4, 0.01), (12, 8, 0.03), (4, 8, 0.08),
                                     (16, 4, 0.04)]):
        cfg = dict(grid=(nx, ny, 1), cell=(3e-9, 3e-9, 3e-9), msat=8e5, aexch=1.3e-11, alpha=1.0,
                   bext=(b, 0.0, 0.0), solver="rk4", dt=2e-13)
        reqs.append(dict(index=i, arrival=0.0, kind="relax", cfg=cfg, fields=None, m_seed=(5, i)))
    return reqs


def _serve_main(rank, world, port, q):
    import importlib
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    if world > 1:
        dist.init_process_group("gloo", rank=rank, world_size=world)
    eng = importlib.import_module("1_b200")
    import oracle as O

    def make_server():
        sv = OracleServer()

        def submit(params, m0, fields, max_torque, max_steps):
            rid = sv.next
            sv.next += 1
            # the request's user-level configuration travels with its params
            cfg = submit.cfg[tuple(params.size)]
            sim = O.OracleSim(O.make_cfg(**cfg), m0, bits=64)
            sv.reqs[rid] = dict(sim=sim, steps=0, done=False, t_done=0.0, max_torque=max_torque,
                                max_steps=max_steps)
            return rid
        submit.cfg = {tuple(eng.mmx_params(**r["cfg"]).size): r["cfg"] for r in _tiny_stream()}
        sv.submit = submit
        return sv

    res = eng.serve_share(_tiny_stream(), rank, world, make_server, realtime=False, max_torque=1e-3,
                          max_steps=400)
    if rank == 0:
        q.put([(r["index"], r["rank"], r["steps"], r["avg_m"].tolist()) for r in res])
    if world > 1:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_rank_serving_matches_one_rank():
    """Each of two gloo ranks serves its share of a stream (an oracle-backed
    serving loop on the CPU), rank 0 gathers the results: every request is
    served exactly once, by the rank the partition names, with the same
    steps and <m> as when one rank serves the whole stream."""
    out = {}
    # tiny grids: one OpenMP thread per rank (the children read this at start)
    old_omp = os.environ.get("OMP_NUM_THREADS")
    os.environ["OMP_NUM_THREADS"] = "1"
    try:
        out = _run_worlds()
    finally:
        if old_omp is None:
            os.environ.pop("OMP_NUM_THREADS", None)
        else:
            os.environ["OMP_NUM_THREADS"] = old_omp
    one, two = out[1], out[2]
    assert [r[0] for r in two] == list(range(6))
    assert {r[1] for r in two} == {0, 1}
    for a, b in zip(one, two):
        assert a[0] == b[0] and a[2] == b[2]
        assert np.allclose(a[3], b[3], rtol=0, atol=0)


def _run_worlds():
    out = {}
    for world in (1, 2):
        ctx = mp.get_context("spawn")
        q = ctx.Queue()
        port = _free_port()
        procs = [ctx.Process(target=_serve_main, args=(r, world, port, q)) for r in range(world)]
        for p in procs:
            p.start()
        out[world] = q.get(timeout=240)
        for p in procs:
            p.join(timeout=60)
            assert p.exitcode == 0
    return out
