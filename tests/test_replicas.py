"""Replica scheduling across ranks: assignment on one process, and the
multi-rank path (share, max-over-ranks timing, gather) as two gloo ranks on
the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from dvc_b200 import replicas


def test_plan_is_a_balanced_partition():
    costs = [5, 1, 1, 1, 1, 4, 3, 2, 2, 8]
    for world in (1, 2, 3, 8, 16):
        p = replicas.plan(costs, world)
        assert len(p) == world
        flat = sorted(i for r in p for i in r)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in r) for r in p]
        # greedy least-loaded: no rank exceeds the lightest by more than the largest job
        assert max(loads) - min(loads) <= max(costs)
    with pytest.raises(ValueError):
        replicas.plan(costs, 0)


def test_single_process_collectives_are_identity():
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.gather({"a": 1}) == [{"a": 1}]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, costs, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        mine = replicas.share(costs, rank, world)
        # each rank "decodes" its streams; the step time is the slowest rank's
        t = float(sum(costs[i] for i in mine))
        slowest = replicas.max_over_ranks(t)
        shares = replicas.gather(mine)
        q.put((rank, mine, t, slowest, shares))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_cover_every_stream_once():
    costs = [7, 3, 3, 2, 9, 1, 4, 4]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, costs, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    shares = out[0][4]
    assert out[1][4] == shares
    assert sorted(i for s in shares for i in s) == list(range(len(costs)))
    assert [o[1] for o in out] == shares
    assert out[0][3] == out[1][3] == max(o[2] for o in out)


class _FakeServer:
    """A server that finishes every request at the next poll, echoing the item."""

    def __init__(self):
        self.pending, self.done, self.n = [], {}, 0

    def submit(self, item):
        self.n += 1
        self.pending.append((self.n, item))
        return self.n

    def poll(self):
        k = len(self.pending)
        for t, it in self.pending:
            self.done[t] = {"recon": it["x"], "latency_ms": 1.0}
        self.pending = []
        return k

    def finished(self):
        return sorted(self.done)

    def result(self, t):
        return self.done.pop(t)

    def close(self):
        pass


def test_multi_server_pins_streams_and_balances_devices():
    ms = replicas.MultiServer([_FakeServer(), _FakeServer(), _FakeServer()])
    costs = {0: 5.0, 1: 1.0, 2: 1.0, 3: 4.0, 4: 1.0}
    tickets = {}
    for rnd in range(3):
        for s, c in costs.items():
            tickets[ms.submit({"x": (s, rnd)}, stream=s, cost=c)] = (s, rnd)
    # every stream on one device, assigned least-loaded at its first request
    assert ms.device_of == {0: 0, 1: 1, 2: 2, 3: 1, 4: 2}
    assert ms.poll() == 15
    got = {}
    for t in ms.finished():
        r = ms.result(t)
        got[t] = r["recon"]
        assert r["device"] == ms.device_of[r["recon"][0]]
    assert got == tickets and ms.finished() == []
