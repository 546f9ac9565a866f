"""Replica scheduling across GPUs (one process per GPU).

WZ frames, GOPs and whole streams are independent given their key frames, so
a multi-GPU deployment needs no exchange step on the data path: every rank
decodes its own share of the streams on its own device and only the results
(or a timing) come back.  This module holds the host side of that:

  plan(costs, world)        least-loaded assignment of streams to ranks;
  share(costs, rank, world) the streams of one rank;
  max_over_ranks(x)         a scalar reduced with MAX over the process group
                            (the device time of a step is the slowest rank's);
  gather(obj)               every rank's object on every rank.

The collectives run on whatever backend the process group was created with:
NCCL between GPUs, gloo on the CPU (as in the tests).
"""
import heapq


def plan(costs, world):
    """Assign stream indices to `world` ranks, heaviest first onto the least
    loaded rank (ties to the lower rank); returns one sorted list per rank."""
    if world < 1:
        raise ValueError("world size must be at least 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(x) for x in out]


def share(costs, rank, world):
    return plan(costs, world)[rank]


def max_over_ranks(x, device=None):
    """MAX of a float over the default process group (x itself with no group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    if device is None:
        device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather(obj):
    """Every rank's `obj`, in rank order."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out


class MultiServer:
    """Serving across several devices: one server (native.Server, or any object
    with its submit/poll/finished/result/close methods) per device, and every
    stream pinned to one of them, so that a stream's frames, which reference
    each other's decoded output, stay on one device.  A new stream goes to the
    device with the least load assigned so far (its cost: the caller's
    estimate, e.g. WZ frames times pixels), ties to the lower device.  Tickets
    are this object's own and map to (device, that server's ticket).  No data
    crosses between devices: each decodes its own streams, as a replica."""

    def __init__(self, servers):
        if not servers:
            raise ValueError("at least one server")
        self.servers = list(servers)
        self.load = [0.0] * len(self.servers)
        self.device_of = {}   # stream id -> device index
        self.where = {}       # our ticket -> (device, its ticket)
        self.back = {}        # (device, its ticket) -> our ticket
        self.next = 1

    def assign(self, stream, cost=1.0):
        """The device of `stream`, chosen (least loaded) at its first request."""
        d = self.device_of.get(stream)
        if d is None:
            d = min(range(len(self.servers)), key=lambda i: (self.load[i], i))
            self.device_of[stream] = d
            self.load[d] += float(cost)
        return d

    def submit(self, item, stream, cost=1.0):
        d = self.assign(stream, cost)
        t = self.servers[d].submit(item)
        ours = self.next
        self.next += 1
        self.where[ours] = (d, t)
        self.back[(d, t)] = ours
        return ours

    def poll(self):
        """Polls every device; the number of requests that finished."""
        return sum(int(s.poll() or 0) for s in self.servers)

    def finished(self):
        out = []
        for d, s in enumerate(self.servers):
            out += [self.back[(d, t)] for t in s.finished() if (d, t) in self.back]
        return sorted(out)

    def result(self, ticket):
        d, t = self.where.pop(ticket)
        del self.back[(d, t)]
        r = self.servers[d].result(t)
        r["device"] = d
        return r

    def close(self):
        for s in self.servers:
            s.close()
