"""The bench's host side on the CPU.  Its serving loop (bench.serve) against a
fake server: every request is served once, a frame that names another frame's
output as its reference is submitted only after that output exists and
receives it, and the loop ends whichever polls finish the work.  Its intra step
(bench.intra_starts): the frames' starting content."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


class FakeServer:
    """Finishes, on each poll, up to `per_poll` of the requests submitted at
    least one poll earlier (newest first, so completions come out of order);
    every `idle`-th poll finishes nothing.  Raises after `max_polls` polls, so a
    loop that stops making progress fails instead of spinning."""

    def __init__(self, per_poll, idle, max_polls=200000):
        self.per_poll, self.idle, self.max_polls = per_poll, idle, max_polls
        self.next, self.polls = 0, 0
        self.queued, self.done, self.collected, self.submitted = [], {}, set(), []

    def submit(self, item):
        for name in ("past", "future"):
            assert item.get(name + "_from") is None, "reference indices reach the server"
            assert item[name] is not None
        t = self.next
        self.next += 1
        self.submitted.append(t)
        self.queued.append((t, self.polls, item))
        return t

    def poll(self):
        self.polls += 1
        assert self.polls < self.max_polls, "the loop stopped making progress"
        if self.polls % self.idle == 0:
            return 0
        eligible = [x for x in self.queued if x[1] < self.polls - 1]
        take = eligible[::-1][:self.per_poll]
        taken = set(t for t, _, _ in take)
        self.queued = [x for x in self.queued if x[0] not in taken]
        for t, _, item in take:
            # the "decoded frame": a function of the frame's own start and its references
            rec = (item["recon"].astype(np.int64) + item["past"] + 2 * item["future"]) % 251
            self.done[t] = dict(recon=rec.astype(np.uint8), wz_bits=int(t), latency_ms=1.0)
        return len(take)

    def finished(self):
        return [t for t in sorted(self.done) if t not in self.collected]

    def result(self, t):
        assert t in self.done and t not in self.collected
        self.collected.add(t)
        return self.done[t]


def gop_items(n_streams, gop, n_gops, shape=(4, 6), seed=0):
    """Items in the bench's form: per stream, the GOP's middle frame first, then
    the frames that name it as a reference (past_from / future_from)."""
    rng = np.random.default_rng(seed)
    its = []
    for _ in range(n_streams):
        for _ in range(n_gops):
            where = {}

            def add(m, b, e):
                it = dict(recon=rng.integers(0, 251, shape, dtype=np.uint8), past=None, future=None)
                for name, ref in (("past", b), ("future", e)):
                    if ref in where:
                        it[name + "_from"] = where[ref]
                    else:
                        it[name] = rng.integers(0, 251, shape, dtype=np.uint8)
                where[m] = len(its)
                its.append(it)

            def level(b, e):
                if e - b < 2:
                    return
                m = (b + e) // 2
                add(m, b, e)
                level(b, m)
                level(m, e)

            level(0, gop)
    return its


def expected(its):
    out = {}
    for i, it in enumerate(its):  # references precede their users
        past = out[it["past_from"]] if it.get("past_from") is not None else it["past"]
        fut = out[it["future_from"]] if it.get("future_from") is not None else it["future"]
        out[i] = ((it["recon"].astype(np.int64) + past + 2 * fut) % 251).astype(np.uint8)
    return out


@pytest.mark.parametrize("per_poll,idle,poll_every", [(1, 3, 16), (5, 2, 1), (64, 1000, 4), (3, 4, 1000)])
def test_serve_all_items_in_dependency_order(per_poll, idle, poll_every):
    its = gop_items(n_streams=5, gop=8, n_gops=3)
    srv = FakeServer(per_poll, idle)
    dt, lat, res = bench.serve(srv, its, poll_every=poll_every)
    assert sorted(res) == list(range(len(its))) and len(lat) == len(its)
    want = expected(its)
    for i in range(len(its)):
        assert np.array_equal(res[i]["recon"], want[i]), i
    assert len(srv.submitted) == len(its)


def test_serve_pool_with_arrivals():
    its = gop_items(n_streams=3, gop=2, n_gops=4)  # GOP 2: no item references another
    assert all(it.get("past_from") is None and it.get("future_from") is None for it in its)
    pool = list(range(len(its)))
    arrivals = np.cumsum(np.full(40, 0.0005))
    srv = FakeServer(per_poll=2, idle=5)
    dt, lat, res = bench.serve(srv, its, pool, arrivals, poll_every=3)
    assert len(lat) == 40 and len(srv.submitted) == 40
    assert dt >= arrivals[-1]


def test_intra_starts_match_a_direct_decode():
    """bench.intra_starts: every frame's starting content equals the key-frame
    content with that frame's intra blocks decoded over it (frames without
    intra blocks: the key-frame content itself)."""
    from dvc_b200 import bitstream as bs, encoder, intra, synth
    ori, key = synth.make_sequence("cif", 9, 77)
    streams, ib = {}, {}
    for gq in ((4, 3), (4, 8)):
        wz, b = encoder.encode_sequence_intra(ori, gq[0], gq[1], 30, 1, 1, 1)
        streams[gq], ib[gq] = bs.parse_wz(wz), b
    starts = bench.intra_starts(streams, ib, key)
    for gq, st in streams.items():
        want = np.array(key, copy=True)
        for m, (px, _) in intra.decode_all(st, ib[gq], key).items():
            want[m] = px
        for m in range(key.shape[0]):
            got = starts[gq][m]
            assert got.dtype == np.uint8 and got.flags.c_contiguous and np.array_equal(got, want[m]), (gq, m)
    assert any(fr.intra_mode for fr in streams[(4, 8)].frames.values())


def test_serving_overlapped_with_the_intra_step():
    """The e2e step's form: intra blocks decoded on a pool while the loop
    submits each frame once its stream's starting content is ready
    (start_of); the results equal those of decoding the intra blocks first."""
    from concurrent.futures import ThreadPoolExecutor
    from dvc_b200 import bitstream as bs, encoder, synth
    ori, key = synth.make_sequence("cif", 9, 78)
    streams, ib = {}, {}
    for gq in ((2, 1), (4, 5), (4, 8)):
        wz, b = encoder.encode_sequence_intra(ori, gq[0], gq[1], 30, 1, 1, 1)
        streams[gq], ib[gq] = bs.parse_wz(wz), b
    its, lev, src = bench.items(streams, key, bench.intra_starts(streams, ib, key))
    want = bench.serve(FakeServer(per_poll=3, idle=4), its)[2]
    for it in its:  # the step must bring its own starting content
        it["recon"] = np.zeros_like(it["recon"])
    with ThreadPoolExecutor(2) as ex:
        fut = bench.intra_starts_async(ex, streams, ib, key)

        def start_of(i):
            gq, m = src[i]
            return fut[gq].result()[m] if fut[gq].done() else None

        got = bench.serve(FakeServer(per_poll=3, idle=4), its, start_of=start_of)[2]
    assert sorted(got) == sorted(want) == list(range(len(its)))
    for i in want:
        assert np.array_equal(got[i]["recon"], want[i]["recon"]), i
