"""GPU: the continuous-batching server gives every frame the same result as decoding
it alone, with QCIF and CIF requests from several streams in flight together."""
import os
import time

import numpy as np
import pytest

from dvc_b200 import bitstream as bs
from dvc_b200 import decoder, encoder, native, synth

pytestmark = pytest.mark.gpu


def _items(kind, n_frames, gop, q, seed):
    ori, key = synth.make_sequence(kind, n_frames, seed)
    st = bs.parse_wz(encoder.encode_sequence(ori, gop, q))
    return [decoder.frame_item(st, st.frames[m], key) for (m, b, e) in bs.sequence_order(st.n_frames, st.gop)]


def test_server_mix_matches_alone(gpu_ctx):
    mix = (_items("qcif", 5, 2, 4, 31) + _items("cif", 3, 2, 3, 32) + _items("qcif", 5, 4, 8, 33)
           + _items("qcif", 3, 2, 1, 34) + _items("cif", 3, 2, 6, 35))
    alone = [gpu_ctx.decode_wz_frames([it])[0] for it in mix]
    srv = gpu_ctx.server(mem_budget_bytes=4 << 30, streams=3, max_cohort=2)
    tickets = []
    # staggered arrivals: half now, the rest while the first cohorts are decoding
    for it in mix[: len(mix) // 2]:
        tickets.append(srv.submit(it))
    done = srv.poll()
    for it in mix[len(mix) // 2:]:
        tickets.append(srv.submit(it))
        done += srv.poll()
    t0 = time.time()
    while done < len(mix) and time.time() - t0 < 120:
        done += srv.poll()
        time.sleep(0.001)
    assert done == len(mix)
    assert sorted(srv.finished()) == sorted(tickets)  # every finished ticket listed, none collected yet
    for t, a in zip(tickets, alone):
        r = srv.result(t)
        assert np.array_equal(r["recon"], a["recon"])
        assert r["wz_bits"] == a["wz_bits"]
        # rate, first code and accepted code per bitplane; column 3 counts the BP
        # iterations run, which depends on how widely the ladder was speculated
        assert np.array_equal(r["planes"][:, :3], a["planes"][:, :3])
        assert r["latency_ms"] > 0
    assert srv.finished() == []
    srv.close()


def test_server_refuses_frame_above_budget(gpu_ctx):
    it = _items("cif", 3, 2, 4, 36)[0]
    srv = gpu_ctx.server(mem_budget_bytes=1 << 20, streams=1, max_cohort=1)
    with pytest.raises(native.DvcError) as ex:
        srv.submit(it)
    assert ex.value.code == native.DVC_E_NOMEM
    srv.close()


def test_bench_e2e_form_matches_session(gpu_ctx):
    """The bench's end-to-end form on a small workload: intra blocks decoded on
    a host pool while the server decodes the frames whose starting content is
    ready (bench.serve with start_of), second-level frames submitted with their
    references' results; every frame equals the device-resident session's."""
    import sys
    from concurrent.futures import ThreadPoolExecutor
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    ori, key = synth.make_sequence("cif", 9, 91)
    streams, ib = {}, {}
    for gq in ((2, 2), (4, 5), (4, 8)):
        wz, b = encoder.encode_sequence_intra(ori, gq[0], gq[1], 30, 1, 1, 1)
        streams[gq], ib[gq] = bs.parse_wz(wz), b
    its, lev, src = bench.items(streams, key, bench.intra_starts(streams, ib, key))
    assert max(lev) == 1
    ses = gpu_ctx.session(its, max_batch=4, streams=2)
    srv = gpu_ctx.server(mem_budget_bytes=4 << 30, streams=2, max_cohort=4)
    try:
        ses.run()
        with ThreadPoolExecutor(2) as ex:
            fut = bench.intra_starts_async(ex, streams, ib, key)

            def start_of(i):
                gq, m = src[i]
                return fut[gq].result()[m] if fut[gq].done() else None

            _, lat, served = bench.serve(srv, its, start_of=start_of, poll_every=2)
        assert sorted(served) == list(range(len(its))) and len(lat) == len(its)
        for i in range(len(its)):
            rec, bits, _ = ses.frame(i)
            assert np.array_equal(served[i]["recon"], rec) and served[i]["wz_bits"] == bits, i
    finally:
        srv.close()
        ses.close()


def test_multi_server_replicas_match_alone(gpu_ctx):
    """Serving over two replicas (dvc_b200.replicas.MultiServer): two contexts,
    each with its own server, here both on device 0 (this run has one GPU; each
    replica would take its own device in a multi-GPU deployment, with nothing
    exchanged between them).  Streams are pinned to a replica; every frame's
    result equals the frame decoded alone."""
    from dvc_b200 import replicas
    streams = [_items("qcif", 5, 2, 4, 41), _items("cif", 3, 2, 3, 42), _items("qcif", 5, 4, 8, 43),
               _items("cif", 3, 2, 6, 44)]
    alone = [[gpu_ctx.decode_wz_frames([it])[0] for it in s] for s in streams]
    ctxs = [native.Context(0), native.Context(0)]
    ms = replicas.MultiServer([c.server(mem_budget_bytes=4 << 30, streams=2, max_cohort=2) for c in ctxs])
    try:
        tickets = {}
        for s, items in enumerate(streams):
            for k, it in enumerate(items):
                tickets[ms.submit(it, stream=s, cost=it["width"] * it["height"] * len(items))] = (s, k)
        done, t0 = 0, time.time()
        while done < len(tickets) and time.time() - t0 < 120:
            done += ms.poll()
            time.sleep(0.001)
        assert done == len(tickets)
        assert sorted(set(ms.device_of.values())) == [0, 1]  # both replicas got streams
        for t in ms.finished():
            s, k = tickets[t]
            r = ms.result(t)
            assert r["device"] == ms.device_of[s]
            assert np.array_equal(r["recon"], alone[s][k]["recon"]) and r["wz_bits"] == alone[s][k]["wz_bits"]
    finally:
        ms.close()
        for c in ctxs:
            c.close()
