"""Serving benchmark with mixed streams: 64 concurrent synthetic streams, 48
QCIF and 16 CIF, through the continuous-batching server (dvc_server_*).

    python -m dvc_b200.serve_bench [--rates 100,300,1000,3000,5000] [--frames 17]

Streams: QCIF streams as the QCIF workload (SkipBlock 0, IntraMode 0,
DeblockingFilter 0), CIF streams as the CIF workload (SkipBlock 1, IntraMode 1,
DeblockingFilter 1, IntraQP 30), each from its own seed, GOP drawn from
{2, 4, 8} and QIndex uniformly from 1..8; the bitstreams come from
dvc_b200.encoder and the intra blocks are decoded on the host before serving
(they are the frames' starting content).  Requests are the WZ frames, in each
stream's decoding order, interleaved round-robin over the streams; they arrive
as a Poisson process at each offered rate.  A request is submitted once it has
arrived and its WZ references have been decoded (their results are its
reference frames), with a 16 GB device-memory budget.  For every rate: offered
rate, throughput (requests over the time to finish them all) and the latency
from submission to completion (p50 / p99).  The plain drop-in (one
dvc_decode_wz_frames call per frame) is timed on the same requests for the
comparison.  Prints one JSON line.
"""
import argparse
import json
import os
import time

import numpy as np


def build(n_frames, seed=2024):
    """Requests of the 64 streams: list of dicts (a session-style item plus
    past_from / future_from request indices and the stream id) in round-robin
    order over the streams."""
    from . import bitstream as bs, decoder, encoder, intra, synth
    rng = np.random.default_rng(seed)
    per_stream = []
    for s in range(64):
        kind = "qcif" if s < 48 else "cif"
        gop = int(rng.choice([2, 4, 8]))
        q = int(rng.integers(1, 9))
        ori, key = synth.make_sequence(kind, n_frames, 1000 + s)
        if kind == "qcif":
            wz, ib = encoder.encode_sequence(ori, gop, q), b""
        else:
            wz, ib = encoder.encode_sequence_intra(ori, gop, q, 30, 1, 1, 1)
        st = bs.parse_wz(wz)
        start = np.array(key, np.uint8, copy=True)
        if ib:
            for m, (px, _) in intra.decode_all(st, ib, key).items():
                start[m] = px
        reqs = []
        for lvl in decoder.decode_levels(st):
            for (m, b, e) in lvl:
                it = decoder.frame_item(st, st.frames[m], start)
                it["_deps"] = [r for r in (b, e) if r in st.frames]
                it["_frame"] = m
                it["_stream"] = s
                it["_kind"] = kind
                reqs.append(it)
        per_stream.append(reqs)
    # round-robin interleave; dependencies by request index
    out, where = [], {}
    k = 0
    while any(k < len(r) for r in per_stream):
        for s, r in enumerate(per_stream):
            if k < len(r):
                it = r[k]
                where[(s, it["_frame"])] = len(out)
                out.append(it)
        k += 1
    for it in out:
        it["_deps"] = [where[(it["_stream"], d)] for d in it["_deps"]]
    return out


def serve(srv, reqs, arrivals):
    """Submit each request once arrived and its references are decoded; poll to
    completion.  Returns (seconds, submit-to-completion latencies in ms, decoded
    frames by request)."""
    n = len(reqs)
    res, tickets, lat = {}, {}, []
    waiting = list(range(n))
    host = {"poll_s": 0.0, "poll_max_ms": 0.0, "submit_s": 0.0, "polls": 0}
    t0 = time.perf_counter()
    while len(res) < n:
        now = time.perf_counter() - t0
        still = []
        for k in waiting:
            it = reqs[k]
            if arrivals[k] > now or any(d not in res for d in it["_deps"]):
                still.append(k)
                continue
            sub = {key: v for key, v in it.items() if not key.startswith("_")}
            for name, d in zip(("past", "future"), (it["past_idx"], it["future_idx"])):
                for dep in it["_deps"]:
                    if reqs[dep]["_frame"] == d:
                        sub[name] = res[dep]
            ts = time.perf_counter()
            tickets[srv.submit(sub)] = k
            host["submit_s"] += time.perf_counter() - ts
        waiting = still
        tp = time.perf_counter()
        got = srv.poll()
        tp = time.perf_counter() - tp
        host["poll_s"] += tp
        host["poll_max_ms"] = max(host["poll_max_ms"], 1e3 * tp)
        host["polls"] += 1
        if got:
            for t in srv.finished():
                r = srv.result(t)
                res[tickets.pop(t)] = r["recon"]
                lat.append(r["latency_ms"])
        else:
            time.sleep(0.0002)
    serve.host = host
    return time.perf_counter() - t0, lat, res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rates", default="100,300,1000,3000,5000")
    ap.add_argument("--frames", type=int, default=17)
    ap.add_argument("--streams", type=int, default=16)
    ap.add_argument("--max-cohort", type=int, default=16)
    ap.add_argument("--batch-window-us", type=int, default=None)
    ap.add_argument("--no-plain", action="store_true")
    args = ap.parse_args()
    # one hardware queue per CUDA stream (the default 8 makes the 16 decode
    # streams share queues and wait behind each other's launches); before CUDA
    # starts, and a value set by the caller wins
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    from . import native
    t_build = time.perf_counter()
    reqs = build(args.frames)
    t_build = time.perf_counter() - t_build
    ctx = native.Context(int(os.environ.get("LOCAL_RANK", "0")))
    srv = ctx.server(mem_budget_bytes=16 << 30, streams=args.streams, max_cohort=args.max_cohort,
                     batch_window_us=args.batch_window_us)
    n = len(reqs)
    serve(srv, reqs, np.zeros(n))  # warm-up at once
    sweep = []
    for rate in [float(r) for r in args.rates.split(",")]:
        rng = np.random.default_rng(7)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
        dt, lat, served = serve(srv, reqs, arrivals)
        sweep.append({"offered_rate": rate, "throughput": n / dt, "requests": n,
                      "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                      "host": dict(serve.host, seconds=dt)})
    srv.close()
    # the plain drop-in on the same requests, in order (references from its own results)
    res_all = {}

    def plain_item(k):
        it = reqs[k]
        sub = {key: v for key, v in it.items() if not key.startswith("_")}
        for name, d in zip(("past", "future"), (it["past_idx"], it["future_idx"])):
            for dep in it["_deps"]:
                if reqs[dep]["_frame"] == d:
                    sub[name] = res_all[dep]
        return sub

    plain_lat = {"qcif": [], "cif": []}
    t0 = time.perf_counter()
    for k in range(0 if args.no_plain else n):
        sub = plain_item(k)
        t1 = time.perf_counter()
        out = ctx.decode_wz_frames([sub])[0]
        plain_lat[reqs[k]["_kind"]].append(1e3 * (time.perf_counter() - t1))
        res_all[k] = out["recon"]
    plain_s = time.perf_counter() - t0
    ctx.close()
    kinds = {k: sum(1 for r in reqs if r["_kind"] == k) for k in ("qcif", "cif")}
    same = None if args.no_plain else all(np.array_equal(served[k], res_all[k]) for k in range(n))
    print(json.dumps({
        "metric": "served WZ frames/s and p50/p99 latency, 64 mixed streams", "requests": n, "by_kind": kinds,
        "streams": 64, "frames_per_stream": args.frames, "mem_budget_gb": 16, "server_streams": args.streams,
        "max_cohort": args.max_cohort, "sweep": sweep,
        "batch_window_us": args.batch_window_us,
        "plain": None if args.no_plain else {"throughput": n / plain_s,
                  "p50_ms": {k: float(np.percentile(v, 50)) for k, v in plain_lat.items() if v},
                  "p99_ms": {k: float(np.percentile(v, 99)) for k, v in plain_lat.items() if v}},
        "served_equals_plain": same, "build_s": t_build}))


if __name__ == "__main__":
    main()
