"""Large-GOP stress run: 8 synthetic CIF streams of 301 frames with fast motion
(dvc_b200.synth "cif_fast": global velocity in [-8, 8] pixels per frame, six
objects of 16-64 pixels moving at up to 10), GOP 8, QIndex 8, SkipBlock 1,
IntraMode 1, DeblockingFilter 1, IntraQP 30.

    python -m dvc_b200.stress_bench [--streams 8] [--frames 301] [--q 8] [--steps 3]

The bitstreams come from dvc_b200.encoder (run in a process pool), the intra
blocks are decoded on the host.  Each stream is one device-resident session
(dvc_session: the three levels of every GOP-8 recursion chained on the
device, 16 CUDA streams, cohorts of 16 frames); after one direct run and one
captured run, the timed runs replay the whole decode step of the stream as
one CUDA graph.  Prints one JSON line: WZ frames/s over all streams (device
time from CUDA events), per-stream step times, the number of dependent
levels, the share of intra and skip blocks, the BP work and the replays.
"""
import argparse
import json
import multiprocessing as mp
import os
import time

import numpy as np


def _encode(args):
    kind, n_frames, seed, gop, q = args
    from dvc_b200 import encoder, synth
    ori, key = synth.make_sequence(kind, n_frames, seed)
    wz, ib = encoder.encode_sequence_intra(ori, gop, q, 30, 1, 1, 1)
    return key, wz, ib


def session_items(st, key, ib):
    """Every WZ frame of a stream in level order, WZ references chained by item index."""
    from dvc_b200 import decoder, intra
    start = np.array(key, np.uint8, copy=True)
    if ib:
        for m, (px, _) in intra.decode_all(st, ib, key).items():
            start[m] = px
    items, where, levels = [], {}, decoder.decode_levels(st)
    for lvl in levels:
        for (m, b, e) in lvl:
            it = decoder.frame_item(st, st.frames[m], start)
            for name, ref in (("past", b), ("future", e)):
                if ref in st.frames:
                    it[name + "_from"], it[name] = where[ref], None
            where[m] = len(items)
            items.append(it)
    return items, len(levels)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--streams", type=int, default=8)
    ap.add_argument("--frames", type=int, default=301)
    ap.add_argument("--gop", type=int, default=8)
    ap.add_argument("--q", type=int, default=8)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--kind", default="cif_fast")
    args = ap.parse_args()
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    t0 = time.perf_counter()
    jobs = [(args.kind, args.frames, 3000 + s, args.gop, args.q) for s in range(args.streams)]
    # the pool starts (spawn) before this process touches the GPU
    with mp.get_context("spawn").Pool(min(len(jobs), os.cpu_count() or 1)) as pool:
        encoded = pool.map(_encode, jobs)
    t_encode = time.perf_counter() - t0
    from dvc_b200 import bitstream as bs, native
    ctx = native.Context(int(os.environ.get("LOCAL_RANK", "0")))
    per_stream, total_frames, total_ms, levels, bp, replays = [], 0, 0.0, 0, 0, 0
    intra_blocks = skip_blocks = all_blocks = 0
    for (key, wz, ib) in encoded:
        st = bs.parse_wz(wz)
        items, nlev = session_items(st, key, ib)
        levels = max(levels, nlev)
        for fr in st.frames.values():
            intra_blocks += int((fr.mode == 1).sum())
            skip_blocks += int((fr.mode == bs.SKIP_B).sum())
            all_blocks += fr.mode.size
        ses = ctx.session(items, max_batch=16, streams=16)
        try:
            ses.run()
            ses.run()  # captured
            ms = [ses.run() for _ in range(args.steps)]
            replays += ses.replays()
            bp += int(sum(int(ses.frame(i)[2][:, 3].sum()) for i in range(len(items))))
        finally:
            ses.close()
        step = float(np.mean(ms))
        per_stream.append({"frames": len(items), "ms_per_step": step})
        total_frames += len(items)
        total_ms += step
    ctx.close()
    print(json.dumps({
        "metric": "WZ frames/s, large-GOP stress", "value": total_frames / (total_ms / 1e3), "unit": "WZ frames/s",
        "config": {"kind": args.kind, "streams": args.streams, "frames_per_stream": args.frames, "gop": args.gop,
                   "qindex": args.q, "skip": 1, "intra": 1, "deblock": 1, "intra_qp": 30},
        "wz_frames": total_frames, "levels": levels, "intra_block_share": intra_blocks / max(1, all_blocks),
        "skip_block_share": skip_blocks / max(1, all_blocks), "bp_block_iterations": bp,
        "graph_replays": replays, "per_stream": per_stream, "encode_s": t_encode}))


if __name__ == "__main__":
    main()
