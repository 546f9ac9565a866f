"""Autotuner for the LDPCA ladder's launch shape.

    python -m dvc_b200.autotune [--out tuning.json] [--streams 4] [--frames 33] [--runs 5]

Two launch parameters of the ladder kernel are chosen by measurement on the
device the tuner runs on:
  - threads per codeword block (512 or 1024; edges per thread = ceil(E / threads),
    19 or 38 for the CIF code's 19,008 edges);
  - the floor of the speculative ladder width: every codeword of a bitplane step
    is decoded by max(floor, SMs / codewords in flight) blocks, each starting at
    another code of the ladder (1 turns speculation off).
The workload is the batched form: CIF streams (GOP 4, QIndex spread over 1..8,
SkipBlock 1, IntraMode 1, DeblockingFilter 1) encoded by dvc_b200.encoder and
decoded as one device-resident session, replayed as a CUDA graph.  Every
setting must decode exactly the same frames, rates and ladder codes as the
first one tried (the launch shape changes only how the work is spread); the
tuner raises otherwise.  The fastest setting is written as JSON together with
every timing; apply(path) puts it into the environment variables the library
reads (DVC_LDPCA_THREADS when a context is created, DVC_LDPCA_SPEC_FLOOR when a
batch is prepared), so a process calls it before creating its Context.

The motion-search kernels have compile-time tile shapes and are not tuned here.
"""
import argparse
import itertools
import json
import os
import time

import numpy as np

THREADS = (512, 1024)
SPEC_FLOORS = (1, 2, 4, 8, 12, 16, 24, 32)
ENV_THREADS, ENV_FLOOR = "DVC_LDPCA_THREADS", "DVC_LDPCA_SPEC_FLOOR"


def space(threads=THREADS, floors=SPEC_FLOORS):
    """The settings tried, as dicts of the library's environment variables."""
    return [{ENV_THREADS: str(t), ENV_FLOOR: str(k)} for t, k in itertools.product(threads, floors)]


def choose(results):
    """The fastest of [{"setting": ..., "ms": [...]}] by median step time
    (ties: the earlier one)."""
    best = None
    for r in results:
        med = float(np.median(r["ms"]))
        if best is None or med < best[0]:
            best = (med, r)
    return best[1]


def signature(outputs):
    """What every setting must reproduce: per frame the decoded frame, its WZ
    bits and, per bitplane, everything but the BP work (which counts the
    speculative blocks, so it depends on the setting)."""
    return [(rec.tobytes(), int(bits), np.ascontiguousarray(planes[:, :3]).tobytes())
            for rec, bits, planes in outputs]


def tune(measure, settings, env=os.environ):
    """measure(setting) -> (step times in ms, per-frame outputs), run with the
    setting's variables in env.  Returns (best result, all results)."""
    results, ref = [], None
    saved = {k: env.get(k) for k in (ENV_THREADS, ENV_FLOOR)}
    try:
        for st in settings:
            env.update(st)
            ms, outputs = measure(st)
            sig = signature(outputs)
            if ref is None:
                ref = sig
            elif sig != ref:
                raise RuntimeError("setting %s decoded differently from %s" % (st, settings[0]))
            results.append({"setting": dict(st), "ms": [float(x) for x in ms]})
    finally:
        for k, v in saved.items():
            if v is None:
                env.pop(k, None)
            else:
                env[k] = v
    return choose(results), results


def save(path, best, results, device):
    with open(path, "w") as f:
        json.dump({"device": device, "best": best["setting"], "median_ms": float(np.median(best["ms"])),
                   "results": results}, f, indent=1)


def apply(path, env=os.environ):
    """Set the tuned variables (values already set in env win); returns them."""
    with open(path) as f:
        best = json.load(f)["best"]
    for k in (ENV_THREADS, ENV_FLOOR):
        if k in best:
            env.setdefault(k, str(best[k]))
    return {k: env.get(k) for k in (ENV_THREADS, ENV_FLOOR)}


def workload(n_streams, n_frames, seed=4100):
    """Session items of n_streams CIF streams (GOP 4, QIndex spread over 1..8)."""
    from . import bitstream as bs, encoder, stress_bench, synth
    items = []
    for s in range(n_streams):
        q = 1 + (s * 7) // max(1, n_streams - 1) if n_streams > 1 else 4
        ori, key = synth.make_sequence("cif", n_frames, seed + s)
        wz, ib = encoder.encode_sequence_intra(ori, 4, q, 30, 1, 1, 1)
        its, _ = stress_bench.session_items(bs.parse_wz(wz), key, ib)
        base = len(items)
        for it in its:  # references by index within the stream -> within the whole list
            for name in ("past_from", "future_from"):
                if it.get(name) is not None:
                    it[name] += base
        items += its
    return items


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="tuning.json")
    ap.add_argument("--streams", type=int, default=4)
    ap.add_argument("--frames", type=int, default=33)
    ap.add_argument("--runs", type=int, default=5)
    ap.add_argument("--max-batch", type=int, default=16)
    ap.add_argument("--cuda-streams", type=int, default=16)
    args = ap.parse_args()
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    t0 = time.perf_counter()
    items = workload(args.streams, args.frames)
    print("workload: %d WZ frames (%.1f s to encode)" % (len(items), time.perf_counter() - t0), flush=True)
    from . import native
    dev = int(os.environ.get("LOCAL_RANK", "0"))

    def measure(setting):
        ctx = native.Context(dev)  # reads DVC_LDPCA_THREADS
        try:
            ses = ctx.session(items, max_batch=args.max_batch, streams=args.cuda_streams)
            try:
                ses.run()
                ses.run()  # captured
                ms = [ses.run() for _ in range(args.runs)]
                outputs = [ses.frame(i) for i in range(len(items))]
            finally:
                ses.close()
        finally:
            ctx.close()
        print("  %s: median %.1f ms" % (setting, float(np.median(ms))), flush=True)
        return ms, outputs

    best, results = tune(measure, space())
    import torch
    device = torch.cuda.get_device_name(dev) if torch.cuda.is_available() else "unknown"
    save(args.out, best, results, device)
    print(json.dumps({"best": best["setting"], "median_ms": float(np.median(best["ms"])), "out": args.out}))


if __name__ == "__main__":
    main()
