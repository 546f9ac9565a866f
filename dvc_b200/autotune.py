"""Autotuner for the decoder's launch shapes.

    python -m dvc_b200.autotune [--out tuning.json] [--streams 4] [--frames 33] [--runs 5] [--bench-workload]

Five launch parameters are chosen by measurement on the device the tuner runs on:
  - threads per CIF codeword block of the LDPCA ladder, 512 or 1024 (edges per
    thread = 19,008 / threads: 38 or 19; columns per thread 13 or 7);
  - threads per QCIF codeword block, 1024, 256 or 512 (edges per thread 5, 19
    or 10; one, four or two codewords per SM);
  - the floor of the speculative ladder width: every codeword of a bitplane step
    is decoded by max(floor, SMs / codewords in flight) blocks, each starting at
    another code of the ladder (1 turns speculation off);
  - threads per updateSI search block, 64, 128 or 256 (one block per WZ 4x4
    block: 2 x 65 candidate columns, two adjacent ones per thread);
  - threads per forward-search block, 128, 256 or 512 (one block per 16x16
    macroblock: 65 x 65 candidate positions over the threads).
The search is coordinate-wise: starting from the library's defaults, each
parameter in turn takes the value that gives the shortest median step with the
others fixed.  The workload is the batched form: CIF streams (GOP 4, QIndex
spread over 1..8, SkipBlock 1, IntraMode 1, DeblockingFilter 1) and QCIF
streams (the same with the QCIF ladder) encoded by dvc_b200.encoder, each size
decoded as one device-resident session replayed as a CUDA graph; a step is
both sessions.  Every setting must decode exactly the same frames, rates and
ladder codes as the first one tried (the launch shape changes only how the work
is spread); the tuner raises otherwise.  The fastest setting is written as
JSON together with every timing; apply(path) puts it into the environment
variables the library reads when a context is created (DVC_LDPCA_SPEC_FLOOR
when a batch is prepared), so a process calls it before creating its Context.
"""
import argparse
import json
import os
import time

import numpy as np

ENV_THREADS, ENV_THREADS_QCIF, ENV_FLOOR = "DVC_LDPCA_THREADS", "DVC_LDPCA_THREADS_QCIF", "DVC_LDPCA_SPEC_FLOOR"
ENV_SI, ENV_FME = "DVC_SI_THREADS", "DVC_FME_THREADS"
KNOBS = [(ENV_THREADS, ("1024", "512")), (ENV_THREADS_QCIF, ("1024", "256", "512")),
         (ENV_FLOOR, ("4", "1", "2", "8", "12", "16", "24", "32")), (ENV_SI, ("64", "128", "256")),
         (ENV_FME, ("256", "128", "512"))]
ENV_ALL = tuple(k for k, _ in KNOBS)
THREADS = ("1024", "512")
SPEC_FLOORS = ("1", "2", "4", "8", "12", "16", "24", "32")


def defaults():
    return {k: v[0] for k, v in KNOBS}


def space(threads=THREADS, floors=SPEC_FLOORS):
    """Every combination of the CIF thread count and the speculation floor (the
    exhaustive form of the two LDPCA knobs), the other knobs at their defaults."""
    out = []
    for t in threads:
        for k in floors:
            st = defaults()
            st.update({ENV_THREADS: str(t), ENV_FLOOR: str(k)})
            out.append(st)
    return out


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


class _Runner:
    """Runs settings with their variables in env, checks the outputs, keeps every timing."""

    def __init__(self, measure, env):
        self.measure, self.env, self.ref, self.results, self.seen = measure, env, None, [], {}

    def __call__(self, st):
        key = tuple(sorted(st.items()))
        if key in self.seen:
            return self.seen[key]
        self.env.update(st)
        ms, outputs = self.measure(st)
        sig = signature(outputs)
        if self.ref is None:
            self.ref = (sig, dict(st))
        elif sig != self.ref[0]:
            raise RuntimeError("setting %s decoded differently from %s" % (st, self.ref[1]))
        r = {"setting": dict(st), "ms": [float(x) for x in ms]}
        self.results.append(r)
        self.seen[key] = r
        return r


def _saved(env):
    return {k: env.get(k) for k in ENV_ALL}


def _restore(env, saved):
    for k, v in saved.items():
        if v is None:
            env.pop(k, None)
        else:
            env[k] = v


def tune(measure, settings, env=os.environ):
    """measure(setting) -> (step times in ms, per-frame outputs), run with the
    setting's variables in env, for every setting given.  Returns (best
    result, all results)."""
    saved = _saved(env)
    try:
        run = _Runner(measure, env)
        for st in settings:
            run(st)
    finally:
        _restore(env, saved)
    return choose(run.results), run.results


def tune_coordinates(measure, knobs=KNOBS, env=os.environ):
    """Coordinate search: from the defaults, each knob in turn set to its
    fastest value with the others fixed.  Returns (best result, all results)."""
    saved = _saved(env)
    try:
        run = _Runner(measure, env)
        cur = {k: v[0] for k, v in knobs}
        best = run(dict(cur))
        for k, values in knobs:
            for v in values:
                st = dict(cur, **{k: v})
                r = run(st)
                if float(np.median(r["ms"])) < float(np.median(best["ms"])):
                    best = r
            cur = dict(best["setting"])
    finally:
        _restore(env, saved)
    return best, run.results


def save(path, best, results, device):
    with open(path, "w") as f:
        json.dump({"device": device, "best": best["setting"], "median_ms": float(np.median(best["ms"])),
                   "results": results}, f, indent=1)


def apply(path, env=os.environ):
    """Set the tuned variables (values already set in env win); returns them."""
    with open(path) as f:
        best = json.load(f)["best"]
    for k in ENV_ALL:
        if k in best:
            env.setdefault(k, str(best[k]))
    return {k: env.get(k) for k in ENV_ALL}


def workload(n_streams, n_frames, seed=4100, kind="cif"):
    """Session items of n_streams streams of one size (GOP 4, QIndex spread over 1..8)."""
    from . import bitstream as bs, encoder, stress_bench, synth
    items = []
    for s in range(n_streams):
        q = 1 + (s * 7) // max(1, n_streams - 1) if n_streams > 1 else 4
        ori, key = synth.make_sequence(kind, n_frames, seed + s)
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
    ap.add_argument("--bench-workload", action="store_true",
                    help="tune on bench.py's workload (640 CIF WZ frames); the QCIF shape is then not searched")
    args = ap.parse_args()
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    t0 = time.perf_counter()
    knobs = KNOBS
    if args.bench_workload:
        import sys
        sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
        import bench
        ori, key, streams, intra_bs = bench.workload()
        sessions = [bench.items(streams, key, bench.intra_starts(streams, intra_bs, key))[0]]
        knobs = [kv for kv in KNOBS if kv[0] != ENV_THREADS_QCIF]
    else:
        sessions = [workload(args.streams, args.frames, kind="cif"),
                    workload(args.streams * 2, args.frames, seed=4200, kind="qcif")]
    print("workload: %s WZ frames (%.1f s to encode)" % ([len(x) for x in sessions], time.perf_counter() - t0),
          flush=True)
    from . import native
    dev = int(os.environ.get("LOCAL_RANK", "0"))

    def measure(setting):
        ctx = native.Context(dev)  # reads the thread counts
        ms_total, outputs = None, []
        try:
            for items in sessions:
                ses = ctx.session(items, max_batch=args.max_batch, streams=args.cuda_streams)
                try:
                    ses.run()
                    ses.run()  # captured
                    ms = np.array([ses.run() for _ in range(args.runs)])
                    outputs += [ses.frame(i) for i in range(len(items))]
                finally:
                    ses.close()
                ms_total = ms if ms_total is None else ms_total + ms
        finally:
            ctx.close()
        print("  %s: median %.1f ms" % (setting, float(np.median(ms_total))), flush=True)
        return ms_total, outputs

    best, results = tune_coordinates(measure, knobs)
    import torch
    device = torch.cuda.get_device_name(dev) if torch.cuda.is_available() else "unknown"
    save(args.out, best, results, device)
    print(json.dumps({"best": best["setting"], "median_ms": float(np.median(best["ms"])), "out": args.out}))


if __name__ == "__main__":
    main()
