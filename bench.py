"""Benchmark of the Wyner-Ziv decoder hot path: WZ frames/s at CIF.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step): every WZ frame of 16 synthetic CIF 352x288 sequences, 65
frames each: GOP 2 and GOP 4, each at QIndex 1..8 (SkipBlock 1, IntraMode 1,
DeblockingFilter 1, IntraQP 30; skip and intra decisions by dvc_b200.encoder:
the reference's skip test, which the moving content never passes, and a
rate-based intra choice that picks none of the 8x8 blocks at Q1-2, about a
tenth at Q4 and nearly all at Q8), the seeded generator of dvc_b200.synth "cif" (six
sinusoids with periods 8-80 px, global motion, four moving 48x48 objects, key
frames = original + N(0,2)) -> 8*32 + 8*48 = 640 WZ frames per step.  GOP-4
frames 1 and 3 of each GOP take the decoded frame 2 as a reference, so a step
has two levels of dependent frames.

Our arm prints one JSON line with:
  value   WZ frames/s of the batched device-resident path (dvc_session: inputs,
          intra pixels included, already in HBM, cohorts of frames on
          concurrent streams, the GOP-4 levels chained on the device; device
          time from CUDA events; L2 flushed between steps);
  e2e     the same through the public serving API with host buffers
          (dvc_server: the host decode of each stream's intra bitstream on a
          thread pool, each frame submitted once its starting content is
          decoded and its references are done, reference frames, starting
          content, syndromes and CRCs copied in and decoded frames copied out,
          all inside the timed region; the second level's references are the
          first level's results);
  served  Poisson arrivals at fractions of the measured capacity through
          dvc_server (requests drawn from the first-level frames): throughput
          and per-frame latency p50/p99 (submit to completion);
  served_mixed  the mixed serving workload (dvc_b200.serve_bench: 64 streams,
          48 QCIF and 16 CIF, GOP 2/4/8, QIndex 1..8) at Poisson rates of
          300, 1000 and 5000 frames/s, with the plain drop-in on the same
          requests and a check that every served frame equals the plain one;
  plain   the one-frame-at-a-time drop-in (one dvc_decode_wz_frames call per
          frame) with per-frame latency p50/p99;
  roofline, cpu_baseline, clocks, gpu_launches.
--impl reference times the reference codec's own CPU path on the same
sequences and settings: streams encoded by the reference encoder
(oracle/_ref/DvcEnc), whole GOPs decoded by the reference decoder
(oracle/_ref/DvcDec, ParallelMode 1 with every host core), a fixed stratified
sample over every (GOP, QIndex) stream and both levels, the workload's rate
estimated from the per-stream times; plus ParallelMode 0 on one core for one
frame.  That process loads none of this repository's native libraries.
Under torchrun each rank decodes its own replica (weak scaling, no collective
on the data path); rank 0 prints the max-over-ranks result.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "WZ frames/s + p50/p99 frame latency at CIF, served vs plain GPU, bit-exact"
N_FRAMES, SEED, KIND = 65, 101, "cif"
GOPS = (2, 4)
QS = tuple(range(1, 9))


INTRA_QP = 30


def workload():
    """Original and key frames, the parsed WZ stream and the intra bitstream of
    every (GOP, Q)."""
    from dvc_b200 import bitstream as bs, encoder, synth
    ori, key = synth.make_sequence(KIND, N_FRAMES, SEED)
    streams, intra_bs = {}, {}
    for g in GOPS:
        cache = {}  # the encoder's side-information estimate does not depend on Q
        for q in QS:
            wz, ib = encoder.encode_sequence_intra(ori, g, q, INTRA_QP, 1, 1, 1, si_cache=cache)
            streams[(g, q)], intra_bs[(g, q)] = bs.parse_wz(wz), ib
    return ori, key, streams, intra_bs


class Starts:
    """Frame index -> starting content of one stream: the key-frame content
    with the frame's intra blocks decoded over it for frames that have intra
    blocks, the key-frame content itself (a view, nothing to decode) for the
    others."""

    def __init__(self, key, decoded):
        self.key, self.decoded = key, decoded

    def __getitem__(self, m):
        px = self.decoded.get(m)
        return self.key[m] if px is None else px


def intra_starts_async(ex, streams, intra_bs, key):
    """Per (GOP, Q): a future of the frames' starting content (Starts), the
    intra blocks of each WZ frame decoded on the host (dvc_intra_decode_frame,
    which releases the GIL) by the executor `ex`, the longest intra bit strings
    submitted first."""
    from dvc_b200 import intra

    def one(gq):
        return Starts(key, {m: px for m, (px, _) in intra.decode_all(streams[gq], intra_bs[gq], key).items()})

    return {gq: ex.submit(one, gq) for gq in sorted(streams, key=lambda gq: -len(intra_bs[gq]))}


def intra_starts(streams, intra_bs, key):
    """Per (GOP, Q): the frames' starting content (Starts), the streams decoded
    on a thread pool."""
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(len(streams), os.cpu_count() or 1)) as ex:
        fut = intra_starts_async(ex, streams, intra_bs, key)
        return {gq: f.result() for gq, f in fut.items()}


def items(streams, key, starts):
    """Every WZ frame of every stream in decode order, as session items: a
    reference that is itself a WZ frame is named by the index of its item
    (past_from / future_from); the level of each item and its (GOP, Q, frame)
    are returned beside it."""
    from dvc_b200 import decoder
    out, level, src = [], [], []
    for (g, q), st in sorted(streams.items()):
        where = {}
        for lv, lvl in enumerate(decoder.decode_levels(st)):
            for (m, b, e) in lvl:
                it = decoder.frame_item(st, st.frames[m], starts[(g, q)])
                for name, ref in (("past", b), ("future", e)):
                    if ref in st.frames:
                        it[name + "_from"] = where[ref]
                        it[name] = None
                where[m] = len(out)
                out.append(it)
                level.append(lv)
                src.append(((g, q), m))
    return out, level, src


def serve(srv, its, pool=None, arrivals=None, poll_every=16, start_of=None):
    """Decode session-style items through a server (native.Server) and poll to
    completion.  pool None: every item, each submitted as soon as the items it
    references (past_from / future_from) are done, their decoded frames passed
    as its references; else request k is item pool[k % len(pool)] (items
    without references), submitted once arrivals[k] seconds have passed.
    start_of(i), when given, is item i's starting content (its "recon"), or
    None while that is not ready; the item waits for it.  During a burst of
    submissions the server is also polled after every `poll_every` of them, so
    that cohorts start while the rest are still being submitted.  Returns
    (seconds, latencies in ms, results by item)."""
    n_req = len(its) if pool is None else len(arrivals)
    tickets, lat, res = {}, [], {}
    waiting = list(range(n_req))
    done = 0

    def pump():
        """One poll; collects every ticket finished so far.  False when the poll finished nothing."""
        nonlocal done
        if not srv.poll():
            return False
        for t in srv.finished():
            r = srv.result(t)
            lat.append(r["latency_ms"])
            res[tickets.pop(t)] = r
            done += 1
        return True

    t0 = time.perf_counter()
    while done < n_req:
        now = time.perf_counter() - t0
        still, burst = [], 0
        for k in waiting:
            i = k if pool is None else pool[k % len(pool)]
            it = its[i]
            deps = [it.get("past_from"), it.get("future_from")]
            if (arrivals is not None and arrivals[k] > now) or any(d is not None and d not in res for d in deps):
                still.append(k)
                continue
            if start_of is not None:
                rec = start_of(i)
                if rec is None:
                    still.append(k)
                    continue
                it = dict(it, recon=rec)
            if deps[0] is not None or deps[1] is not None:
                it = dict(it)
                for name, d in zip(("past", "future"), deps):
                    if d is not None:
                        it[name] = res[d]["recon"]
                        it.pop(name + "_from")
            tickets[srv.submit(it)] = i
            burst += 1
            if burst % poll_every == 0:
                pump()
        waiting = still
        if not pump():
            time.sleep(0.0002)
    return time.perf_counter() - t0, lat, res


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 4 + i and r[4 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


class RefStreams:
    """The bench workload for the reference's own CPU codec: the same synthetic
    sequence (dvc_b200.synth, numpy only) written to YUV files and every
    (GOP, QIndex) stream encoded by the reference encoder (oracle/_ref/DvcEnc,
    SkipBlock 1, IntraMode 1, DeblockingFilter 1, IntraQP 30), so that the
    process timing the reference loads none of this repository's native code.
    Samples are whole GOPs decoded by the reference decoder (oracle/_ref/DvcDec)
    with its -startFrame/-endFrame range; the time is the decoder's own
    "Total decoding time" (its timed region, DvcDec/src/main.cpp:109-145)."""

    def __init__(self, workdir):
        from oracle import refrun
        from dvc_b200 import synth
        self.refrun = refrun
        ori, key = synth.make_sequence(KIND, N_FRAMES, SEED)
        self.dir = workdir
        self.oy, self.ky = os.path.join(workdir, "ori.yuv"), os.path.join(workdir, "key.yuv")
        self.stat = os.path.join(workdir, "stat.txt")
        synth.write_yuv420(self.oy, ori)
        synth.write_yuv420(self.ky, key)
        synth.write_frame_stat(self.stat, N_FRAMES)
        self.streams = {}
        for g in GOPS:
            for q in QS:
                d = refrun._workdir(workdir)  # holds the ladder directory the encoder opens
                wz, ib, _ = refrun.encode(self.oy, self.ky, N_FRAMES, "CIF", g, q, skip=1, intra=1,
                                          intra_qp=INTRA_QP, deblock=1, workdir=d)
                self.streams[(g, q)] = (wz, ib)

    @staticmethod
    def wz_frames(g):
        """WZ frames of a (g) stream in the bench workload."""
        return sum(e - b - 1 for b, e in ((i, min(i + g, N_FRAMES - 1)) for i in range(0, N_FRAMES - 1, g)))

    def decode_gop(self, gq, k, mode, cores):
        """Decode GOP k of stream gq; returns (decoder seconds, WZ frames decoded)."""
        g = gq[0]
        wz, ib = self.streams[gq]
        r = self.refrun.decode(self.oy, wz, ib, self.ky, self.stat, mode=mode, cores=cores, start=k * g,
                               end=(k + 1) * g)
        t = None
        for line in r["rd"].splitlines():
            if line.startswith("Total decoding time:"):
                t = float(line.split(":")[1].split()[0])
        return (t if t else r["seconds"]), g - 1


def ref_encoder_session(ctx, rs, key, args):
    """WZ frames/s of the batched session on the reference encoder's streams
    of the workload (RefStreams): the same timing as `value`."""
    import torch
    from dvc_b200 import bitstream as bs
    streams = {gq: bs.parse_wz(open(wz, "rb").read()) for gq, (wz, ib) in rs.streams.items()}
    intra_bs = {gq: open(ib, "rb").read() for gq, (wz, ib) in rs.streams.items()}
    its, lev, src = items(streams, key, intra_starts(streams, intra_bs, key))
    ses = ctx.session(its, max_batch=args.max_batch, streams=args.streams)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    try:
        for _ in range(3):
            ses.run()
        ms = []
        for _ in range(max(3, args.steps)):
            flush.zero_()
            torch.cuda.synchronize()
            ms.append(ses.run())
    finally:
        ses.close()
    return {"value": len(its) / (float(np.mean(ms)) / 1e3), "unit": "WZ frames/s", "frames": len(its),
            "ms_per_step": float(np.mean(ms)),
            "note": "the workload's 16 streams encoded by the reference encoder (its skip and intra decisions), "
                    "decoded by the batched session as for value"}


def ref_plan(n_samples, per_step=4):
    """A fixed stratified sample of the workload: step i decodes one GOP of each
    of `per_step` streams, cycling through all (GOP, QIndex) streams; the GOP
    index moves along each stream's sequence from one visit to the next, so a
    run covers every stream, both levels of GOP 4 and several parts of the
    sequences."""
    keys = [(g, q) for g in GOPS for q in QS]
    plan = []
    for i in range(n_samples):
        step = []
        for j in range(per_step):
            c = i * per_step + j
            gq = keys[c % len(keys)]
            visit = c // len(keys)
            n_gops = (N_FRAMES - 1) // gq[0]
            step.append((gq, (7 * visit + 3 * QS.index(gq[1])) % n_gops))
        plan.append(step)
    return plan


def ref_estimate(samples):
    """WZ frames/s of the whole workload from per-stream samples: every stream's
    seconds per WZ frame, weighted by its share of the workload's frames
    (streams not sampled are left out of both sides)."""
    per = {}
    for gq, t, n in samples:
        a = per.setdefault(gq, [0.0, 0])
        a[0] += t
        a[1] += n
    frames = sum(RefStreams.wz_frames(gq[0]) for gq in per)
    secs = sum(RefStreams.wz_frames(gq[0]) * t / n for gq, (t, n) in per.items())
    return frames / secs, frames


def run_reference(args, rank):
    if rank != 0:
        return
    from oracle import refrun
    if not refrun.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (make -C oracle ref)"}))
        return
    cores = os.cpu_count() or 1
    rs = RefStreams(tempfile.mkdtemp())
    plan = ref_plan(args.warmup + args.steps)
    for step in plan[:args.warmup]:
        for gq, k in step:
            rs.decode_gop(gq, k, 1, cores)
    samples, step_s = [], []
    for step in plan[args.warmup:]:
        tot = 0.0
        for gq, k in step:
            t, n = rs.decode_gop(gq, k, 1, cores)
            samples.append((gq, t, n))
            tot += t
        step_s.append(tot)
    fps, covered = ref_estimate(samples)
    # ParallelMode 0 (the sequential decoder, one core) on one GOP-2 frame at QIndex 4
    t0, n0 = rs.decode_gop((2, 4), 0, 0, 1)
    total_frames = sum(RefStreams.wz_frames(g) for g in GOPS for _ in QS)
    line = {"impl": "reference", "metric": METRIC, "value": fps, "unit": "WZ frames/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(step_s)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
            "config": {"workload": "CIF 352x288, 65-frame sequences at GOP 2 and GOP 4, QIndex 1..8 -> %d WZ frames "
                                   "(SkipBlock 1, IntraMode 1, DeblockingFilter 1, IntraQP 30), encoded by the "
                                   "reference encoder; reference DvcDec ParallelMode 1 on every host core"
                                   % total_frames,
                       "frames_per_step": float(np.mean([sum(g - 1 for (g, _), _ in st) for st in plan[args.warmup:]])),
                       "estimate": "stratified: seconds per WZ frame of each (GOP, QIndex) stream from its "
                                   "sampled GOPs, weighted by the stream's frames in the workload",
                       "frames_covered": covered, "samples": len(samples)},
            "cpu_baseline": {"value": fps, "unit": "WZ frames/s", "cores": cores, "kind": "reference",
                             "sample": "%d GOPs over the %d streams (4 per step), reference DvcDec ParallelMode 1, "
                                       "decoder-reported decoding time" % (len(samples), len(GOPS) * len(QS))},
            "mode0": {"value": n0 / t0, "unit": "WZ frames/s", "cores": 1,
                      "sample": "reference DvcDec ParallelMode 0 (sequential), the first GOP-2 WZ frame at QIndex 4"},
            "e2e": {"value": fps, "unit": "WZ frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed 64-stream serving workload")
    ap.add_argument("--max-batch", type=int, default=16)
    ap.add_argument("--streams", type=int, default=16)
    args = ap.parse_args()
    # one hardware queue per CUDA stream (the default 8 makes the 16 decode
    # streams share queues and wait behind each other's launches); before CUDA
    # starts, and a value set by the caller wins
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import torch.distributed as dist
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    from dvc_b200 import native

    ori, key, streams, intra_bs = workload()
    its, lev, src = items(streams, key, intra_starts(streams, intra_bs, key))
    ctx = native.Context(local)
    ses = ctx.session(its, max_batch=args.max_batch, streams=args.streams)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        ses.run()
    barrier()
    dev_ms = []
    with Clocks(local) as clk:
        barrier()
        for i in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            dev_ms.append(ses.run())
        barrier()
    # kernel-level figures from one more, untimed run (a profiled run records an
    # event pair around every LDPCA launch and is not replayed as a graph)
    flush.zero_()
    ses.run(profile=True)
    prof = ses.profile()
    from dvc_b200 import replicas
    step_ms = replicas.max_over_ranks(float(np.mean(dev_ms)))
    frames_per_step = len(its)
    value = world * frames_per_step / (step_ms / 1e3)

    # parity spot check of the timed path against a second decode path
    rec0, bits0, planes0 = ses.frame(0)
    # belief-propagation work of one step: block-iterations summed over every
    # bitplane's ladder (speculative blocks included)
    bp_iters = int(sum(int(ses.frame(i)[2][:, 3].sum()) for i in range(len(its))))

    # e2e through the public serving API with host buffers: submit a whole step, wait for it
    fs = 352 * 288
    qb = sum(len(it["crc"]) for it in its)
    h2d = sum(2 * fs + fs + it["acc"].nbytes + it["crc"].nbytes + 64 + 16 * 4 for it in its)
    d2h = len(its) * fs + qb * 20
    srv = ctx.server(mem_budget_bytes=16 << 30, streams=args.streams, max_cohort=args.max_batch)

    level0 = [i for i in range(len(its)) if lev[i] == 0]

    def serve_all(pool=None, arrivals=None):
        return serve(srv, its, pool, arrivals)

    from concurrent.futures import ThreadPoolExecutor
    intra_pool = ThreadPoolExecutor(max_workers=min(len(streams), os.cpu_count() or 1))

    def e2e_step():
        """One step end to end: every stream's intra blocks decoded on the host
        pool (the host part of the decode) while the server already decodes the
        frames whose starting content is ready."""
        fut = intra_starts_async(intra_pool, streams, intra_bs, key)

        def start_of(i):
            gq, m = src[i]
            f = fut[gq]
            return f.result()[m] if f.done() else None

        return serve(srv, its, start_of=start_of)

    e2e_step()  # warm
    barrier()
    e2e_t = []
    for _ in range(max(1, args.steps)):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, _, served = e2e_step()
        e2e_t.append(time.perf_counter() - t0)
    intra_pool.shutdown()
    barrier()
    e2e_s = replicas.max_over_ranks(float(np.mean(e2e_t)))
    # the served results equal the session's (both bit-exact paths), second level included
    for i in (0, len(its) // 2, len(its) - 1, max(i for i in range(len(its)) if lev[i] > 0)):
        rec_i, bits_i, _ = ses.frame(i)
        assert np.array_equal(served[i]["recon"], rec_i) and served[i]["wz_bits"] == bits_i

    # served: Poisson arrivals at fractions of the measured device capacity
    capacity = frames_per_step / (step_ms / 1e3)
    served_sweep = []
    for frac in (0.25, 0.5, 0.7, 0.9):
        rate = frac * capacity
        rng = np.random.default_rng(7)
        n_req = max(64, int(rate * 2.0))
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
        srv_dt, srv_lat, _ = serve_all(level0, arrivals)
        served_sweep.append({"offered_rate": rate, "throughput": n_req / srv_dt, "requests": n_req,
                             "p50_ms": float(np.percentile(srv_lat, 50)), "p99_ms": float(np.percentile(srv_lat, 99))})
    srv.close()
    served_main = served_sweep[2]

    # the mixed serving workload: 64 streams (48 QCIF, 16 CIF), GOP 2/4/8,
    # QIndex 1..8, Poisson arrivals, 16 GB budget (dvc_b200.serve_bench)
    mixed = None
    if not args.no_mixed:
        from dvc_b200 import serve_bench as sb
        t_build = time.perf_counter()
        mreqs = sb.build(17)
        t_build = time.perf_counter() - t_build
        msrv = ctx.server(mem_budget_bytes=16 << 30, streams=args.streams, max_cohort=args.max_batch)
        sb.serve(msrv, mreqs, np.zeros(len(mreqs)))  # warm
        msweep = []
        for rate in (300.0, 1000.0, 5000.0):
            arr = np.cumsum(np.random.default_rng(7).exponential(1.0 / rate, len(mreqs)))
            dt, lat, mserved = sb.serve(msrv, mreqs, arr)
            msweep.append({"offered_rate": rate, "throughput": len(mreqs) / dt, "p50_ms": float(np.percentile(lat, 50)),
                           "p99_ms": float(np.percentile(lat, 99))})
        msrv.close()
        # the plain drop-in on the same requests (one dvc_decode_wz_frames call each, in order)
        pres, plat = {}, []
        for k, it in enumerate(mreqs):
            sub = {key: v for key, v in it.items() if not key.startswith("_")}
            for name, d in zip(("past", "future"), (it["past_idx"], it["future_idx"])):
                for dep in it["_deps"]:
                    if mreqs[dep]["_frame"] == d:
                        sub[name] = pres[dep]
            t1 = time.perf_counter()
            pres[k] = ctx.decode_wz_frames([sub])[0]["recon"]
            plat.append(time.perf_counter() - t1)
        mixed = {"workload": "64 streams (48 QCIF SkipBlock 0 IntraMode 0, 16 CIF SkipBlock 1 IntraMode 1 "
                             "DeblockingFilter 1), GOP 2/4/8, QIndex 1..8, 17 frames each, Poisson arrivals, "
                             "16 GB budget", "requests": len(mreqs), "sweep": msweep,
                 "plain": {"throughput": len(mreqs) / sum(plat), "p50_ms": 1e3 * float(np.percentile(plat, 50)),
                           "p99_ms": 1e3 * float(np.percentile(plat, 99))},
                 "served_equals_plain": all(np.array_equal(mserved[k], pres[k]) for k in range(len(mreqs))),
                 "build_s": t_build}

    # plain one-frame-at-a-time drop-in: one first-level frame per Q
    plain_lat = []
    for q in QS:
        it = its[min(i for i in level0 if its[i]["qindex"] == q)]
        ctx.decode_wz_frames([it])
        t0 = time.perf_counter()
        ctx.decode_wz_frames([it])
        plain_lat.append(time.perf_counter() - t0)
    plain_fps = len(plain_lat) / sum(plain_lat)

    # roofline of the dominant kernel (the LDPCA ladder).  Unit: one belief-
    # propagation iteration of one thread block on a CIF codeword; its
    # algorithmic DRAM bytes are the phi-table reads, one 4-byte entry per edge
    # in each of the two message passes (2 * 19008 * 4); messages, signs and
    # row sums stay in shared memory.
    E_CIF = 19008
    alg_bytes_unit = 2 * E_CIF * 4
    ld_avg_ms = prof["ldpca_ms"] / max(1, prof["ldpca_launches"])
    cw_per_launch = prof["ldpca_codewords"] / max(1, prof["ldpca_launches"])
    units_per_launch = bp_iters / max(1, prof["ldpca_launches"])
    achieved = alg_bytes_unit * units_per_launch / (ld_avg_ms / 1e3) / 1e9
    aggregate = alg_bytes_unit * bp_iters / (step_ms / 1e3) / 1e9
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        peak, peak_src = float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "ldpca_traffic.json")
    if os.path.exists(tpath):
        per_unit = json.load(open(tpath)).get("dram_bytes_per_block_iteration")
        if per_unit is not None:
            traffic = per_unit * units_per_launch
    # compulsory device I/O of the whole decode, per CIF WZ frame: the past and
    # future frames, their two 4x-size half-pel planes, the decoded frame, each
    # bitplane's accumulated syndrome (N/8 bytes, N = 6336) and CRC byte, and the
    # 8x8 block-mode map; over the batched step time, against the same peak
    frame_io = len(its) * (11 * fs + fs // 64) + qb * (6336 // 8 + 1)
    frame_io_gbs = frame_io / (step_ms / 1e3) / 1e9

    cpu, ref_enc = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import refrun
            if refrun.ref_available():
                cores = os.cpu_count() or 1
                rs = RefStreams(tempfile.mkdtemp())
                samples = [(gq, *rs.decode_gop(gq, k, 1, cores)) for gq, k in ref_plan(4)[0] + ref_plan(4)[2]]
                fps, _ = ref_estimate(samples)
                cpu = {"value": fps, "unit": "WZ frames/s", "cores": cores, "kind": "reference",
                       "sample": "8 GOPs of 8 streams (GOP 2 and 4, QIndex 1-4 and 5-8 in turn) of the same sequence, "
                                 "encoded by the reference encoder, reference DvcDec ParallelMode 1 with every core "
                                 "(decoder-reported decoding time), weighted by the streams' frames"}
                # the same 640 frames with the reference encoder's mode decisions (the streams the
                # reference arm decodes), through the same device-resident session
                ref_enc = ref_encoder_session(ctx, rs, key, args)
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "WZ frames/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": "failed: %s" % str(ex)[:200]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "WZ frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32/f64 (reference arithmetic, bit-exact)", "data": "synthetic",
            "config": {"workload": "CIF 352x288, 65-frame sequences at GOP 2 and GOP 4, QIndex 1..8 -> %d WZ "
                                   "frames per step in two dependent levels (SkipBlock 1, IntraMode 1, "
                                   "DeblockingFilter 1, IntraQP 30)"
                                   % frames_per_step,
                       "frames_per_step": frames_per_step, "max_batch": args.max_batch, "streams": args.streams,
                       "l2": "flushed (256 MB write) before every timed step",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "e2e": {"value": world * frames_per_step / e2e_s, "unit": "WZ frames/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "plain": {"value": plain_fps, "unit": "WZ frames/s",
                      "p50_ms": 1e3 * float(np.percentile(plain_lat, 50)),
                      "p99_ms": 1e3 * float(np.percentile(plain_lat, 99)), "frames": len(plain_lat)},
            "served": dict(served_main, unit="WZ frames/s",
                           arrivals="Poisson at 70% of the batched capacity, first-level frames",
                           streams=args.streams, max_cohort=args.max_batch, sweep=served_sweep),
            "served_mixed": mixed,
            "roofline": {"bound": "hbm", "kernel": "ldpca_ladder_kernel", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                         "unit_of_work": "BP block-iteration on a CIF codeword, %d algorithmic bytes (phi-table "
                                         "reads)" % alg_bytes_unit,
                         "units_per_launch": units_per_launch,
                         "aggregate_achieved": aggregate, "aggregate_frac": aggregate / peak,
                         "frame_io": {"bytes_per_frame": frame_io / len(its), "achieved": frame_io_gbs,
                                      "frac": frame_io_gbs / peak,
                                      "note": "compulsory I/O of the whole WZ-frame decode (references, half-pel "
                                              "planes, output, syndromes and CRCs, mode map) at the batched rate: "
                                              "the path is bound by its gathers and compute, not by moving "
                                              "these bytes"},
                         "note": "4-byte phi values gathered at random, one 16-byte record each through the "
                                 "texture path, from a packed 166 MB table whose hot part mostly stays in L2 (84% "
                                 "L2 hits, ~125 KB of DRAM traffic per block-iteration in ncu); the kernel is bound "
                                 "by the latency of those gathers, not by DRAM bandwidth.  Launches of 16 streams "
                                 "overlap, so the per-launch figure understates the device-wide rate "
                                 "(aggregate_achieved: all launches of a step over the step time)"},
            "cpu_baseline": cpu,
            "value_reference_encoder_streams": ref_enc,
            "clocks": clk.summary(),
            "gpu_launches": int(prof["kernel_launches"]) * args.steps,
            "graph_replays": ses.replays(),
            "ldpca": {"ms_per_launch": ld_avg_ms, "codewords_per_launch": cw_per_launch,
                      "kernel_ms_per_step": prof["ldpca_ms"],
                      "bp_block_iterations_per_step": bp_iters,
                      "bp_block_iterations_per_s": bp_iters / (step_ms / 1e3)},
        }
        print(json.dumps(line))
    ses.close()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
