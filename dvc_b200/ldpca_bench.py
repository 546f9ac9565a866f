"""Batched LDPCA microbenchmark: many independent codewords in one launch.

    python -m dvc_b200.ldpca_bench [--count 8192] [--max-iter 50|100] [--seed 11] [--per-length]

Codewords (seeded): source bits x ~ Bernoulli(0.5); the side information
flips each bit with a per-codeword probability p ~ U[0.01, 0.25]; the
intrinsic likelihood ratio of bit k is (1-p)/p where the side information
bit is 0 and p/(1-p) where it is 1 (so log LR = +-log((1-p)/p), float32);
the accumulated syndrome and CRC-8 come from the encoder construction
(LdpcaEncoder.cpp:64-95).  Each codeword walks the request ladder from its
seeded request level (seeded_starts) to the first code whose BP converges
with a matching CRC (or the full-rate inverse), as LdpcaDecoder does
(LdpcaDecoder.cpp:646-771); the reference stops BP after 50 iterations
(LdpcaDecoder.h:4), --max-iter 100 gives the longer variant.  All 8192
codewords, QCIF and CIF interleaved, go to the device in one
dvc_ldpca_decode_batch call: one persistent launch whose work queue hands out
(codeword, ladder code) pairs over every SM.  The line printed reports
codewords/s over the launch's device time and over the whole call, the BP
iterations run, how many codewords decode to their source, and how many equal
the reference decoder's result (rate, accepted code, decoded bits) recorded in
tests/golden/ldpca_batch.npz.  --per-length also times the frame path's kernel
on the same codewords (one launch per length, entropy-bound starts).
"""
import argparse
import json
import os
import time

import numpy as np

from . import encoder


def make_codewords(n, count, seed):
    """(lr float32 [count,n], acc bytes uint8 [count,n/8], crc uint8 [count], x uint8 [count,n])."""
    rng = np.random.default_rng(seed)
    L = encoder._ladder(n)
    x = rng.integers(0, 2, (count, n), dtype=np.uint8)
    p = rng.uniform(0.01, 0.25, count).astype(np.float32)
    flip = (rng.random((count, n)) < p[:, None]).astype(np.uint8)
    y = x ^ flip
    hi = ((np.float32(1) - p) / p).astype(np.float32)
    lo = (p / (np.float32(1) - p)).astype(np.float32)
    lr = np.where(y == 0, hi[:, None], lo[:, None]).astype(np.float32)
    acc = np.stack([np.packbits(encoder.accumulated_syndrome(L, x[i]), bitorder="big") for i in range(count)])
    crc = np.array([encoder.crc8_bits(x[i]) for i in range(count)], np.uint8)
    return lr, acc, crc, x


def code_rates(n):
    """Rate of each ladder code as the decoder compares it (syndrome length / n, float32)."""
    L = encoder._ladder(n)
    m = [(n // L["period"]) * b for b in L["bpp"]]
    return np.array([np.float32(x) / np.float32(n) for x in m], np.float32)


def seeded_starts(n, count, seed):
    """Seeded request level of each codeword of make_codewords(n, count, seed):
    the first ladder code whose rate reaches the binary entropy h(p) of the
    codeword's flip probability, moved by a seeded offset in [-3, 2] and kept
    below full rate.  The decoder starts its ladder there instead of at the
    code its own conditional-entropy bound selects."""
    rng = np.random.default_rng(seed)
    rng.integers(0, 2, (count, n), dtype=np.uint8)  # the draws of make_codewords, in order
    p = rng.uniform(0.01, 0.25, count).astype(np.float32).astype(np.float64)
    h = -(p * np.log2(p) + (1.0 - p) * np.log2(1.0 - p))
    rates = code_rates(n).astype(np.float64)
    base = np.searchsorted(rates, h, side="left")
    off = np.random.default_rng(seed + 1).integers(-3, 3, count)
    return np.clip(base + off, 0, len(rates) - 2).astype(np.int32)


def run(ctx, lr, acc, crc, max_iter, reps=3):
    """Decode every codeword `reps` times; returns (results, best seconds)."""
    ctx.ldpca_decode(lr[:1], acc[:1], crc[:1], max_iter)  # warm
    best, out = None, None
    for _ in range(reps):
        t0 = time.perf_counter()
        out = ctx.ldpca_decode(lr, acc, crc, max_iter)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    return out, best


def interleaved(count, seed):
    """The mixed workload: count/2 codewords of each length, alternating
    QCIF and CIF, with their seeded start levels.  Returns (lengths, lr, acc,
    crc, start, sources, (length, index) of each codeword)."""
    parts = []
    for n in (1584, 6336):
        c = count // 2
        lr, acc, crc, x = make_codewords(n, c, seed + n)
        parts.append((n, lr, acc, crc, seeded_starts(n, c, seed + n), x))
    where = [(n, i) for i in range(count // 2) for n in (1584, 6336)]
    get = {1584: parts[0], 6336: parts[1]}
    lengths = np.array([n for n, _ in where], np.int32)
    lr = np.concatenate([get[n][1][i] for n, i in where])
    acc = np.concatenate([get[n][2][i] for n, i in where])
    crc = np.array([get[n][3][i] for n, i in where], np.uint8)
    start = np.array([get[n][4][i] for n, i in where], np.int32)
    src = [get[n][5][i] for n, i in where]
    return lengths, lr, acc, crc, start, src, where


def reference_agreement(res, dec, lengths, where, seed, count):
    """Codewords whose rate, accepted code and decoded bits equal the reference
    decoder's (the committed per-codeword results of the reference's
    LdpcaDecoder on this workload, tests/golden/ldpca_batch.npz), or None when
    that file is absent or holds another workload."""
    import hashlib
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                        "ldpca_batch.npz")
    if not os.path.exists(path):
        return None
    g = np.load(path)
    if int(g["count"]) != count or int(g["seed"]) != seed:
        return None
    off = np.concatenate([[0], np.cumsum(lengths)])
    ok = 0
    for k, (n, i) in enumerate(where):
        d = dec[off[k]:off[k + 1]]
        h = int.from_bytes(hashlib.blake2b(d.tobytes(), digest_size=8).digest(), "little")
        ok += int(res[k, 0] == g["n%d_rate" % n][i] and res[k, 2] == g["n%d_accepted" % n][i]
                  and h == int(g["n%d_decoded_hash" % n][i]))
    return ok


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=8192)
    ap.add_argument("--max-iter", type=int, default=50)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--per-length", action="store_true",
                    help="also time the frame path's ladder kernel: one dvc_ldpca_decode launch per length, "
                         "start levels from the entropy bound")
    args = ap.parse_args()
    from . import native
    lengths, lr, acc, crc, start, src, where = interleaved(args.count, args.seed)
    ctx = native.Context(0)
    ctx.ldpca_decode_batch(lengths[:2], lr[:1584 + 6336], acc[:(1584 + 6336) // 8], crc[:2], start[:2],
                           args.max_iter)  # warm
    best = None
    for _ in range(args.reps):
        t0 = time.perf_counter()
        dec, res, ent, work, ms = ctx.ldpca_decode_batch(lengths, lr, acc, crc, start, args.max_iter)
        wall = time.perf_counter() - t0
        if best is None or ms < best[1]:
            best = (wall, ms, work)
    wall, ms, work = best
    off = np.concatenate([[0], np.cumsum(lengths)])
    equal_src = sum(int(np.array_equal(dec[off[k]:off[k + 1]], src[k])) for k in range(len(lengths)))
    agree = reference_agreement(res, dec, lengths, where, args.seed, args.count) if args.max_iter == 50 else None
    line = {"workload": "LDPCA batched microbench (one persistent launch)", "codewords": int(len(lengths)),
            "lengths": "1584/6336 interleaved", "max_iter": args.max_iter, "start": "seeded level",
            "codewords_per_s": len(lengths) / (ms / 1e3), "kernel_ms": ms,
            "codewords_per_s_e2e": len(lengths) / wall, "call_ms": wall * 1e3,
            "bp_iterations": int(work), "bp_iterations_per_s": work / (ms / 1e3),
            "ladder_bp_iterations": int(res[:, 3].sum()),
            "decoded_equal_source": equal_src, "reference_agreement": agree}
    print(json.dumps(line))
    if args.per_length:
        total_t, total_it = 0.0, 0
        for n in (1584, 6336):
            sel = [k for k in range(len(lengths)) if lengths[k] == n]
            l2 = np.stack([lr[off[k]:off[k + 1]] for k in sel])
            a2 = np.stack([acc[off[k] // 8:off[k + 1] // 8] for k in sel])
            (d2, r2, e2), t = run(ctx, l2, a2, crc[sel], args.max_iter, args.reps)
            total_t += t
            total_it += int(r2[:, 3].sum())
        print(json.dumps({"workload": "LDPCA per-length launches (frame path kernel, entropy-bound start)",
                          "codewords": int(len(lengths)), "codewords_per_s": len(lengths) / total_t,
                          "seconds": total_t, "ladder_bp_iterations": total_it}))
    ctx.close()


if __name__ == "__main__":
    main()
