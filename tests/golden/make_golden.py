"""Generate the committed golden fixtures from the reference codec.

Runs oracle/_ref (the reference DvcEnc/DvcDec built from its own sources by
oracle/Makefile) on seeded synthetic sequences and stores what the reference
decoder computed:

  seq_<name>.npz   WZ bitstream bytes, the sequence parameters (the synthetic
                   frames are regenerated from the seed), the reference's
                   decoded Y for every frame, per-frame bits and PSNR from its RD
                   report, and per-bitplane LDPCA records (start code, accepted
                   code, rate, entropy) captured through oracle/ref_capture.cpp.
  ldpca_<n>.npz    LDPCA known-answer vectors: LR, accumulated syndrome bytes,
                   CRC, and the reference's entropy bound, rate, decoded bits.
  jbig_maps.npz    mode maps coded by the reference's JBIG encoder, with the
                   map its JBIG decoder returns and the bytes it consumes
                   (oracle/_ref/libjbig{enc,dec}.so, oracle/jbig_ref.cpp).

The *_skip sequences are encoded with SkipBlock 1 on still-camera content, so
their WZ frames carry JBIG-coded skip maps; the *_intra sequences with
SkipBlock 1 and IntraMode 1, so they also carry intra maps and an intra
bitstream (stored as ``intra``); the *_full sequences add DeblockingFilter 1.

Every sequence fixture also holds the likelihood ratios the reference passed
to LdpcaDecoder for the bitplanes of its first decoded WZ frame (condBitProb's
output, noiseModel.cpp:191-310): a 64-bit digest of each bitplane's float
bytes (``lr0_hash``) and the first bitplanes in full (``lr0_head``).

  bench_first_gops.npz  the first GOP of every (GOP, QIndex) stream of the
                   bench.py workload (CIF, 65-frame sequences, seed, IntraQP,
                   SkipBlock 1, IntraMode 1, DeblockingFilter 1), encoded once
                   by the reference encoder and once by dvc_b200.encoder (the
                   bench's own streams), decoded by the reference: per WZ frame
                   a digest of the decoded Y, bits and PSNR; per bitplane the
                   first and accepted ladder codes and the entropy bound.
  ldpca_batch.npz  the batched LDPCA workload (dvc_b200.ldpca_bench: 8192
                   codewords, half of each length, seeded flip probability and
                   start level): per codeword the reference LdpcaDecoder's rate
                   and a digest of its decoded bits (oracle/ldpca_ref.cpp).
  ranges.npz       the reference decoder run with -startFrame/-endFrame on
                   committed sequences: its decoded luma and RD report.
  ldpca_fullrate.npz codewords so noisy that no ladder code below full rate
                   decodes them, so the reference ends at the GF(2) inverse
                   (LdpcaDecoder.cpp:695-716): LR, accumulated syndrome, CRC,
                   rate and decoded bits.

Usage (in the build container, after `make -C oracle ref` and
`python oracle/ladder_dir.py oracle/_ref`):
    python tests/golden/make_golden.py [fixture names] [-j N]   # default: all
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "dvc_b200", "ladders"))
os.environ.setdefault("OMP_NUM_THREADS", "1")

from dvc_b200 import synth  # noqa: E402
from oracle import refrun  # noqa: E402
import ladders as lad  # noqa: E402

# name: (kind, frames, gop, qindex, seed[, skip[, intra[, deblock[, own]]]]); own=1: the
# bitstreams come from this package's encoder (dvc_b200.encoder, skip and intra
# decisions of its own) instead of the reference encoder, and are decoded by the
# reference decoder as usual
SEQUENCES = {
    "qcif_g2_q4": ("qcif", 5, 2, 4, 11),
    "qcif_g4_q8": ("qcif", 5, 4, 8, 12),
    "qcif_g2_q1": ("qcif", 3, 2, 1, 13),
    "cif_g2_q2": ("cif", 3, 2, 2, 21),
    "qcif_still_g2_q4_skip": ("qcif_still", 5, 2, 4, 41, 1),
    "cif_still_g4_q6_skip": ("cif_still", 5, 4, 6, 42, 1),
    "qcif_g2_q4_intra": ("qcif", 5, 2, 4, 11, 1, 1),
    "cif_g4_q6_intra": ("cif", 5, 4, 6, 21, 1, 1),
    "qcif_g4_q8_allintra": ("qcif", 5, 4, 8, 12, 1, 1),
    "qcif_g2_q4_full": ("qcif", 5, 2, 4, 11, 1, 1, 1),
    "cif_g4_q6_full": ("cif", 5, 4, 6, 21, 1, 1, 1),
    "qcif_still_g4_q4_full": ("qcif_still", 5, 4, 4, 41, 1, 1, 1),
    "cif_g4_q4_own_full": ("cif", 9, 4, 4, 21, 1, 1, 1, 1),
    "qcif_g2_q8_own_full": ("qcif", 5, 2, 8, 12, 1, 1, 1, 1),
    "qcif_still_g4_q4_own_full": ("qcif_still", 5, 4, 4, 41, 1, 1, 1, 1),
    "qcif_g2_q4_db": ("qcif", 5, 2, 4, 11, 0, 0, 1),
    "qcif_g4_q6_db": ("qcif", 5, 4, 6, 14, 0, 0, 1),
    "cif_fast_g8_q8_own_full": ("cif_fast", 9, 8, 8, 51, 1, 1, 1, 1),
    "cif_fast_g8_q4_own_full": ("cif_fast", 9, 8, 4, 52, 1, 1, 1, 1),
    # the configuration the benchmark times (CIF, SkipBlock 1, IntraMode 1,
    # DeblockingFilter 1) at the QIndex values not covered above, GOP 2 and 4
    "cif_g2_q1_full": ("cif", 9, 2, 1, 61, 1, 1, 1),
    "cif_g4_q3_full": ("cif", 9, 4, 3, 62, 1, 1, 1),
    "cif_g2_q5_full": ("cif", 9, 2, 5, 63, 1, 1, 1),
    "cif_g4_q7_full": ("cif", 9, 4, 7, 64, 1, 1, 1),
    "cif_g4_q8_full": ("cif", 9, 4, 8, 65, 1, 1, 1),
    # QIndex 8 with every block Wyner-Ziv coded (IntraMode 0): 15 bands, 63 bitplanes
    "cif_g2_q8_wz": ("cif", 9, 2, 8, 66, 1, 0, 1),
    # the reference's plain CPU run: QCIF, 17 frames, GOP 2, QIndex 4, all options off
    "qcif_g2_q4_cfg0": ("qcif", 17, 2, 4, 71),
}

LR0_HEAD = 4  # bitplanes of the first WZ frame stored in full


def run(name, kind, n_frames, gop, q, seed, tmp, skip=0, intra=0, deblock=0, own=0):
    w, h = synth.SHAPES[kind]
    size = "QCIF" if w == 176 else "CIF"
    ori, key = synth.make_sequence(kind, n_frames, seed)
    d = os.path.join(tmp, name)
    os.makedirs(d, exist_ok=True)
    oy, ky, st = os.path.join(d, "ori.yuv"), os.path.join(d, "key.yuv"), os.path.join(d, "stat.txt")
    synth.write_yuv420(oy, ori)
    synth.write_yuv420(ky, key)
    synth.write_frame_stat(st, n_frames)
    if own:
        from dvc_b200 import encoder
        wzb, ib = encoder.encode_sequence_intra(ori, gop, q, 30, deblock, skip, intra)
        wz, intra_bs = os.path.join(d, "s.wz"), os.path.join(d, "s.intra")
        open(wz, "wb").write(wzb)
        open(intra_bs, "wb").write(ib)
    else:
        wz, intra_bs, _ = refrun.encode(oy, ky, n_frames, size, gop, q, skip=skip, intra=intra, deblock=deblock)
    cap = os.path.join(d, "cap.bin")
    r = refrun.decode(oy, wz, intra_bs, ky, st, mode=0, capture=cap)
    dec_y = np.frombuffer(r["yuv"], np.uint8).reshape(-1, h, w)
    rd = refrun.parse_rd(r["rd"])
    caps = refrun.read_capture(cap)
    recs = refrun.ldpca_records(caps)
    L = lad.ladder_for(lad.read_compact(os.path.join(ROOT, "dvc_b200", "ladders", "ldpca_ladders.bin")), w * h // 16)
    nc, n, e, period, jc, codes = lad.expand(L)
    synd = [(n // period) * c[0] for c in codes]
    rate_f = np.array(synd, np.float32) / np.float32(n)
    starts, accepted = [], []
    for rec in recs:
        s = 0
        while s < nc - 1 and rate_f[s] < np.float32(rec["entropy"]):
            s += 1
        starts.append(s)
        accepted.append(synd.index(rec["rate"] - 8))
    frames = sorted(rd)
    np.savez_compressed(
        os.path.join(HERE, f"seq_{name}.npz"),
        kind=kind, n_frames=n_frames, gop=gop, qindex=q, seed=seed, skip=skip, own=own,
        wz=np.frombuffer(open(wz, "rb").read(), np.uint8),
        intra=np.frombuffer(open(intra_bs, "rb").read(), np.uint8),
        dec_y=dec_y,
        frames=np.array(frames), bits=np.array([rd[f][0] for f in frames]),
        psnr=np.array([rd[f][1] for f in frames]),
        is_wz=np.array([rd[f][2] == "WZ" for f in frames]),
        ld_start=np.array(starts), ld_accepted=np.array(accepted),
        ld_rate=np.array([x["rate"] for x in recs]),
        ld_entropy=np.array([x["entropy"] for x in recs], np.float32),
        **lr_first_frame(recs, q),
    )
    return recs, n


def digest64(a):
    """64-bit digest of an array's bytes (blake2b)."""
    import hashlib
    return int.from_bytes(hashlib.blake2b(np.ascontiguousarray(a).tobytes(), digest_size=8).digest(), "little")


def lr_first_frame(recs, q):
    """The reference's LdpcaDecoder input LRs for the bitplanes of the first
    decoded WZ frame (records are in decode order, QbitsNumPerBlk per frame)."""
    from dvc_b200 import bitstream as bs
    qb = bs.qbits_per_block(q)
    lrs = [recs[i]["LR"] for i in range(min(qb, len(recs)))]
    return dict(lr0_hash=np.array([digest64(x) for x in lrs], np.uint64),
                lr0_head=np.stack(lrs[:LR0_HEAD]).astype(np.float32))


def ldpca_fixture(recs, n, name, limit):
    """Known-answer LDPCA vectors, preferring bitplanes that needed several requests."""
    order = sorted(range(len(recs)), key=lambda i: -recs[i]["rate"])
    pick = sorted(set(order[: limit // 2]) | set(range(0, len(recs), max(1, len(recs) // (limit // 2)))))[:limit]
    lr = np.stack([recs[i]["LR"] for i in pick])
    acc_bits = np.stack([recs[i]["acc"] for i in pick])
    acc_bytes = np.packbits(acc_bits, axis=1, bitorder="big")
    np.savez_compressed(
        os.path.join(HERE, f"ldpca_{name}.npz"), n=n, lr=lr, acc=acc_bytes,
        crc=np.array([recs[i]["crc"] for i in pick], np.uint8),
        entropy=np.array([recs[i]["entropy"] for i in pick], np.float32),
        rate=np.array([recs[i]["rate"] for i in pick], np.int32),
        decoded=np.stack([recs[i]["decoded"] for i in pick]),
        llr=np.stack([recs[i]["LLR"] for i in pick]),
    )


def jbig_fixture(count=240, seed=77):
    """Random and blocky mode maps of both sizes through the reference's JBIG code."""
    import ctypes as C
    enc = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libjbigenc.so"))
    dec = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libjbigdec.so"))
    rng = np.random.default_rng(seed)
    streams, maps, used, sizes = [], [], [], []
    for t in range(count):
        w, h = ((22, 18), (44, 36))[t % 2]
        p = rng.uniform(0.0, 1.0)
        if t % 3 == 0:
            m = np.kron((rng.random(((h + 1) // 2, (w + 1) // 2)) < p).astype(np.uint8),
                        np.ones((2, 2), np.uint8))[:h, :w]
        else:
            m = (rng.random((h, w)) < p).astype(np.uint8)
        m = np.ascontiguousarray(m)
        out = np.zeros(8192, np.uint8)
        n = enc.jbigref_encode(m.ctypes.data_as(C.c_void_p), w, h, out.ctypes.data_as(C.c_void_p), 8192)
        back = np.zeros((h, w), np.uint8)
        u = dec.jbigref_decode(out.ctypes.data_as(C.c_void_p), n, w, h, back.ctypes.data_as(C.c_void_p))
        assert np.array_equal(back, m) and u == n
        streams.append(out[:n].copy())
        maps.append(m.reshape(-1))
        used.append(u)
        sizes.append((w, h))
    off = np.cumsum([0] + [len(x) for x in streams])
    np.savez_compressed(os.path.join(HERE, "jbig_maps.npz"), data=np.concatenate(streams), offsets=off,
                        maps=np.concatenate(maps), map_offsets=np.cumsum([0] + [len(x) for x in maps]),
                        used=np.array(used), sizes=np.array(sizes))


def _ldpcaref(n):
    """The reference's LdpcaDecoder (oracle/_ref/libldpcaref.so) loaded with the ladder of length n."""
    import ctypes as C
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libldpcaref.so"))
    lib.ldpcaref_load.argtypes = [C.c_char_p, C.c_char_p]
    lib.ldpcaref_code_rate.restype = C.c_float
    lib.ldpcaref_compute_ce.restype = C.c_float
    lib.ldpcaref_compute_ce.argtypes = [C.c_void_p]
    lib.ldpcaref_decode.argtypes = [C.c_void_p, C.c_void_p, C.c_ubyte, C.c_float, C.c_void_p]
    d = os.path.join(ROOT, "oracle", "_ref", "LDPCA_LadderFile")
    got = lib.ldpcaref_load(os.path.join(d, "RegDecoder%d.lad" % n).encode(),
                            os.path.join(d, "Inverse_Matrix_H_Reg%d.bin" % n).encode())
    assert got == n, got
    return lib


def _ref_decode_chunk(n, lr, acc_bytes, crc, bounds):
    """Worker: reference decode of codewords; returns (rates, decoded)."""
    lib = _ldpcaref(n)
    rates, dec = [], np.zeros((len(lr), n), np.uint8)
    for i in range(len(lr)):
        l = np.ascontiguousarray(lr[i], np.float32)
        a = np.ascontiguousarray(np.unpackbits(acc_bytes[i], bitorder="big")[:n])
        rates.append(lib.ldpcaref_decode(l.ctypes.data, a.ctypes.data, int(crc[i]), float(bounds[i]),
                                         dec[i].ctypes.data))
    return np.array(rates, np.int32), dec


def ldpca_batch_fixture(pool, count=8192, seed=11):
    """The batched LDPCA workload of dvc_b200.ldpca_bench through the reference,
    codeword by codeword, from each codeword's seeded start level."""
    from dvc_b200 import ldpca_bench as lb
    out = {}
    for n in (1584, 6336):
        c = count // 2
        lr, acc, crc, x = lb.make_codewords(n, c, seed + n)
        starts = lb.seeded_starts(n, c, seed + n)
        rates = lb.code_rates(n)
        bounds = rates[starts]
        step = 64
        futs = [pool.submit(_ref_decode_chunk, n, lr[i:i + step], acc[i:i + step], crc[i:i + step],
                            bounds[i:i + step]) for i in range(0, c, step)]
        res = [f.result() for f in futs]
        rate = np.concatenate([r[0] for r in res])
        dec = np.concatenate([r[1] for r in res])
        synd = [int(round(float(r) * n)) for r in rates]
        out["n%d_start" % n] = starts
        out["n%d_rate" % n] = rate
        out["n%d_accepted" % n] = np.array([synd.index(r - 8) for r in rate], np.int32)
        out["n%d_decoded_hash" % n] = np.array([digest64(d) for d in dec], np.uint64)
        out["n%d_equal_source" % n] = (dec == x).all(axis=1)
        out["n%d_input_hash" % n] = np.array([digest64(lr), digest64(acc), digest64(crc)], np.uint64)
        print("ldpca_batch n=%d: accepted codes %s" % (n, np.bincount(out["n%d_accepted" % n])))
    np.savez_compressed(os.path.join(HERE, "ldpca_batch.npz"), count=count, seed=seed, **out)


def ldpca_fullrate_fixture(pool):
    """Codewords at flip probabilities where every ladder code below full rate
    fails, so the reference ends at its GF(2) inverse (rate N + 8); the start
    code comes from the reference's ComputeCE of the LRs, as in the decoder."""
    from dvc_b200 import encoder
    cases = [(6336, 0.30, 1), (6336, 0.36, 2), (6336, 0.42, 3), (6336, 0.48, 4), (1584, 0.38, 5), (1584, 0.46, 6)]
    lrs, accs, crcs, ents, keys = {}, {}, {}, {}, []
    for n, p, seed in cases:
        rng = np.random.default_rng(1000 + seed)
        x = rng.integers(0, 2, n, dtype=np.uint8)
        y = x ^ (rng.random(n) < p).astype(np.uint8)
        hi, lo = np.float32((1 - np.float32(p)) / np.float32(p)), np.float32(np.float32(p) / (1 - np.float32(p)))
        lr = np.where(y == 0, hi, lo).astype(np.float32)
        L = encoder._ladder(n)
        acc = np.packbits(encoder.accumulated_syndrome(L, x), bitorder="big")
        lib = _ldpcaref(n)
        ent = np.float32(lib.ldpcaref_compute_ce(lr.ctypes.data))
        keys.append((n, lr, acc, encoder.crc8_bits(x), ent, x))
    futs = [pool.submit(_ref_decode_chunk, n, lr[None], acc[None], np.array([crc], np.uint8),
                        np.array([ent], np.float32)) for (n, lr, acc, crc, ent, x) in keys]
    out = {}
    for k, ((n, lr, acc, crc, ent, x), f) in enumerate(zip(keys, futs)):
        rate, dec = f.result()
        assert rate[0] == n + 8, "codeword %d did not reach full rate" % k
        out["c%d_n" % k] = n
        out["c%d_lr" % k] = lr
        out["c%d_acc" % k] = acc
        out["c%d_crc" % k] = np.uint8(crc)
        out["c%d_entropy" % k] = ent
        out["c%d_rate" % k] = rate[0]
        out["c%d_decoded" % k] = dec[0]
        assert np.array_equal(dec[0], x)
    np.savez_compressed(os.path.join(HERE, "ldpca_fullrate.npz"), count=len(keys), **out)


def _bench_gop(enc, g, q, tmp):
    """Worker: the first GOP of the bench's (g, q) stream, encoded by `enc`
    ("ref": the reference encoder, "own": dvc_b200.encoder) and decoded by
    the reference."""
    import hashlib
    import bench
    from dvc_b200 import bitstream as bs
    ori65, key65 = synth.make_sequence(bench.KIND, bench.N_FRAMES, bench.SEED)
    ori, key = ori65[:g + 1], key65[:g + 1]
    h, w = ori.shape[1:]
    d = os.path.join(tmp, "bench_%s_g%d_q%d" % (enc, g, q))
    os.makedirs(d, exist_ok=True)
    oy, ky, st = os.path.join(d, "ori.yuv"), os.path.join(d, "key.yuv"), os.path.join(d, "stat.txt")
    synth.write_yuv420(oy, ori)
    synth.write_yuv420(ky, key)
    synth.write_frame_stat(st, g + 1)
    if enc == "own":
        from dvc_b200 import encoder
        wzb, ib = encoder.encode_sequence_intra(ori, g, q, bench.INTRA_QP, 1, 1, 1)
        wz, intra_bs = os.path.join(d, "s.wz"), os.path.join(d, "s.intra")
        open(wz, "wb").write(wzb)
        open(intra_bs, "wb").write(ib)
    else:
        wz, intra_bs, _ = refrun.encode(oy, ky, g + 1, "CIF", g, q, skip=1, intra=1, intra_qp=bench.INTRA_QP,
                                        deblock=1)
    cap = os.path.join(d, "cap.bin")
    r = refrun.decode(oy, wz, intra_bs, ky, st, mode=0, capture=cap)
    dec_y = np.frombuffer(r["yuv"], np.uint8).reshape(-1, h, w)
    rd = refrun.parse_rd(r["rd"])
    recs = refrun.ldpca_records(refrun.read_capture(cap))
    L = lad.ladder_for(lad.read_compact(os.path.join(ROOT, "dvc_b200", "ladders", "ldpca_ladders.bin")), w * h // 16)
    nc, n, e, period, jc, codes = lad.expand(L)
    synd = [(n // period) * c[0] for c in codes]
    rate_f = np.array(synd, np.float32) / np.float32(n)
    starts = []
    for rec in recs:
        s = 0
        while s < nc - 1 and rate_f[s] < np.float32(rec["entropy"]):
            s += 1
        starts.append(s)
    wz_frames = [f for f in sorted(rd) if rd[f][2] == "WZ"]
    order = [m for (m, _, _) in bs.sequence_order(g + 1, g)]
    return dict(
        wz=open(wz, "rb").read(), intra=open(intra_bs, "rb").read(),
        frames=wz_frames, order=order,
        y_sha=[hashlib.sha256(dec_y[f].tobytes()).hexdigest() for f in wz_frames],
        bits=[rd[f][0] for f in wz_frames], psnr=[rd[f][1] for f in wz_frames],
        start=starts, accepted=[synd.index(x["rate"] - 8) for x in recs],
        entropy=[x["entropy"] for x in recs])


def bench_first_gops_fixture(pool, tmp):
    """The first GOP of every stream of the bench workload, both encoders, decoded by the reference."""
    import bench
    keys = [(enc, g, q) for enc in ("ref", "own") for g in bench.GOPS for q in bench.QS]
    futs = {k: pool.submit(_bench_gop, *k, tmp) for k in keys}
    out = {}
    for (enc, g, q), f in futs.items():
        r = f.result()
        p = "%s_g%d_q%d_" % (enc, g, q)
        if enc == "ref":
            out[p + "wz"] = np.frombuffer(r["wz"], np.uint8)
            out[p + "intra"] = np.frombuffer(r["intra"], np.uint8)
        out[p + "stream_hash"] = np.array([digest64(np.frombuffer(r["wz"], np.uint8)),
                                           digest64(np.frombuffer(r["intra"], np.uint8))], np.uint64)
        out[p + "frames"] = np.array(r["frames"], np.int32)
        out[p + "order"] = np.array(r["order"], np.int32)
        out[p + "y_sha"] = np.array(r["y_sha"])
        out[p + "bits"] = np.array(r["bits"], np.int64)
        out[p + "psnr"] = np.array(r["psnr"], np.float64)
        out[p + "ld_start"] = np.array(r["start"], np.int32)
        out[p + "ld_accepted"] = np.array(r["accepted"], np.int32)
        out[p + "ld_entropy"] = np.array(r["entropy"], np.float32)
        print("bench first GOP %s g%d q%d: %d WZ frames, %d bitplanes" % (enc, g, q, len(r["frames"]),
                                                                         len(r["start"])))
    np.savez_compressed(os.path.join(HERE, "bench_first_gops.npz"), **out)


RANGES = [("qcif_g2_q4_full", 2, 4), ("qcif_g2_q4_full", 0, 2), ("cif_g4_q3_full", 4, 8),
          ("qcif_g2_q4_cfg0", 6, 12)]


def range_fixture(tmp):
    """The reference decoder run with -startFrame/-endFrame on committed
    sequences (main.cpp:118-142: skipGOP replays the intra bitstream of the
    GOPs before the start; frame.cpp:99-103: the decoded luma ends one frame
    before endFrame unless endFrame is the sequence's last frame): its decoded
    luma file and RD report per range."""
    out = {}
    for k, (name, a, b) in enumerate(RANGES):
        g = np.load(os.path.join(HERE, "seq_%s.npz" % name))
        ori, key = synth.make_sequence(str(g["kind"]), int(g["n_frames"]), int(g["seed"]))
        d = os.path.join(tmp, "range%d" % k)
        os.makedirs(d, exist_ok=True)
        oy, ky, st = os.path.join(d, "ori.yuv"), os.path.join(d, "key.yuv"), os.path.join(d, "stat.txt")
        synth.write_yuv420(oy, ori)
        synth.write_yuv420(ky, key)
        synth.write_frame_stat(st, int(g["n_frames"]))
        wz, ib = os.path.join(d, "s.wz"), os.path.join(d, "s.intra")
        g["wz"].tofile(wz)
        g["intra"].tofile(ib)
        r = refrun.decode(oy, wz, ib, ky, st, mode=0, start=a, end=b)
        out["r%d_seq" % k] = name
        out["r%d_start" % k] = a
        out["r%d_end" % k] = b
        out["r%d_yuv" % k] = np.frombuffer(r["yuv"], np.uint8)
        out["r%d_rd" % k] = np.array(r["rd"])
    np.savez_compressed(os.path.join(HERE, "ranges.npz"), count=len(RANGES), **out)


def _sequence_job(name, args, tmp):
    recs, n = run(name, *args[:5], tmp, *args[5:])
    if name == "qcif_g4_q8":
        ldpca_fixture(recs, n, "qcif", 48)
    if name == "cif_g2_q2":
        ldpca_fixture(recs, n, "cif", 11)
    return name, len(recs)


def main():
    import multiprocessing as mp
    import tempfile
    from concurrent.futures import ProcessPoolExecutor
    argv = sys.argv[1:]
    jobs = os.cpu_count() or 4
    if "-j" in argv:
        k = argv.index("-j")
        jobs = int(argv[k + 1])
        argv = argv[:k] + argv[k + 2:]
    tmp = tempfile.mkdtemp(prefix="dvc_golden_")
    want = set(argv)
    with ProcessPoolExecutor(max_workers=jobs, mp_context=mp.get_context("spawn")) as pool:
        if not want or "jbig_maps" in want:
            jbig_fixture()
        futs = [pool.submit(_sequence_job, name, args, tmp) for name, args in SEQUENCES.items()
                if not want or name in want]
        if not want or "bench_first_gops" in want:
            bench_first_gops_fixture(pool, tmp)
        if not want or "ldpca_fullrate" in want:
            ldpca_fullrate_fixture(pool)
        if not want or "ldpca_batch" in want:
            ldpca_batch_fixture(pool)
        if not want or "ranges" in want:
            range_fixture(tmp)
        for f in futs:
            name, nb = f.result()
            print(name, "bitplanes", nb)


if __name__ == "__main__":
    main()
