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

Usage (in the build container, after `make -C oracle ref` and
`python oracle/ladder_dir.py oracle/_ref`):
    python tests/golden/make_golden.py [fixture names]   # default: all
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "dvc_b200", "ladders"))

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
}


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
    )
    return recs, n


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


def main():
    import tempfile
    tmp = tempfile.mkdtemp(prefix="dvc_golden_")
    want = set(sys.argv[1:])
    if not want or "jbig_maps" in want:
        jbig_fixture()
    for name, args in SEQUENCES.items():
        if want and name not in want:
            continue
        recs, n = run(name, *args[:5], tmp, *args[5:])
        print(name, "bitplanes", len(recs))
        if name == "qcif_g4_q8":
            ldpca_fixture(recs, n, "qcif", 48)
        if name == "cif_g2_q2":
            ldpca_fixture(recs, n, "cif", 11)


if __name__ == "__main__":
    main()
