"""CPU tests: the C restatement oracle against the reference's golden vectors."""
import os

import numpy as np
import pytest

from dvc_b200 import bitstream as bs
from dvc_b200 import synth
from oracle import pyoracle as po


def load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name), allow_pickle=False)


@pytest.mark.parametrize("name", ["qcif", "cif"])
def test_oracle_ldpca_matches_reference(golden_dir, name):
    g = load(golden_dir, f"ldpca_{name}.npz")
    n = int(g["n"])
    L = po.OracleLadder.get(n)
    for i in range(len(g["crc"])):
        lr = g["lr"][i]
        ent = po.compute_ce(lr)
        assert np.float32(ent) == g["entropy"][i]
        acc_bits = np.unpackbits(g["acc"][i], bitorder="big")[:n]
        dec, rate, start, acc_code, llr = po.ldpca_decode(L, lr, acc_bits, int(g["crc"][i]), ent)
        assert rate == g["rate"][i]
        assert np.array_equal(dec, g["decoded"][i])
        assert np.array_equal(llr.view(np.uint32), g["llr"][i].view(np.uint32))


def test_crc_and_accumulated_syndrome_round_trip():
    L = po.OracleLadder.get(1584)
    rng = np.random.default_rng(5)
    src = rng.integers(0, 2, 1584, dtype=np.uint8)
    acc = po.accumulated_syndrome(L, src)
    crc = po.crc8_bits(src)
    # a near-perfect LR ratio towards the source decodes at the first code
    lr = np.where(src == 0, np.float32(0.9999 / 0.0001), np.float32(0.0001 / 0.9999)).astype(np.float32)
    dec, rate, start, acc_code, _ = po.ldpca_decode(L, lr, acc, crc, 0.0)
    assert np.array_equal(dec, src)
    assert acc_code == 0 and start == 0


@pytest.mark.parametrize("seq", ["qcif_g2_q4", "qcif_g4_q8", "qcif_g2_q1", "qcif_still_g2_q4_skip", "qcif_g2_q4_db",
                                 "qcif_g4_q6_db", "qcif_g2_q4_intra", "qcif_g4_q8_allintra", "qcif_g2_q4_full",
                                 "qcif_still_g4_q4_full", "qcif_g2_q8_own_full", "qcif_still_g4_q4_own_full"])
def test_oracle_sequence_matches_reference(golden_dir, seq):
    """Whole sequences through the oracle against the reference decoder's
    output: pixels, rates, PSNR and every bitplane's first and accepted code;
    the intra, skip and deblocking fixtures carry the sequence's intra bit
    string, which the oracle's own CAVLC decoder reads."""
    g = load(golden_dir, f"seq_{seq}.npz")
    kind = str(g["kind"])
    ori, key = synth.make_sequence(kind, int(g["n_frames"]), int(g["seed"]))
    st = bs.parse_wz(g["wz"].tobytes())
    kb = {f: 4000 for f in range(st.n_frames)}
    kp = {f: 40.0 for f in range(st.n_frames)}
    intra_bs = g["intra"].tobytes() if "intra" in g.files else None
    res = po.decode_sequence(st, key, ori, kb, kp, intra_bitstream=intra_bs)
    assert np.array_equal(res["recon"], g["dec_y"])
    for f, b, p, wz in zip(g["frames"], g["bits"], g["psnr"], g["is_wz"]):
        if wz:
            assert res["bits"][int(f)] == b
            assert "%.2f" % res["psnr"][int(f)] == "%.2f" % p
    starts = np.concatenate([res["planes"][m][0] for (m, _, _) in bs.sequence_order(st.n_frames, st.gop)])
    accepted = np.concatenate([res["planes"][m][1] for (m, _, _) in bs.sequence_order(st.n_frames, st.gop)])
    assert np.array_equal(starts, g["ld_start"])
    assert np.array_equal(accepted, g["ld_accepted"])


@pytest.mark.skipif(not __import__("oracle.refrun", fromlist=["ref_available"]).ref_available(),
                    reason="reference build absent")
@pytest.mark.parametrize("seq", ["qcif_g2_q4_full", "qcif_still_g4_q4_full"])
def test_oracle_deblocking_matches_reference_filter(golden_dir, seq, tmp_path):
    """The oracle's deblocking filter against the reference's own, frame by
    frame: the reference capture decoder records the filter's inputs (frame,
    change flags, block modes, past reference) and its output."""
    import struct
    from oracle import refrun
    g = load(golden_dir, f"seq_{seq}.npz")
    ori, key = synth.make_sequence(str(g["kind"]), int(g["n_frames"]), int(g["seed"]))
    st = bs.parse_wz(g["wz"].tobytes())
    oy, ky, sf = str(tmp_path / "o.yuv"), str(tmp_path / "k.yuv"), str(tmp_path / "s.txt")
    wz, ib = str(tmp_path / "s.wz"), str(tmp_path / "s.intra")
    synth.write_yuv420(oy, ori)
    synth.write_yuv420(ky, key)
    synth.write_frame_stat(sf, int(g["n_frames"]))
    open(wz, "wb").write(g["wz"].tobytes())
    open(ib, "wb").write(g["intra"].tobytes())
    cap = str(tmp_path / "cap.bin")
    refrun.decode(oy, wz, ib, ky, sf, mode=0, capture=cap)
    recs = refrun.read_capture(cap)
    h, w = st.height, st.width
    checked = 0
    cur = {}
    for tag, b in recs:
        if tag in ("DBIN", "DBFG", "DBMD"):
            cur[tag] = np.frombuffer(b, np.uint8)
        elif tag == "DBBG":
            (cur["begin"],) = struct.unpack("<i", b)
        elif tag == "DBOU":
            begin = cur["begin"]
            past = st.frames.get(begin)
            out = po.deblock(cur["DBIN"].reshape(h, w), cur["DBFG"], cur["DBMD"],
                             None if past is None else past.mode, st.qindex, st.intra_qp)
            assert np.array_equal(out.reshape(-1), np.frombuffer(b, np.uint8)), f"frame {checked}"
            checked += 1
            cur = {}
    assert checked == len(st.frames)


class _Geom:
    def __init__(self, **kw):
        self.__dict__.update(kw)


@pytest.mark.parametrize("size", [(144, 176), (288, 352)])
@pytest.mark.parametrize("qp", [0, 12, 30, 51])
@pytest.mark.parametrize("content", ["noise", "ramp", "half_intra"])
def test_oracle_intra_reads_encoder_blocks(qp, content, size):
    """The oracle's CAVLC reader on intra blocks written by the library's
    encoder (dvc_intra_encode_frame): every bit consumed and every intra pixel
    equal to the reconstruction the encoder reports, and the library's host
    decoder (dvc_intra_decode_frame) equal to the oracle.  IntraQP 0 on noise takes
    the level_prefix 15 escape (about 4,500 times in the frame) and the 6-bit
    coeff_token of nC >= 8 (about 1,600 blocks); IntraQP 51 leaves mostly empty
    blocks."""
    from dvc_b200 import intra
    rng = np.random.default_rng(qp * 7 + len(content) + size[0])
    h, w = size
    if content == "noise":
        ori = rng.integers(0, 256, (h, w), dtype=np.uint8)
    else:
        ori = np.clip(128 + np.cumsum(rng.integers(-9, 10, (h, w)), axis=1), 0, 255).astype(np.uint8)
    mode = np.ones((h // 8, w // 8), np.uint8) if content != "half_intra" else \
        (rng.random((h // 8, w // 8)) < 0.5).astype(np.uint8)
    buf = np.zeros(1 << 20, np.uint8)
    end, rec = intra.encode_frame(ori, mode, qp, buf, 5)  # a string that starts mid-byte
    data = buf[:(end + 7) // 8].copy()
    out = np.zeros((h, w), np.uint8)
    geom = _Geom(width=w, height=h, intra_qp=qp)
    fr = _Geom(mode=mode.reshape(-1), idx=1)
    assert po.intra_decode_frame(geom, fr, data, 5, out) == end
    px = np.kron(mode, np.ones((8, 8), np.uint8)).astype(bool)
    assert np.array_equal(out[px], rec[px])
    assert not out[~px].any()  # pixels of other blocks are left alone
    # the library's own host decoder reads the same string to the same pixels and end
    import ctypes as C
    from dvc_b200 import native
    lib_out = np.zeros((h, w), np.uint8)
    off = C.c_size_t(5)
    assert native.lib().dvc_intra_decode_frame(data.ctypes.data_as(C.c_void_p), data.size, C.byref(off), w, h, qp,
                                               fr.mode.ctypes.data_as(C.c_void_p),
                                               lib_out.ctypes.data_as(C.c_void_p)) == native.DVC_OK
    assert off.value == end and np.array_equal(lib_out, out)
    with pytest.raises(RuntimeError):  # a string cut short inside the last block
        po.intra_decode_frame(geom, fr, data[:max(1, (end - 40) // 8)], 5, np.zeros((h, w), np.uint8))


def test_oracle_cif_intra_deblocked_frame_matches_reference(golden_dir):
    """CIF geometry through the oracle's intra, WZ and deblocking paths: the
    first decoded frame of a CIF GOP-4 sequence with SkipBlock, IntraMode and
    DeblockingFilter on (302 intra 8x8 blocks), against the reference decoder."""
    g = load(golden_dir, "seq_cif_g4_q6_full.npz")
    ori, key = synth.make_sequence(str(g["kind"]), int(g["n_frames"]), int(g["seed"]))
    st = bs.parse_wz(g["wz"].tobytes())
    m = bs.sequence_order(st.n_frames, st.gop)[0][0]
    assert (st.frames[m].mode == 1).sum() > 0 and st.deblock
    res = po.decode_sequence(st, key, ori, {}, {}, frames={m}, intra_bitstream=g["intra"].tobytes())
    assert np.array_equal(res["recon"][m], g["dec_y"][m])
    k = list(g["frames"]).index(m)
    assert res["bits"][m] == g["bits"][k]
    assert "%.2f" % res["psnr"][m] == "%.2f" % g["psnr"][k]
    qb = len(res["planes"][m][0])
    assert np.array_equal(res["planes"][m][0], g["ld_start"][:qb])
    assert np.array_equal(res["planes"][m][1], g["ld_accepted"][:qb])


def test_oracle_config0_sequence_matches_reference(golden_dir):
    """The reference's plain CPU run (QCIF, 17 frames, GOP 2, QIndex 4, every
    option off) through the oracle: pixels, rates, PSNR and ladder codes."""
    test_oracle_sequence_matches_reference(golden_dir, "qcif_g2_q4_cfg0")


@pytest.mark.parametrize("k", [4, 5])
def test_oracle_full_rate_matches_reference(golden_dir, k):
    """QCIF codewords that only the GF(2) inverse decodes: the oracle's ladder
    walks every code to full rate as the reference's did."""
    g = load(golden_dir, "ldpca_fullrate.npz")
    n = int(g["c%d_n" % k])
    L = po.OracleLadder.get(n)
    lr = g["c%d_lr" % k]
    ent = po.compute_ce(lr)
    assert np.float32(ent) == g["c%d_entropy" % k]
    acc_bits = np.unpackbits(g["c%d_acc" % k], bitorder="big")[:n]
    dec, rate, start, acc_code, _ = po.ldpca_decode(L, lr, acc_bits, int(g["c%d_crc" % k]), ent)
    assert rate == int(g["c%d_rate" % k]) == n + 8 and acc_code == 64
    assert np.array_equal(dec, g["c%d_decoded" % k])


def _digest64(a):
    import hashlib
    return int.from_bytes(hashlib.blake2b(np.ascontiguousarray(a).tobytes(), digest_size=8).digest(), "little")


@pytest.mark.parametrize("n,count", [(1584, 24), (6336, 6)])
def test_oracle_batch_codewords_match_reference(golden_dir, n, count):
    """The first codewords of the batched LDPCA workload (dvc_b200.ldpca_bench:
    seeded sources, flip probabilities and start levels): the generator
    reproduces the inputs the reference decoded, and the oracle started at each
    codeword's seeded level reaches the reference's rate and decoded bits."""
    from dvc_b200 import ldpca_bench as lb
    g = load(golden_dir, "ldpca_batch.npz")
    half = int(g["count"]) // 2
    seed = int(g["seed"]) + n
    lr, acc, crc, x = lb.make_codewords(n, half, seed)
    assert [_digest64(lr), _digest64(acc), _digest64(crc)] == [int(v) for v in g["n%d_input_hash" % n]]
    starts = lb.seeded_starts(n, half, seed)
    assert np.array_equal(starts, g["n%d_start" % n])
    rates = lb.code_rates(n)
    L = po.OracleLadder.get(n)
    for i in range(count):
        bits = np.unpackbits(acc[i], bitorder="big")[:n]
        dec, rate, start, acc_code, _ = po.ldpca_decode(L, lr[i], bits, int(crc[i]), float(rates[starts[i]]))
        assert start == starts[i]
        assert rate == g["n%d_rate" % n][i]
        assert _digest64(dec) == int(g["n%d_decoded_hash" % n][i])
