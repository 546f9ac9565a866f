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
                                 "qcif_g4_q6_db"])
def test_oracle_sequence_matches_reference(golden_dir, seq):
    g = load(golden_dir, f"seq_{seq}.npz")
    kind = str(g["kind"])
    ori, key = synth.make_sequence(kind, int(g["n_frames"]), int(g["seed"]))
    st = bs.parse_wz(g["wz"].tobytes())
    kb = {f: 4000 for f in range(st.n_frames)}
    kp = {f: 40.0 for f in range(st.n_frames)}
    res = po.decode_sequence(st, key, ori, kb, kp)
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
