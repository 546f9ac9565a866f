"""GPU parity: whole WZ frames decoded on the device against the reference decoder."""
import os

import numpy as np
import pytest

from dvc_b200 import bitstream as bs
from dvc_b200 import decoder, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seq", ["qcif_g2_q4", "qcif_g4_q8", "qcif_g2_q1", "cif_g2_q2", "qcif_still_g2_q4_skip",
                                 "cif_still_g4_q6_skip", "qcif_g2_q4_intra", "cif_g4_q6_intra",
                                 "qcif_g4_q8_allintra", "qcif_g2_q4_full", "cif_g4_q6_full",
                                 "qcif_still_g4_q4_full", "cif_g4_q4_own_full", "qcif_g2_q8_own_full",
                                 "qcif_still_g4_q4_own_full", "cif_fast_g8_q8_own_full",
                                 "cif_fast_g8_q4_own_full", "qcif_g2_q4_db", "qcif_g4_q6_db",
                                 "cif_g2_q1_full", "cif_g4_q3_full", "cif_g2_q5_full", "cif_g4_q7_full",
                                 "cif_g4_q8_full", "cif_g2_q8_wz", "qcif_g2_q4_cfg0"])
def test_sequence_matches_reference(gpu_ctx, golden_dir, seq):
    """Every WZ frame of a reference-decoded sequence: decoded Y, bits and PSNR,
    and per bitplane the first and accepted ladder codes and the bits of the
    conditional-entropy bound; no reconstruction step may sit near a rounding
    tie that the C library's exp and the device's could resolve differently."""
    g = np.load(os.path.join(golden_dir, f"seq_{seq}.npz"))
    ori, key = synth.make_sequence(str(g["kind"]), int(g["n_frames"]), int(g["seed"]))
    st = bs.parse_wz(g["wz"].tobytes())
    intra_bs = g["intra"].tobytes() if "intra" in g.files else None
    ties0 = gpu_ctx.recon_near_ties()
    res = decoder.decode_sequence(gpu_ctx, st, key, ori, intra_bitstream=intra_bs)
    assert gpu_ctx.recon_near_ties() == ties0, "a reconstruction step sat near a rounding tie"
    for f, b, p, wz in zip(g["frames"], g["bits"], g["psnr"], g["is_wz"]):
        if wz:
            f = int(f)
            assert np.array_equal(res["recon"][f], g["dec_y"][f]), f"frame {f} Y differs"
            assert res["bits"][f] == b
            assert "%.2f" % res["psnr"][f] == "%.2f" % p
    order = bs.sequence_order(st.n_frames, st.gop)
    start = np.concatenate([res["planes"][m][:, 1] for (m, _, _) in order])
    acc = np.concatenate([res["planes"][m][:, 2] for (m, _, _) in order])
    assert np.array_equal(start, g["ld_start"])
    assert np.array_equal(acc, g["ld_accepted"])
    ent = np.concatenate([res["entropy"][m] for (m, _, _) in order]).astype(np.float32)
    assert np.array_equal(ent.view(np.uint32), g["ld_entropy"].astype(np.float32).view(np.uint32)), \
        "conditional-entropy bounds differ"


def _digest64(a):
    import hashlib
    return int.from_bytes(hashlib.blake2b(np.ascontiguousarray(a).tobytes(), digest_size=8).digest(), "little")


@pytest.mark.parametrize("seq", ["qcif_g2_q4", "cif_g2_q2", "qcif_g2_q4_full", "cif_g2_q5_full", "cif_g2_q8_wz",
                                 "cif_g4_q7_full", "qcif_g2_q4_cfg0"])
def test_first_frame_likelihood_ratios_match_reference(gpu_ctx, golden_dir, seq):
    """The likelihood ratios of every bitplane of the first decoded WZ frame
    (condBitProb's output, the LDPCA decoder's input) against the ones the
    reference passed to its LdpcaDecoder: bit for bit (a digest per bitplane;
    the first bitplanes are stored in full and also checked to 1e-6 relative,
    so that a failure shows the size of the difference)."""
    from dvc_b200 import intra
    g = np.load(os.path.join(golden_dir, f"seq_{seq}.npz"))
    ori, key = synth.make_sequence(str(g["kind"]), int(g["n_frames"]), int(g["seed"]))
    st = bs.parse_wz(g["wz"].tobytes())
    m, b, e = bs.sequence_order(st.n_frames, st.gop)[0]
    recon = np.array(key, np.uint8, copy=True)
    if st.frames[m].intra_mode:
        recon[m] = intra.decode_all(st, g["intra"].tobytes(), recon)[m][0]
    out = gpu_ctx.debug_wz_frame_lr(decoder.frame_item(st, st.frames[m], recon))
    lr = out["lr"]
    head = g["lr0_head"]
    assert lr.shape[0] == len(g["lr0_hash"])
    rel = np.abs(lr[:len(head)].astype(np.float64) - head) / np.maximum(np.abs(head.astype(np.float64)), 1e-30)
    assert rel.max() <= 1e-6, "likelihood ratio off by %g relative" % rel.max()
    assert np.array_equal(lr[:len(head)].view(np.uint32), head.view(np.uint32)), "likelihood ratios differ in bits"
    got = np.array([_digest64(x) for x in lr], np.uint64)
    bad = np.nonzero(got != g["lr0_hash"])[0]
    assert len(bad) == 0, "likelihood ratios of bitplanes %s differ" % bad.tolist()


@pytest.mark.parametrize("seq", ["qcif_g2_q4", "cif_g2_q2"])
def test_first_frame_stages_match_oracle(gpu_ctx, golden_dir, seq):
    """Stage-level check of the first WZ frame against the C oracle: side information,
    noise parameters, refined side information and the decoded frame."""
    from oracle import pyoracle as po
    g = np.load(os.path.join(golden_dir, f"seq_{seq}.npz"))
    ori, key = synth.make_sequence(str(g["kind"]), int(g["n_frames"]), int(g["seed"]))
    st = bs.parse_wz(g["wz"].tobytes())
    m, b, e = bs.sequence_order(st.n_frames, st.gop)[0]
    fr = st.frames[m]
    ref = po.decode_frame(st, fr, key[b], key[e], want=("alpha", "si"))
    out = gpu_ctx.debug_wz_frame(decoder.frame_item(st, fr, key))
    assert np.array_equal(out["si_initial"], ref["si_initial"]), "initial side information"
    assert np.array_equal(out["alpha"].view(np.uint32), ref["alpha"].view(np.uint32)), "alpha"
    assert np.array_equal(out["planes"][:, 2], ref["accepted"]), "accepted codes"
    assert np.array_equal(out["si_final"], ref["si_final"]), "refined side information"
    assert np.array_equal(out["recon"], ref["recon"]), "decoded frame"


@pytest.mark.parametrize("seq", ["qcif_g4_q8"])
def test_session_levels_match_reference(gpu_ctx, golden_dir, seq):
    """A GOP-4 sequence as one device-resident session: frames 1 and 3 of each GOP
    name frame 2's decoded output as their reference (past_from / future_from),
    so the second level starts on the device without a host round trip; run
    three times: the first run is eager, the later ones replay the run captured
    as a CUDA graph, and a profiled run is eager again."""
    g = np.load(os.path.join(golden_dir, f"seq_{seq}.npz"))
    ori, key = synth.make_sequence(str(g["kind"]), int(g["n_frames"]), int(g["seed"]))
    st = bs.parse_wz(g["wz"].tobytes())
    items, where = [], {}
    for lvl in decoder.decode_levels(st):
        for (m, b, e) in lvl:
            it = decoder.frame_item(st, st.frames[m], key)
            for name, ref in (("past", b), ("future", e)):
                if ref in st.frames:
                    it[name + "_from"], it[name] = where[ref], None
            where[m] = len(items)
            items.append(it)
    assert any(it.get("past_from") is not None or it.get("future_from") is not None for it in items)
    ses = gpu_ctx.session(items, max_batch=3, streams=2)
    try:
        for r in range(4):
            ses.run(profile=(r == 3))
            for m, i in where.items():
                rec, bits, planes = ses.frame(i)
                assert np.array_equal(rec, g["dec_y"][m]), f"frame {m} Y differs"
                k = list(g["frames"]).index(m)
                assert bits == g["bits"][k] - st.frames[m].skip_bits - st.frames[m].intra_map_bits
        assert ses.replays() == 2  # runs 2 and 3 replayed the graph, the profiled run 4 did not
    finally:
        ses.close()
