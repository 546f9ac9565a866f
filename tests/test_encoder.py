"""CPU: the package's WZ encoder reproduces the reference encoder's bitstreams."""
import ctypes as C
import os

import numpy as np
import pytest

from dvc_b200 import encoder, synth


@pytest.mark.parametrize("seq", ["qcif_g2_q4", "qcif_g4_q8", "qcif_g2_q1", "cif_g2_q2", "qcif_still_g2_q4_skip",
                                 "cif_still_g4_q6_skip"])
def test_encoder_matches_reference_bitstream(golden_dir, seq):
    g = np.load(os.path.join(golden_dir, f"seq_{seq}.npz"))
    ori, _ = synth.make_sequence(str(g["kind"]), int(g["n_frames"]), int(g["seed"]))
    skip = int(g["skip"]) if "skip" in g else 0
    out = encoder.encode_sequence(ori, int(g["gop"]), int(g["qindex"]), skip=skip)
    assert out == g["wz"].tobytes()


def test_skip_test_matches_reference_maps(golden_dir):
    """The encoder's skip test marks exactly the blocks of the reference's skip maps."""
    from dvc_b200 import bitstream as bs
    for seq in ("qcif_still_g2_q4_skip", "cif_still_g4_q6_skip"):
        g = np.load(os.path.join(golden_dir, f"seq_{seq}.npz"))
        ori, _ = synth.make_sequence(str(g["kind"]), int(g["n_frames"]), int(g["seed"]))
        st = bs.parse_wz(g["wz"].tobytes())
        for m, fr in st.frames.items():
            assert fr.skip_mode == 1
            got = encoder.skip_blocks(ori[m], ori[fr.past]).reshape(-1)
            assert np.array_equal(got, fr.mode == bs.SKIP_B)


@pytest.mark.skipif(not __import__("oracle.refrun", fromlist=["ref_available"]).ref_available(),
                    reason="reference build absent")
def test_skip_and_deblock_options_match_reference_encoder(tmp_path):
    """SkipBlock 1 on content where no block passes the skip test, and the
    deblocking header flag: byte-identical to the reference encoder's output."""
    from oracle import refrun
    ori, key = synth.make_sequence("cif", 5, 101)
    oy, ky = str(tmp_path / "o.yuv"), str(tmp_path / "k.yuv")
    synth.write_yuv420(oy, ori)
    synth.write_yuv420(ky, key)
    for gop, q in ((2, 3), (4, 7)):
        wz, _, _ = refrun.encode(oy, ky, 5, "CIF", gop, q, skip=1, intra=0, deblock=1)
        assert encoder.encode_sequence(ori, gop, q, deblock=1, skip=1) == open(wz, "rb").read()


@pytest.mark.parametrize("seq", ["cif_g4_q4_own_full", "qcif_g2_q8_own_full", "qcif_still_g4_q4_own_full",
                                 "cif_fast_g8_q4_own_full"])
def test_own_intra_streams_are_reproduced(golden_dir, seq):
    """Streams with this encoder's skip and intra decisions (decoded by the
    reference decoder into the fixture) come out the same again."""
    from dvc_b200 import bitstream as bs
    g = np.load(os.path.join(golden_dir, f"seq_{seq}.npz"))
    ori, _ = synth.make_sequence(str(g["kind"]), int(g["n_frames"]), int(g["seed"]))
    st = bs.parse_wz(g["wz"].tobytes())
    wz, ib = encoder.encode_sequence_intra(ori, int(g["gop"]), int(g["qindex"]), st.intra_qp, st.deblock, 1, 1)
    assert wz == g["wz"].tobytes() and ib == g["intra"].tobytes()
    assert any((fr.mode == 1).any() for fr in st.frames.values())


def test_intra_coder_round_trip():
    """The intra coder's reconstruction is what the decoder reads back, bit for
    bit, and it consumes exactly the bits written, on random modes and QPs."""
    from dvc_b200 import intra
    rng = np.random.default_rng(9)
    ori, _ = synth.make_sequence("cif", 2, 3)
    for qp in (4, 20, 30, 45):
        mode = (rng.random((36, 44)) < 0.5).astype(np.uint8)
        buf = np.zeros(352 * 288 * 2, np.uint8)
        end, rec = intra.encode_frame(ori[1], mode, qp, buf, 5)
        off = C.c_size_t(5)
        back = np.zeros((288, 352), np.uint8)
        from dvc_b200 import native
        rc = native.lib().dvc_intra_decode_frame(buf.ctypes.data_as(C.c_void_p), len(buf), C.byref(off), 352, 288,
                                                qp, mode.ctypes.data_as(C.c_void_p), back.ctypes.data_as(C.c_void_p))
        assert rc == 0 and off.value == end and np.array_equal(back, rec)
        m = np.kron(mode.astype(bool), np.ones((8, 8), bool))
        err = np.abs(rec.astype(int) - ori[1].astype(int))[m].mean()
        assert err < 2.0 + qp / 3.0, (qp, err)  # a working quantiser, not only a valid syntax


def test_intra_choice_follows_the_rate_comparison():
    """The intra share grows with QIndex as the WZ rate estimate grows: none of
    the 8x8 blocks of the moving CIF content at Q2, most of them at Q8; skip
    blocks are never intra."""
    ori, _ = synth.make_sequence("cif", 3, 101)
    share = {}
    for q in (2, 8):
        it, coded = encoder.intra_decision(ori[1], ori[0], ori[2], None, q)
        share[q] = float(it.mean())
        assert (coded is None) == (not it.any())
    assert share[2] == 0.0 and share[8] > 0.5
    skip = np.zeros((36, 44), bool)
    skip[::2] = True
    it, _ = encoder.intra_decision(ori[1], ori[0], ori[2], skip, 8)
    assert not (it & skip).any()
