"""CPU: the package's WZ encoder reproduces the reference encoder's bitstreams."""
import os

import numpy as np
import pytest

from dvc_b200 import encoder, synth


@pytest.mark.parametrize("seq", ["qcif_g2_q4", "qcif_g4_q8", "qcif_g2_q1", "cif_g2_q2"])
def test_encoder_matches_reference_bitstream(golden_dir, seq):
    g = np.load(os.path.join(golden_dir, f"seq_{seq}.npz"))
    ori, _ = synth.make_sequence(str(g["kind"]), int(g["n_frames"]), int(g["seed"]))
    out = encoder.encode_sequence(ori, int(g["gop"]), int(g["qindex"]))
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
