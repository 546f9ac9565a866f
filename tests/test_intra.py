"""Intra blocks (IntraMode 1): the library's host decoder of the intra
bitstream against the reference decoder's output pixels (golden sequences
encoded by the reference with IntraMode 1, DeblockingFilter 0, so the decoded
frames hold the intra blocks exactly as intraRecon wrote them)."""
import os

import numpy as np
import pytest

from dvc_b200 import bitstream as bs
from dvc_b200 import intra, synth


@pytest.mark.parametrize("seq", ["qcif_g2_q4_intra", "cif_g4_q6_intra", "qcif_g4_q8_allintra"])
def test_intra_pixels_match_reference(golden_dir, seq):
    g = np.load(os.path.join(golden_dir, f"seq_{seq}.npz"))
    ori, key = synth.make_sequence(str(g["kind"]), int(g["n_frames"]), int(g["seed"]))
    st = bs.parse_wz(g["wz"].tobytes())
    res = intra.decode_all(st, g["intra"].tobytes(), key)
    assert res, "the sequence has no intra blocks"
    h, w = key.shape[1:]
    total_bits = 0
    for m, (rec, nbits) in res.items():
        fr = st.frames[m]
        blk = np.kron((fr.mode.reshape(h // 8, w // 8) == bs.INTRA_B).astype(np.uint8), np.ones((8, 8), np.uint8)) > 0
        assert blk.any()
        assert np.array_equal(rec[blk], g["dec_y"][m][blk]), f"frame {m}"
        assert np.array_equal(rec[~blk], key[m][~blk])  # other pixels untouched
        total_bits += nbits
    # the frames' blocks use the whole intra bitstream (up to the final byte's padding)
    assert len(g["intra"]) * 8 - 8 < total_bits <= len(g["intra"]) * 8


def test_truncated_intra_bitstream_is_refused(golden_dir):
    g = np.load(os.path.join(golden_dir, "seq_qcif_g2_q4_intra.npz"))
    st = bs.parse_wz(g["wz"].tobytes())
    with pytest.raises(ValueError):
        intra.decode_all(st, g["intra"].tobytes()[: len(g["intra"]) // 3])
