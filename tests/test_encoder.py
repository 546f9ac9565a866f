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
