"""The WZ bitstream parser (dvc_b200.bitstream) on damaged input: every
truncation and every bad header field raises ValueError."""
import os

import numpy as np
import pytest

from dvc_b200 import bitstream as bs


@pytest.mark.parametrize("seq", ["qcif_still_g4_q4_full", "cif_g4_q6_full"])
def test_damaged_wz_bitstreams_raise_value_error(golden_dir, seq):
    wz = np.load(os.path.join(golden_dir, f"seq_{seq}.npz"))["wz"].tobytes()
    st = bs.parse_wz(wz)
    assert st.frames
    cuts = sorted(set(list(range(0, 64)) + list(range(64, len(wz), 37))))
    for n in cuts:
        with pytest.raises(ValueError):
            bs.parse_wz(wz[:n])
    for data in (bytes([7]) + wz[1:], wz[:1] + bytes([0]) + wz[2:], wz[:1] + bytes([9]) + wz[2:]):
        with pytest.raises(ValueError):
            bs.parse_wz(data)
