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


def _decode_raw(data, off, w, h, qp, mode, rec):
    import ctypes as C
    from dvc_b200 import native
    o = C.c_size_t(off)
    vp = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)  # noqa: E731
    rc = native.lib().dvc_intra_decode_frame(vp(data), 0 if data is None else data.size, C.byref(o), w, h, qp,
                                            vp(mode), vp(rec))
    return rc, o.value


def test_intra_decoder_refuses_bad_arguments():
    from dvc_b200 import native
    data = np.full(64, 0x80, np.uint8)
    mode = np.zeros(396, np.uint8)
    rec = np.zeros((144, 176), np.uint8)
    assert _decode_raw(data, 0, 176, 144, 30, mode, rec)[0] == native.DVC_OK  # no intra block: nothing read
    for args in ((data, 0, 176, 144, 52, mode, rec), (data, 0, 176, 144, -1, mode, rec),
                 (data, 0, 160, 144, 30, mode, rec), (data, 0, 176, 144, 30, None, rec),
                 (data, 0, 176, 144, 30, mode, None), (None, 0, 176, 144, 30, mode, rec)):
        assert _decode_raw(*args)[0] == native.DVC_E_ARG


def test_intra_decoder_on_arbitrary_bytes_stays_in_bounds():
    """Random bit strings under random intra maps: each call either decodes,
    with the offset inside the string, or reports a data error; strings cut at
    every byte of a real frame's blocks are refused, never read past."""
    from dvc_b200 import native
    rng = np.random.default_rng(9)
    for t in range(300):
        w, h = (176, 144) if t % 2 else (352, 288)
        n = int(rng.integers(1, 400))
        data = rng.integers(0, 256, n, dtype=np.uint8) if t % 3 else np.zeros(n, np.uint8)
        mode = (rng.random((h // 8) * (w // 8)) < rng.random()).astype(np.uint8)
        rec = np.zeros((h, w), np.uint8)
        rc, end = _decode_raw(data, int(rng.integers(0, 8)), w, h, int(rng.integers(0, 52)), mode, rec)
        assert rc in (native.DVC_OK, native.DVC_E_DATA)
        if rc == native.DVC_OK:
            assert end <= 8 * n
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "seq_qcif_g2_q4_intra.npz"))
    st = bs.parse_wz(g["wz"].tobytes())
    m = [m for (m, b, e) in bs.sequence_order(st.n_frames, st.gop) if st.frames[m].intra_mode][0]
    mode = np.ascontiguousarray(st.frames[m].mode, np.uint8)
    full = g["intra"]
    rc, end = _decode_raw(full, 0, st.width, st.height, st.intra_qp, mode, np.zeros((st.height, st.width), np.uint8))
    assert rc == native.DVC_OK
    for cut in range(0, (end + 7) // 8 - 1):
        part = np.ascontiguousarray(full[:cut])
        rc, _ = _decode_raw(part if cut else np.zeros(0, np.uint8), 0, st.width, st.height, st.intra_qp, mode,
                            np.zeros((st.height, st.width), np.uint8))
        assert rc == native.DVC_E_DATA, cut
