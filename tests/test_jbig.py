"""JBIG mode maps: the library's T.82 decoder against maps coded and decoded by
the reference's own JBIG code (committed fixtures; fresh random maps as well
when oracle/_ref holds the reference build)."""
import ctypes as C
import os

import numpy as np
import pytest

from dvc_b200 import jbig

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


def test_fixture_maps_decode_exactly(golden_dir):
    g = np.load(os.path.join(golden_dir, "jbig_maps.npz"))
    off, moff = g["offsets"], g["map_offsets"]
    for i, (w, h) in enumerate(g["sizes"]):
        data = g["data"][off[i]:off[i + 1]].tobytes()
        # the reader sees the rest of the bitstream after the map
        m, used = jbig.decode_mode_map(data + bytes(range(37)), int(w), int(h))
        assert used == g["used"][i]
        assert np.array_equal(m.reshape(-1), g["maps"][moff[i]:moff[i + 1]])


def test_truncated_and_unsupported_streams_are_refused(golden_dir):
    g = np.load(os.path.join(golden_dir, "jbig_maps.npz"))
    data = g["data"][g["offsets"][0]:g["offsets"][1]].tobytes()
    w, h = (int(x) for x in g["sizes"][0])
    with pytest.raises(ValueError):
        jbig.decode_mode_map(data[:-2], w, h)  # closing marker missing
    with pytest.raises(ValueError):
        jbig.decode_mode_map(b"\xff\x06" + bytes(6) + data, w, h)  # adaptive-template move


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "libjbigenc.so")), reason="reference JBIG build absent")
def test_fresh_maps_against_reference_codec():
    enc = C.CDLL(os.path.join(REF, "libjbigenc.so"))
    rng = np.random.default_rng(2024)
    for t in range(300):
        w, h = ((22, 18), (44, 36))[t % 2]
        m = np.ascontiguousarray((rng.random((h, w)) < rng.uniform(0, 1)).astype(np.uint8))
        out = np.zeros(8192, np.uint8)
        n = enc.jbigref_encode(m.ctypes.data_as(C.c_void_p), w, h, out.ctypes.data_as(C.c_void_p), 8192)
        got, used = jbig.decode_mode_map(out[:n].tobytes(), w, h)
        assert used == n and np.array_equal(got, m)
        # the library's encoder writes the reference encoder's bytes
        assert jbig.encode_mode_map(m) == out[:n].tobytes()


def test_encoder_writes_the_fixture_bytes(golden_dir):
    g = np.load(os.path.join(golden_dir, "jbig_maps.npz"))
    for i in range(len(g["used"])):
        w, h = (int(v) for v in g["sizes"][i])
        m = g["maps"][g["map_offsets"][i]:g["map_offsets"][i + 1]].reshape(h, w)
        data = g["data"][g["offsets"][i]:g["offsets"][i + 1]].tobytes()
        assert jbig.encode_mode_map(m) == data, i
    # all-zero, all-one and single-pixel maps round-trip through the decoder
    for m in (np.zeros((36, 44), np.uint8), np.ones((18, 22), np.uint8), np.eye(18, 22, dtype=np.uint8)):
        got, used = jbig.decode_mode_map(jbig.encode_mode_map(m) + bytes(5), m.shape[1], m.shape[0])
        assert np.array_equal(got, m) and used == len(jbig.encode_mode_map(m))
