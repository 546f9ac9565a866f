"""GPU: the reference's own DvcDec with its ParallelMode 2 WZ decode bound to
this library (oracle/dvcdec_binding.cpp, built by oracle/Makefile into
oracle/_ref/DvcDec_b200): the reference's main, configuration, bitstream
reader, intra decoder, frame I/O and RD report, unmodified, with every WZ
frame decoded by dvc_decode_wz_frames.  Its decoded luma, per-frame bits and
PSNR must equal the reference decoder's own ParallelMode 0 run (the golden
sequences), the bitstream reaching the library exactly as the reference read
it."""
import os

import numpy as np
import pytest

from dvc_b200 import synth
from oracle import refrun

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("seq", ["qcif_g2_q4_full", "qcif_g4_q8", "cif_g4_q6_full", "qcif_still_g4_q4_full",
                                 "cif_g2_q8_wz"])
def test_reference_dvcdec_bound_to_library_matches_mode0(golden_dir, tmp_path, seq):
    binary = os.path.join(refrun.REF, "DvcDec_b200")
    assert os.path.exists(binary), "oracle/_ref/DvcDec_b200 was not built (make -C oracle binding)"
    g = np.load(os.path.join(golden_dir, f"seq_{seq}.npz"))
    n = int(g["n_frames"])
    ori, key = synth.make_sequence(str(g["kind"]), n, int(g["seed"]))
    d = str(tmp_path)
    oy, ky, st = os.path.join(d, "o.yuv"), os.path.join(d, "k.yuv"), os.path.join(d, "s.txt")
    synth.write_yuv420(oy, ori)
    synth.write_yuv420(ky, key)
    synth.write_frame_stat(st, n)
    g["wz"].tofile(os.path.join(d, "s.wz"))
    g["intra"].tofile(os.path.join(d, "s.intra"))
    env = {"DVC_B200_DATA": os.path.join(ROOT, "dvc_b200", "ladders"),
           "DVC_B200_TABLES": os.path.join(ROOT, "dvc_b200", "_tables")}
    r = refrun.decode(oy, os.path.join(d, "s.wz"), os.path.join(d, "s.intra"), ky, st, mode=2,
                      binary="DvcDec_b200", env_extra=env, timeout=600)
    h, w = g["dec_y"].shape[1:]
    dec = np.frombuffer(r["yuv"], np.uint8).reshape(-1, h, w)
    assert np.array_equal(dec, g["dec_y"])
    rd = refrun.parse_rd(r["rd"])
    for f, b, p, wz in zip(g["frames"], g["bits"], g["psnr"], g["is_wz"]):
        assert rd[int(f)][0] == b and "%.2f" % rd[int(f)][1] == "%.2f" % p
        assert (rd[int(f)][2] == "WZ") == bool(wz)
