"""dvcdec, the DvcDec-compatible executable: configuration handling on the CPU,
golden sequences decoded through it on the GPU (RD report and decoded luma)."""
import os
import subprocess

import numpy as np
import pytest

from dvc_b200 import build, synth

CFG = """# decoder configuration (the reference decoder's keys)
OriginalSequence  = "{d}/ori.yuv"
WZBitstream       = "{d}/seq.wz"
KeyFrameSequence  = "{d}/key.yuv"
KeyFrameInfo      = "{d}/stat.txt"
RDFile            = "{d}/rd"
OutputSequences   = "{d}/dec"
FrameRate         = 15
ParallelMode      = 2
UseCoreNum        = 1
IntraBitstream    = "{d}/seq.intra"
"""


def _cli():
    if not os.path.exists(build.CLI):
        build.build()
    return build.CLI


def _setup(tmp_path, g):
    d = str(tmp_path)
    ori, key = synth.make_sequence(str(g["kind"]), int(g["n_frames"]), int(g["seed"]))
    synth.write_yuv420(os.path.join(d, "ori.yuv"), ori)
    synth.write_yuv420(os.path.join(d, "key.yuv"), key)
    synth.write_frame_stat(os.path.join(d, "stat.txt"), int(g["n_frames"]))
    g["wz"].tofile(os.path.join(d, "seq.wz"))
    if "intra" in g:
        g["intra"].tofile(os.path.join(d, "seq.intra"))
    else:
        open(os.path.join(d, "seq.intra"), "wb").close()
    cfg = os.path.join(d, "decoder.cfg")
    open(cfg, "w").write(CFG.format(d=d))
    return d, cfg


def test_cli_rejects_bad_arguments(tmp_path):
    r = subprocess.run([_cli()], capture_output=True, text=True)
    assert r.returncode != 0 and "Usage" in r.stderr
    bad = tmp_path / "bad.cfg"
    bad.write_text('NoSuchKey = "x"\n')
    r = subprocess.run([_cli(), "-d", str(bad)], capture_output=True, text=True)
    assert r.returncode != 0 and "not recognized" in r.stderr
    short = tmp_path / "short.cfg"
    short.write_text('WZBitstream = "x"\n')
    r = subprocess.run([_cli(), "-d", str(short)], capture_output=True, text=True)
    assert r.returncode != 0 and "Too few parameters" in r.stderr


def test_cli_refuses_damaged_wz_bitstreams(tmp_path, golden_dir):
    """Truncated WZ bitstreams (cut in headers, AC ranges, JBIG mode maps and
    syndromes) and bad header fields end with an error message and a non-zero
    exit, never a signal; the bitstream is parsed before any GPU work."""
    g = dict(np.load(os.path.join(golden_dir, "seq_qcif_still_g4_q4_full.npz")))
    d, cfg = _setup(tmp_path, g)
    wz = g["wz"].tobytes()
    path = os.path.join(d, "seq.wz")
    cases = [wz[:n] for n in sorted(set(list(range(0, 40)) + list(range(40, len(wz) - 1, max(1, len(wz) // 40)))))]
    cases += [bytes([7]) + wz[1:], wz[:1] + bytes([0]) + wz[2:], wz[:1] + bytes([9]) + wz[2:], wz[:3] + bytes([0]) + wz[4:]]
    for data in cases:
        with open(path, "wb") as f:
            f.write(data)
        r = subprocess.run([_cli(), "-d", cfg], capture_output=True, text=True, timeout=60)
        assert r.returncode > 0, (len(data), r.returncode, r.stderr[-300:])
        assert any(m in r.stderr for m in ("truncated", "shorter than its header", "could not be decoded",
                                           "Unsupport resolution", "Qindex out of range", "GOP must be")), r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("seq", ["qcif_g4_q8", "cif_g2_q2", "qcif_still_g2_q4_skip", "cif_g4_q6_intra",
                                 "cif_g4_q6_full", "qcif_g2_q8_own_full"])
def test_cli_decodes_golden_sequence(tmp_path, golden_dir, seq):
    g = dict(np.load(os.path.join(golden_dir, f"seq_{seq}.npz")))
    d, cfg = _setup(tmp_path, g)
    r = subprocess.run([_cli(), "-d", cfg, "-GPUid=0"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    n = int(g["n_frames"])
    h, w = g["dec_y"].shape[1:]
    dec = np.fromfile(os.path.join(d, "dec.yuv"), np.uint8).reshape(n, h, w)
    rd = open(os.path.join(d, "rd.txt")).read().splitlines()
    for f, b, p, wz in zip(g["frames"], g["bits"], g["psnr"], g["is_wz"]):
        f = int(f)
        line = [x for x in rd if x.startswith("FrameNo: %d," % f)][0]
        if wz:
            assert np.array_equal(dec[f], g["dec_y"][f]), f"frame {f}"
            assert "Bits: %d, PSNR: %.2f (WZ)" % (b, p) in line
        else:
            assert "(KY)" in line
    assert any(x.startswith("Average WZ decoding speed:") for x in rd)


@pytest.mark.gpu
@pytest.mark.parametrize("k", range(4))
def test_cli_frame_range_matches_reference(tmp_path, golden_dir, k):
    """dvcdec -startFrame=a -endFrame=b against the reference decoder run with
    the same flags (tests/golden/ranges.npz): the GOPs before the start only
    advance the intra bitstream (skipGOP, DVC_Decoder.cpp:477-517), the RD
    report lists frames a..b (frame.cpp:255-270) and the decoded luma holds
    frames a..b, or a..b-1 when b is not the last frame (frame.cpp:99-103).
    Every line of the report is compared except the timing figures and the
    reference's per-stage timing section."""
    rg = np.load(os.path.join(golden_dir, "ranges.npz"))
    seq, a, b = str(rg["r%d_seq" % k]), int(rg["r%d_start" % k]), int(rg["r%d_end" % k])
    g = dict(np.load(os.path.join(golden_dir, f"seq_{seq}.npz")))
    d, cfg = _setup(tmp_path, g)
    r = subprocess.run([_cli(), "-d", cfg, "-GPUid=0", "-startFrame=%d" % a, "-endFrame=%d" % b],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert np.array_equal(np.fromfile(os.path.join(d, "dec.yuv"), np.uint8), rg["r%d_yuv" % k])

    def stable(text):
        """The report without its timings: no decoding times, and nothing from the
        reference's per-stage timing section on (SHOW_TIME_INFO, frame.cpp:289-333)."""
        out = []
        for line in text.split("\nTime information of each component:")[0].splitlines():
            if line.startswith(("Total decoding time", "Average WZ decoding speed")):
                continue
            out.append(line.split(", Decoding time")[0])
        while out and not out[-1].strip():
            out.pop()
        return out

    assert stable(open(os.path.join(d, "rd.txt")).read()) == stable(str(rg["r%d_rd" % k]))
