"""Test infrastructure: run the reference codec built by oracle/Makefile.

Each run gets its own working directory holding ``LDPCA_LadderFile/`` (the
reference opens its ladders relative to the cwd, DvcDec/src/main.cpp:82-83 and
DvcEnc/src/main.cpp:61-64).  The reference decoder names its outputs with an
overlapping sprintf (DvcDec/src/wzbitstream.cpp:178-179), which with this libc
writes ``./.txt`` and ``./.yuv`` into the cwd; ``decode`` reads them from there.
"""
import os
import shutil
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "_ref")


def ref_available():
    return all(os.path.exists(os.path.join(REF, b)) for b in ("DvcEnc", "DvcDec", "DvcDec_capture")) \
        and os.path.isdir(os.path.join(REF, "LDPCA_LadderFile"))


def _workdir(root=None):
    d = tempfile.mkdtemp(prefix="dvcref_", dir=root)
    os.symlink(os.path.join(REF, "LDPCA_LadderFile"), os.path.join(d, "LDPCA_LadderFile"))
    return d


def encode(yuv, key_yuv, n_frames, size, gop, qindex, skip=0, intra=0, intra_qp=30, deblock=0, workdir=None):
    """Run the reference encoder; returns (wz_path, intra_path, workdir)."""
    d = workdir or _workdir()
    wz = os.path.join(d, "s.wz")
    intra_bs = os.path.join(d, "s.intra")
    cfg = os.path.join(d, "enc.cfg")
    with open(cfg, "w") as f:
        f.write(f'InputFile = "{yuv}"\nFramesToBeEncoded = {n_frames}\nSequenceSize = "{size}"\n'
                f'WZBitstreamFile = "{wz}"\nGOP = {gop}\nQIndex = {qindex}\nSkipBlock = {skip}\n'
                f'IntraMode = {intra}\nKeyFrameSequence = "{key_yuv}"\nIntraBitstreamFile = "{intra_bs}"\n'
                f'IntraQP = {intra_qp}\nDeblockingFilter = {deblock}\n')
    r = subprocess.run([os.path.join(REF, "DvcEnc"), "-d", cfg], cwd=d, capture_output=True, text=True)
    if r.returncode != 0 or not os.path.exists(wz):
        raise RuntimeError("DvcEnc failed: " + r.stdout[-2000:] + r.stderr[-2000:])
    if not os.path.exists(intra_bs):
        open(intra_bs, "wb").close()
    return wz, intra_bs, d


def decode(ori_yuv, wz, intra_bs, key_yuv, stat, mode=0, cores=1, capture=None, capture_pdf=False,
           start=None, end=None, frame_rate=15, binary="DvcDec", timeout=None, env_extra=None):
    """Run the reference decoder in its own cwd.

    Returns dict(rd=<RD text>, yuv=<bytes of the Y-only output>, stdout=..., seconds=wall).
    """
    import time
    d = _workdir()
    cfg = os.path.join(d, "dec.cfg")
    with open(cfg, "w") as f:
        f.write(f'OriginalSequence = "{ori_yuv}"\nWZBitstream = "{wz}"\nKeyFrameSequence = "{key_yuv}"\n'
                f'KeyFrameInfo = "{stat}"\nRDFile = "rd"\nOutputSequences = "dec"\nFrameRate = {frame_rate}\n'
                f'ParallelMode = {mode}\nUseCoreNum = {cores}\nIntraBitstream = "{intra_bs}"\n')
    env = dict(os.environ)
    env.update(env_extra or {})
    if capture:
        env["DVC_CAPTURE"] = capture
        binary = "DvcDec_capture"
        if capture_pdf:
            env["DVC_CAPTURE_PDF"] = "1"
    args = [os.path.join(REF, binary), "-d", cfg]
    if start is not None:
        args += [f"-startFrame={start}", f"-endFrame={end}"]
    t0 = time.time()
    r = subprocess.run(args, cwd=d, capture_output=True, text=True, env=env, timeout=timeout)
    dt = time.time() - t0
    if r.returncode != 0:
        raise RuntimeError("DvcDec failed: " + r.stdout[-3000:] + r.stderr[-2000:])
    rd_path = [p for p in (os.path.join(d, ".txt"), os.path.join(d, "rd.txt")) if os.path.exists(p)][0]
    yuv_path = [p for p in (os.path.join(d, ".yuv"), os.path.join(d, "dec.yuv")) if os.path.exists(p)][0]
    out = dict(rd=open(rd_path).read(), yuv=open(yuv_path, "rb").read(), stdout=r.stdout, seconds=dt)
    shutil.rmtree(d, ignore_errors=True)
    return out


def parse_rd(text):
    """Per-frame (bits, psnr, kind) from the reference RD report (frame.cpp:255-270)."""
    frames = {}
    for line in text.splitlines():
        if line.startswith("FrameNo:"):
            parts = line.replace(",", "").split()
            i = int(parts[1])
            bits = int(parts[3])
            psnr = float(parts[5])
            kind = "WZ" if "(WZ)" in line else "KY"
            frames[i] = (bits, psnr, kind)
    return frames


def read_capture(path):
    """Parse the record stream written by ref_capture.cpp into (tag, bytes) pairs."""
    data = open(path, "rb").read()
    off, out = 0, []
    while off < len(data):
        tag = data[off:off + 4].decode()
        (n,) = struct.unpack_from("<I", data, off + 4)
        out.append((tag, data[off + 8:off + 8 + n]))
        off += 8 + n
    return out


def ldpca_records(caps):
    """Group the LdpcaDecoder records: list of dicts with N, crc, entropy, LR, acc, LLR, decoded, rate."""
    res, cur = [], None
    for tag, b in caps:
        if tag == "LDIN":
            n, crc = struct.unpack_from("<ii", b)
            (ent,) = struct.unpack_from("<f", b, 8)
            cur = dict(N=n, crc=crc, entropy=ent)
        elif tag == "LDLR":
            cur["LR"] = np.frombuffer(b, "<f4").copy()
        elif tag == "LDAS":
            cur["acc"] = np.frombuffer(b, np.uint8).copy()
        elif tag == "LDLL":
            cur["LLR"] = np.frombuffer(b, "<f4").copy()
        elif tag == "LDDE":
            cur["decoded"] = np.frombuffer(b, np.uint8).copy()
        elif tag == "LDRT":
            (cur["rate"],) = struct.unpack("<i", b)
            res.append(cur)
            cur = None
    return res
