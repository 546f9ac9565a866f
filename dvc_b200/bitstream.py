"""Reader for the reference's WZ bitstream and key-frame side files.

WZ bitstream (DvcDec/src/wzbitstream.cpp:129-210, readGOP :13-126):
    header: resolution u8 (0 QCIF, 1 CIF), Qindex u8, IntraQP u8, GOP u8,
            frame count u16 big-endian, deblocking mode u8;
    then, per GOP [i, min(i+GOP, frames-1)] and in hierarchical (recursive
    mid-point) order, per WZ frame:
        ACRange u16 big-endian for each zig-zag AC band with Qtable > 0,
        skipMode u8 [+ JBIG-coded 8x8 skip map],
        intraMode u8 [+ JBIG-coded 8x8 intra map],
        per bitplane: CRC-8 u8 + N/8 bytes of accumulated syndrome (MSB first).

The JBIG mode maps are decoded by ``jbig.decode_mode_map`` (the library's T.82
decoder).
"""
import numpy as np

ZIGZAG = (0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15)  # global.cpp:36-41

QTABLE = (  # reconstruction.cpp:9-43
    (0,) * 16,
    (16, 8, 0, 0, 8, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0),
    (32, 8, 0, 0, 8, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0),
    (32, 8, 4, 0, 8, 4, 0, 0, 4, 0, 0, 0, 0, 0, 0, 0),
    (32, 16, 8, 4, 16, 8, 4, 0, 8, 4, 0, 0, 4, 0, 0, 0),
    (32, 16, 8, 4, 16, 8, 4, 4, 8, 4, 4, 0, 4, 4, 0, 0),
    (64, 16, 8, 8, 16, 8, 8, 4, 8, 8, 4, 4, 8, 4, 4, 0),
    (64, 32, 16, 8, 32, 16, 8, 4, 16, 8, 4, 4, 8, 4, 4, 0),
    (128, 64, 32, 16, 64, 32, 16, 8, 32, 16, 8, 4, 16, 8, 4, 0),
)
QBITS = (  # reconstruction.cpp:44-78
    (0,) * 16,
    (4, 3, 0, 0, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0),
    (5, 3, 0, 0, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0),
    (5, 3, 2, 0, 3, 2, 0, 0, 2, 0, 0, 0, 0, 0, 0, 0),
    (5, 4, 3, 2, 4, 3, 2, 0, 3, 2, 0, 0, 2, 0, 0, 0),
    (5, 4, 3, 2, 4, 3, 2, 2, 3, 2, 2, 0, 2, 2, 0, 0),
    (6, 4, 3, 3, 4, 3, 3, 2, 3, 3, 2, 2, 3, 2, 2, 0),
    (6, 5, 4, 3, 5, 4, 3, 2, 4, 3, 2, 2, 3, 2, 2, 0),
    (7, 6, 5, 4, 6, 5, 4, 3, 5, 4, 3, 2, 4, 3, 2, 0),
)

WZ_B, INTRA_B, SKIP_B = 0, 1, 2


def qbits_per_block(q):
    return sum(QBITS[q])


def coded_ac_bands(q):
    """Zig-zag AC band indices with Qtable > 0 (stops at the first zero, as readGOP does)."""
    out = []
    for j in range(1, 16):
        idx = ZIGZAG[j]
        if QTABLE[q][idx] > 0:
            out.append(idx)
        else:
            break
    return out


def gop_order(begin, end):
    """WZ frame indices of one GOP in the reference's hierarchical order (decodeGOP recursion)."""
    out = []

    def rec(b, e):
        m = (b + e) // 2
        if m > b:
            out.append((m, b, e))
            rec(b, m)
            rec(m, e)

    rec(begin, end)
    return out


def sequence_order(n_frames, gop, start=0, end=None):
    """(frame, past, future) triples in decode order for frames [start, end] (main.cpp:118-142)."""
    if end is None:
        end = n_frames - 1
    out = []
    for i in range(start, end + 1, gop):
        e = min(i + gop, end)
        out += gop_order(i, e)
    return out


class WZFrame:
    __slots__ = ("idx", "past", "future", "ac_range", "skip_mode", "intra_mode", "mode",
                 "skip_bits", "intra_map_bits", "crc", "acc_synd")


class WZStream:
    def __init__(self, width, height, qindex, intra_qp, gop, n_frames, deblock):
        self.width, self.height = width, height
        self.qindex, self.intra_qp, self.gop = qindex, intra_qp, gop
        self.n_frames, self.deblock = n_frames, deblock
        self.frames = {}

    @property
    def n_blocks44(self):
        return self.width * self.height // 16

    @property
    def n_blocks88(self):
        return self.width * self.height // 64


def parse_wz(data):
    """Parse a WZ bitstream (bytes) into a WZStream."""
    data = bytes(data)
    if len(data) < 7:
        raise ValueError("WZ bitstream shorter than its 7-byte header")
    res, q, iqp, gop = data[0], data[1], data[2], data[3]
    n = (data[4] << 8) | data[5]
    deb = data[6]
    if res == 0:
        w, h = 176, 144
    elif res == 1:
        w, h = 352, 288
    else:
        raise ValueError("unsupported resolution code %d (QCIF=0, CIF=1)" % res)
    if not 1 <= q <= 8:
        raise ValueError("Qindex %d out of range 1..8" % q)
    if gop < 1:
        raise ValueError("GOP must be >= 1")
    st = WZStream(w, h, q, iqp, gop, n, deb)
    nb = st.n_blocks44
    synd_bytes = nb // 8
    qb = qbits_per_block(q)
    bands = coded_ac_bands(q)
    pos = [7]

    def take(k):
        p = pos[0]
        if p + k > len(data):
            raise ValueError("truncated WZ bitstream at byte %d (need %d more)" % (p, k))
        pos[0] = p + k
        return data[p:p + k]

    def read_map(b88w, b88h):
        from . import jbig
        buf = data[pos[0]:]
        bitmap, used = jbig.decode_mode_map(buf, b88w, b88h)
        pos[0] += used
        return bitmap, used

    for i in range(0, n, gop):
        e = i + gop
        if e >= n:
            e = n - 1
        for (m, b, fe) in gop_order(i, e):
            fr = WZFrame()
            fr.idx, fr.past, fr.future = m, b, fe
            fr.ac_range = [0] * 16
            for idx in bands:
                u, l = take(2)
                fr.ac_range[idx] = (u << 8) | l
            fr.mode = np.zeros(st.n_blocks88, np.uint8)
            (fr.skip_mode,) = take(1)
            fr.skip_bits = 1
            if fr.skip_mode == 1:
                bm, used = read_map(w // 8, h // 8)
                fr.skip_bits = (used << 3) + 1
                fr.mode[bm.reshape(-1) == 1] = SKIP_B
            (fr.intra_mode,) = take(1)
            fr.intra_map_bits = 1
            if fr.intra_mode == 1:
                bm, used = read_map(w // 8, h // 8)
                fr.intra_map_bits = (used << 3) + 1
                fr.mode[bm.reshape(-1) == 1] = INTRA_B
            fr.crc = np.zeros(qb, np.uint8)
            fr.acc_synd = np.zeros((qb, synd_bytes), np.uint8)
            for j in range(qb):
                fr.crc[j] = take(1)[0]
                fr.acc_synd[j] = np.frombuffer(take(synd_bytes), np.uint8)
            st.frames[m] = fr
    st.consumed = pos[0]
    return st


def parse_frame_stat(path, n_frames):
    """Key-frame bits and PSNR from a per_frame_stat file (frame.cpp:197-247)."""
    bits, psnr = {}, {}
    toks = open(path).read().split()
    for i, t in enumerate(toks):
        if t == "FrameNo:":
            f = int(toks[i + 1])
            if f not in bits:
                bits[f] = int(toks[i + 3])
                psnr[f] = float(np.float32(float(toks[i + 9])))
    missing = [f for f in range(n_frames) if f not in bits]
    if missing:
        raise ValueError("frame %d not found in key-frame info" % missing[0])
    return bits, psnr
