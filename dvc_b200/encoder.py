"""Wyner-Ziv encoder for test and benchmark inputs (no skip or intra blocks).

Restates the reference encoder's path for SkipBlock=0, IntraMode=0
(DvcEnc/src, paths relative to the reference tree):
  forwardTransform + AC dynamic range   transform.cpp:229-275
  quantize / quantize44                 quantization.cpp:81-140
  extractBitplane                       bitplane.cpp:4-39
  LdpcaEncoder (CRC-8, H*x, accumulate) LdpcaEncoder.cpp:64-95
  writeWZbitstream / outputGOP          wzbitstream.cpp:7-97
so that its bitstreams are byte-identical to the reference encoder's for those
settings (checked by tests/test_encoder.py against the golden bitstreams).
Vectorised with numpy over all 4x4 blocks of a frame.
"""
import os

import numpy as np

from . import bitstream as bs
from .ladders import ladders as lad

_HERE = os.path.dirname(os.path.abspath(__file__))
_LADDERS = None


def _ladder(n):
    global _LADDERS
    if _LADDERS is None:
        _LADDERS = lad.read_compact(os.path.join(_HERE, "ladders", "ldpca_ladders.bin"))
    return lad.ladder_for(_LADDERS, n)


def _post_scale():
    """initTransform, DvcEnc transform.cpp (same constants as the decoder's)."""
    a, b = 0.5, np.sqrt(0.4)
    a2, b2, ab = 0.25, 0.4, a * b
    return np.array([a2, ab / 2, a2, ab / 2, ab / 2, b2 / 4, ab / 2, b2 / 4,
                     a2, ab / 2, a2, ab / 2, ab / 2, b2 / 4, ab / 2, b2 / 4], np.float64)


def _round(x):
    """ROUND, defines.h: half away from zero, truncating conversion."""
    return np.where(x >= 0.0, np.trunc(x + 0.5), -np.trunc(-x + 0.5)).astype(np.int64)


def forward_transform(frame):
    """4x4 integer transform of every block: (H/4, W/4, 16) int64 in block raster order."""
    h, w = frame.shape
    x = frame.astype(np.int64).reshape(h // 4, 4, w // 4, 4).transpose(0, 2, 1, 3)  # (bi, bj, m, n)
    r0, r1, r2, r3 = x[:, :, 0, :], x[:, :, 1, :], x[:, :, 2, :], x[:, :, 3, :]
    t0 = r0 + r1 + r2 + r3
    t1 = 2 * r0 + r1 - r2 - 2 * r3
    t2 = r0 - r1 - r2 + r3
    t3 = r0 - 2 * r1 + 2 * r2 - r3
    t = np.stack([t0, t1, t2, t3], axis=2)  # (bi, bj, row, col)
    c0, c1, c2, c3 = t[..., 0], t[..., 1], t[..., 2], t[..., 3]
    o = np.stack([c0 + c1 + c2 + c3, 2 * c0 + c1 - c2 - 2 * c3, c0 - c1 - c2 + c3, c0 - 2 * c1 + 2 * c2 - c3],
                 axis=3)
    o = o.reshape(h // 4, w // 4, 16)
    return _round(o.astype(np.float64) * _post_scale())


def encode_wz_frame(frame, q):
    """Encode one WZ frame. Returns (ac_range[16], crc[qbits], acc_synd[qbits, n/8])."""
    h, w = frame.shape
    n = w * h // 16
    qt, qbt = bs.QTABLE[q], bs.QBITS[q]
    T = forward_transform(frame).reshape(n, 16)
    ac_range = np.zeros(16, np.int64)
    ac_range[1:] = np.abs(T[:, 1:]).max(axis=0)
    ac_range[0] = 0
    step = np.zeros(16, np.int64)
    step[0] = 1024 // qt[0]
    ls = np.zeros(16, np.int64)
    for i in range(1, 16):
        if qt[i] > 0:
            step[i] = int(np.ceil(float((int(ac_range[i]) + 1) << 1) / float(qt[i])))
            ls[i] = (qt[i] - 2) // 2
    Q = np.zeros_like(T)
    Q[:, 0] = np.sign(T[:, 0]) * (np.abs(T[:, 0]) // step[0])
    for i in range(1, 16):
        if step[i] > 0:
            Q[:, i] = (np.sign(T[:, i]) * (np.abs(T[:, i]) // step[i])) + ls[i]
    planes = []
    band = 0
    while band < 16 and qbt[bs.ZIGZAG[band]] > 0:
        idx = bs.ZIGZAG[band]
        for b in range(qbt[idx] - 1, -1, -1):
            planes.append(((Q[:, idx] >> b) & 1).astype(np.uint8))
        band += 1
    L = _ladder(n)
    crc = np.array([crc8_bits(p) for p in planes], np.uint8)
    acc = np.stack([np.packbits(accumulated_syndrome(L, p), bitorder="big") for p in planes])
    return ac_range.astype(np.int32), crc, acc


_CRC_TABLE = None


def crc8_bits(bits):
    """CRC-8 (x^8+x^2+x+1, init 0) of a bit vector packed MSB first (crc8.h, BitToByte)."""
    global _CRC_TABLE
    if _CRC_TABLE is None:
        t = []
        for b in range(256):
            c = b
            for _ in range(8):
                c = ((c << 1) ^ 0x07) & 0xFF if c & 0x80 else (c << 1) & 0xFF
            t.append(c)
        _CRC_TABLE = t
    crc = 0
    for byte in np.packbits(bits, bitorder="big").tolist():
        crc = _CRC_TABLE[crc ^ byte]
    return crc


def accumulated_syndrome(L, src):
    """Full-rate syndrome H*x followed by the prefix xor (LdpcaEncoder.cpp:76-85)."""
    n = L["N"]
    cols = np.repeat(np.arange(n), np.diff(L["jc"]))
    s = np.zeros(n, np.int64)
    np.add.at(s, L["ir_full"], src[cols].astype(np.int64))
    return (np.bitwise_xor.accumulate((s & 1).astype(np.uint8))).astype(np.uint8)


def skip_blocks(cur, past):
    """8x8 blocks the reference encoder would skip: MSE against the past original
    below 10 (DvcEnc/src/skipBlock.cpp:7-45, defines.h:10)."""
    h, w = cur.shape
    d = cur.astype(np.float64) - past.astype(np.float64)
    mse = (d * d).reshape(h // 8, 8, w // 8, 8).sum(axis=(1, 3)) / 64.0
    return mse < 10.0


def encode_sequence(frames, gop, q, intra_qp=30, deblock=0, skip=0):
    """WZ bitstream (bytes) of a luma sequence with key frames every `gop` frames.

    skip=1 runs the encoder's skip test; a frame with no qualifying block keeps
    skip mode off, as the reference does (its minimum-count rule cancels skip
    mode, skipBlock.cpp:47-66).  Coding a frame that has skip blocks needs a
    JBIG encoder, which this encoder does not have: it raises.  IntraMode is
    always 0 (the reference then also leaves the deblocking filter to the
    decoder, DVC_Encoder.cpp:41-81, so deblock only sets the header byte)."""
    t, h, w = frames.shape
    if (w, h) == (176, 144):
        res = 0
    elif (w, h) == (352, 288):
        res = 1
    else:
        raise ValueError("only QCIF and CIF")
    out = bytearray([res, q, intra_qp, gop, (t >> 8) & 0xFF, t & 0xFF, deblock])
    bands = bs.coded_ac_bands(q)
    for i in range(0, t, gop):
        e = min(i + gop, t - 1)
        for (m, b, fe) in bs.gop_order(i, e):
            if skip and skip_blocks(frames[m], frames[b]).any():
                raise NotImplementedError("frame %d has skip blocks; coding its JBIG skip map is not implemented" % m)
            acr, crc, acc = encode_wz_frame(frames[m], q)
            for idx in bands:
                out += bytes([(int(acr[idx]) >> 8) & 0xFF, int(acr[idx]) & 0xFF])
            out += bytes([0, 0])  # no skip map, no intra map
            for j in range(len(crc)):
                out.append(int(crc[j]))
                out += acc[j].tobytes()
    return bytes(out)
