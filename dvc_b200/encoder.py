"""Wyner-Ziv encoder for test and benchmark inputs.

Restates the reference encoder's WZ path, SkipBlock 0 or 1 (DvcEnc/src, paths
relative to the reference tree):
  findSkipBlock + minimum-count rule    skipBlock.cpp:7-66
  forwardTransform + AC dynamic range   transform.cpp:229-275
  quantize / quantize44                 quantization.cpp:81-140
  extractBitplane                       bitplane.cpp:4-39
  LdpcaEncoder (CRC-8, H*x, accumulate) LdpcaEncoder.cpp:64-95
  writeWZbitstream / outputGOP          wzbitstream.cpp:7-97 (JBIG maps by
                                        the library's T.82 encoder)
so that its bitstreams are byte-identical to the reference encoder's for
IntraMode 0 (checked by tests/test_encoder.py against the golden bitstreams).
IntraMode 1 (``encode_sequence_intra``) follows the reference's principle and
syntax with estimates of its own: the intra map from a rate comparison
(``intra_decision``) and the intra blocks coded by this library's CAVLC coder
(dvc_intra_encode_frame); its streams decode identically in the reference
decoder and in this library (golden *_own_full sequences).
Vectorised with numpy over all 4x4 blocks of a frame.
"""
import os

import numpy as np

from . import bitstream as bs
from . import jbig
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


def _blocks44(mask88):
    """8x8-block mask [H/8, W/8] -> per 4x4 block in raster order [H/4 * W/4]."""
    return np.repeat(np.repeat(np.asarray(mask88, bool), 2, axis=0), 2, axis=1).reshape(-1)


def encode_wz_frame(frame, q, skip88=None, other88=None):
    """Encode one WZ frame. Returns (ac_range[16], crc[qbits], acc_synd[qbits, n/8]).

    skip88: 8x8 blocks left out of the AC ranges and coded as zero bits
    (forwardTransform, transform.cpp:229-275; extractBitplane, bitplane.cpp:13-34);
    other88: further 8x8 blocks coded as zero bits (intra blocks)."""
    h, w = frame.shape
    n = w * h // 16
    qt, qbt = bs.QTABLE[q], bs.QBITS[q]
    T = forward_transform(frame).reshape(n, 16)
    skip = _blocks44(skip88) if skip88 is not None else np.zeros(n, bool)
    zero = skip | (_blocks44(other88) if other88 is not None else False)
    ac_range = np.zeros(16, np.int64)
    if (~skip).any():
        ac_range[1:] = np.abs(T[~skip, 1:]).max(axis=0)
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
            planes.append(np.where(zero, 0, (Q[:, idx] >> b) & 1).astype(np.uint8))
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


def skip_decision(cur, past, q):
    """The reference encoder's skip map of a frame (findSkipBlock,
    skipBlock.cpp:7-66): blocks passing the MSE test, cancelled (all zero) when
    fewer than (int)(8 * coded map bytes * U / QbitsNumPerBlk) qualify (U = 3.0,
    defines.h:11).  Returns (map [H/8, W/8] bool, coded map bytes or None)."""
    sk = skip_blocks(cur, past)
    coded = jbig.encode_mode_map(sk)
    qbits = int(sum(bs.QBITS[q]))
    skip_min = int(float(len(coded) << 3) * 3.0 / float(qbits))
    if int(sk.sum()) < skip_min:
        return np.zeros_like(sk), None
    return sk, coded


# intra decision: search range of the encoder's side-information estimate
INTRA_SEARCH = 4
GAMA = 2.0  # rate-estimate constant of the reference's mode decision (defines.h:16)


def _coef_variance():
    """Relative variances K of the 16 transform coefficients of a separable
    first-order Markov source (rho = 0.6): diag(C R C^T)_i diag(C R C^T)_j
    times the post-scale squared, as the reference's mode decision models them
    (transform.cpp:67-111)."""
    rho = 0.6
    R = np.array([[rho ** abs(i - j) for j in range(4)] for i in range(4)])
    Cm = np.array([[1, 1, 1, 1], [2, 1, -1, -2], [1, -1, -1, 1], [1, -2, 2, -1]], np.float64)
    d = np.diag(Cm @ R @ Cm.T)
    return (np.outer(d, d).reshape(16) * _post_scale() ** 2)


def _best_match(cur, ref, r):
    """Per 8x8 block of cur, the ref block within +-r integer pixels with the
    lowest SAD (first in (dy, dx) raster order on ties; the frame edge is
    extended), as [H/8, 8, W/8, 8]."""
    h, w = cur.shape
    hb, wb = h // 8, w // 8
    c = cur.astype(np.int16)
    pad = np.pad(ref.astype(np.int16), r, mode="edge")
    best = np.full((hb, wb), np.iinfo(np.int32).max, np.int32)
    bdy = np.zeros((hb, wb), np.int32)
    bdx = np.zeros((hb, wb), np.int32)
    for dy in range(-r, r + 1):
        for dx in range(-r, r + 1):
            d = np.abs(c - pad[r + dy:r + dy + h, r + dx:r + dx + w]).astype(np.int32)
            sad = d.reshape(hb, 8, w).sum(axis=1).reshape(hb, wb, 8).sum(axis=2)
            better = sad < best
            best = np.where(better, sad, best)
            bdy = np.where(better, dy, bdy)
            bdx = np.where(better, dx, bdx)
    k = np.arange(8)
    rows = (np.arange(hb)[:, None] * 8 + r + bdy)[:, :, None] + k  # [hb, wb, 8]
    cols = (np.arange(wb)[None, :] * 8 + r + bdx)[:, :, None] + k
    blk = pad[rows[:, :, :, None], cols[:, :, None, :]].astype(np.int32)  # [hb, wb, 8, 8]
    return blk.transpose(0, 2, 1, 3)


def _steps(T, skip44, q):
    """AC ranges over non-skip blocks and the quantiser step of each coefficient."""
    qt = bs.QTABLE[q]
    ac_range = np.zeros(16, np.int64)
    if (~skip44).any():
        ac_range[1:] = np.abs(T[~skip44, 1:]).max(axis=0)
    step = np.zeros(16, np.int64)
    step[0] = 1024 // qt[0]
    for i in range(1, 16):
        if qt[i] > 0:
            step[i] = int(np.ceil(float((int(ac_range[i]) + 1) << 1) / float(qt[i])))
    return ac_range, step


def side_estimate(cur, past, future):
    """The encoder's side-information estimate: the average of the best
    +-INTRA_SEARCH-pixel matches of each 8x8 block in the past and future
    originals, as [H, W] int32."""
    h, w = cur.shape
    si = (_best_match(cur, past, INTRA_SEARCH) + _best_match(cur, future, INTRA_SEARCH) + 1) >> 1
    return si.reshape(h, w)


def intra_decision(cur, past, future, skip88, q, intra_qp=30, si=None):
    """This encoder's intra map of a frame, by the reference's principle
    (intra_selection, modeSelection.cpp): an 8x8 block is intra when the
    estimated WZ rate of its four 4x4 blocks exceeds their intra rate.
    WZ rate: per coefficient with step 0 < D < 4 sqrt(K) MAD, log(4 GAMA
    sqrt(K) MAD / D) rounded, summed (the reference's Laplacian estimate), with
    MAD = (sum |cur - SI| + 8) >> 4 against a side-information estimate (the
    average of the best +-4-pixel matches in the past and future originals;
    the reference interpolates with its own motion search, FastMCFI.cpp).
    Intra rate: the bits this library's intra coder spends on each block
    coded with every non-skip block intra (the reference fits a rate model).
    The reference's minimum-count rule then applies (recal_decision, U = 3.0).
    Returns (map [H/8, W/8] bool, coded map bytes or None)."""
    from . import intra as intra_codec
    h, w = cur.shape
    skip = np.zeros((h // 8, w // 8), bool) if skip88 is None else np.asarray(skip88, bool)
    T = forward_transform(cur).reshape(-1, 16)
    _, step = _steps(T, _blocks44(skip), q)
    if si is None:
        si = side_estimate(cur, past, future)
    mad = (np.abs(cur.astype(np.int32) - si).reshape(h // 4, 4, w // 4, 4).sum(axis=(1, 3)) + 8) >> 4
    sk = np.sqrt(_coef_variance())
    lim = 4.0 * sk[None, None, :] * mad[..., None]  # 4 / alpha
    with np.errstate(divide="ignore", invalid="ignore"):
        temp = 4.0 * GAMA * sk[None, None, :] * mad[..., None] / step[None, None, :]
        r = np.where((step[None, None, :] > 0) & (step[None, None, :] < lim) & (temp >= 1.0), np.log(temp), 0.0)
    rwz = np.floor(r + 0.5).sum(axis=2)  # [H/4, W/4]
    buf = np.zeros(w * h + 64, np.uint8)
    _, _, riw = intra_codec.encode_frame(cur, ~skip, intra_qp, buf, 0, with_bits=True)
    rwz88 = rwz.reshape(h // 8, 2, w // 8, 2).sum(axis=(1, 3))
    riw88 = riw.reshape(h // 8, 2, w // 8, 2).sum(axis=(1, 3))
    cand = (rwz88 > riw88) & ~skip
    if not cand.any():
        return cand, None
    coded = jbig.encode_mode_map(cand)
    if int(cand.sum()) < int(float(len(coded) << 3) * 3.0 / float(int(sum(bs.QBITS[q])))):
        return np.zeros_like(cand), None
    return cand, coded


def encode_sequence(frames, gop, q, intra_qp=30, deblock=0, skip=0):
    """WZ bitstream (bytes) of a luma sequence with key frames every `gop` frames.

    skip=1 runs the reference encoder's skip test against the past key or WZ
    original, with its minimum-count rule, and codes the map with JBIG.
    IntraMode is 0 here (the reference then also leaves the deblocking filter
    to the decoder, DVC_Encoder.cpp:41-81, so deblock only sets the header
    byte); ``encode_sequence_intra`` adds intra blocks."""
    return encode_sequence_intra(frames, gop, q, intra_qp, deblock, skip, intra=0)[0]


def encode_sequence_intra(frames, gop, q, intra_qp=30, deblock=0, skip=0, intra=1, si_cache=None):
    """(WZ bitstream, intra bitstream) of a luma sequence; intra=1 chooses intra
    blocks with ``intra_decision`` and codes them (dvc_intra_encode_frame) into
    one bit string, frames in coding order, as the reference's IntraBitstream
    file holds them.  The WZ bitplanes of skip and intra blocks are zero, and
    the AC ranges leave out skip blocks only (bitplane.cpp:13-34,
    transform.cpp:229-275).  si_cache: a dict shared by calls on the same
    frames (the side-information estimate does not depend on q)."""
    from . import intra as intra_codec
    t, h, w = frames.shape
    if (w, h) == (176, 144):
        res = 0
    elif (w, h) == (352, 288):
        res = 1
    else:
        raise ValueError("only QCIF and CIF")
    out = bytearray([res, q, intra_qp, gop, (t >> 8) & 0xFF, t & 0xFF, deblock])
    ibuf = np.zeros(t * w * h + 64, np.uint8)
    ibits = 0
    bands = bs.coded_ac_bands(q)
    for i in range(0, t, gop):
        e = min(i + gop, t - 1)
        for (m, b, fe) in bs.gop_order(i, e):
            sk, coded = skip_decision(frames[m], frames[b], q) if skip else (None, None)
            it, icoded = None, None
            if intra:
                si = None if si_cache is None else si_cache.get((m, b, fe))
                if si is None:
                    si = side_estimate(frames[m], frames[b], frames[fe])
                    if si_cache is not None:
                        si_cache[(m, b, fe)] = si
                it, icoded = intra_decision(frames[m], frames[b], frames[fe], sk, q, intra_qp, si)
            acr, crc, acc = encode_wz_frame(frames[m], q, skip88=sk, other88=it if icoded is not None else None)
            for idx in bands:
                out += bytes([(int(acr[idx]) >> 8) & 0xFF, int(acr[idx]) & 0xFF])
            out += (bytes([1]) + coded) if coded is not None else bytes([0])
            out += (bytes([1]) + icoded) if icoded is not None else bytes([0])
            if icoded is not None:
                ibits, _ = intra_codec.encode_frame(frames[m], it, intra_qp, ibuf, ibits)
            for j in range(len(crc)):
                out.append(int(crc[j]))
                out += acc[j].tobytes()
    return bytes(out), ibuf[:(ibits + 7) >> 3].tobytes()
