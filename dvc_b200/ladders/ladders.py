"""Compact LDPCA ladder data: read/write, expansion into the reference decoder's
ladder tables, GF(2) inverse of the full-rate matrix, and writers for the
reference's text/binary ladder file formats.

Ladder tables of the reference decoder (ReadLdpcaLadderFile_LdpcaDecoder.cpp:150-184):
numCodes, codeLength N, numEdges E, period, jc[N+1] (edge ranges per column),
and per code: bitsPerPeriod, idxPerPeriod[bpp], ir[E] (row of every edge),
syndLength = (N/period)*bpp, codeRate = syndLength/N.

Compact file layout (little endian), written by ``write_compact``:
    b"LDLA", u32 version=1, u32 n_ladders
    per ladder: u32 N, E, period, numCodes; u16 jc[N+1]; u16 ir_full[E];
                per code: u16 bpp, u16 idx[bpp]
"""
import struct

import numpy as np

MAGIC = b"LDLA"


def read_decoder_lad(path):
    """Parse a reference decoder ladder (.lad text, ReadLadder_decoder)."""
    t = np.array(open(path).read().split(), dtype=np.int64)
    n_codes, n, e, period = (int(v) for v in t[:4])
    i = 4
    jc = t[i:i + n + 1]
    i += n + 1
    codes = []
    for _ in range(n_codes):
        b = int(t[i]); i += 1
        idx = t[i:i + b]; i += b
        ir = t[i:i + e]; i += e
        codes.append((b, idx, ir))
    assert i == len(t), path
    return n_codes, n, e, period, jc, codes


def write_compact(path, ladders):
    with open(path, "wb") as f:
        f.write(MAGIC + struct.pack("<II", 1, len(ladders)))
        for L in ladders:
            f.write(struct.pack("<IIII", L["N"], L["E"], L["period"], len(L["bpp"])))
            f.write(np.asarray(L["jc"], dtype="<u2").tobytes())
            f.write(np.asarray(L["ir_full"], dtype="<u2").tobytes())
            for b, idx in zip(L["bpp"], L["idx"]):
                f.write(struct.pack("<H", b))
                f.write(np.asarray(idx, dtype="<u2").tobytes())


def read_compact(path):
    data = open(path, "rb").read()
    assert data[:4] == MAGIC
    ver, nl = struct.unpack_from("<II", data, 4)
    assert ver == 1
    off = 12
    out = []
    for _ in range(nl):
        n, e, period, nc = struct.unpack_from("<IIII", data, off); off += 16
        jc = np.frombuffer(data, "<u2", n + 1, off).astype(np.int64); off += 2 * (n + 1)
        ir = np.frombuffer(data, "<u2", e, off).astype(np.int64); off += 2 * e
        bpp, idx = [], []
        for _ in range(nc):
            (b,) = struct.unpack_from("<H", data, off); off += 2
            idx.append(np.frombuffer(data, "<u2", b, off).astype(np.int64)); off += 2 * b
            bpp.append(b)
        out.append(dict(N=n, E=e, period=period, jc=jc, ir_full=ir, bpp=bpp, idx=idx))
    return out


def ladder_for(ladders, n):
    for L in ladders:
        if L["N"] == n:
            return L
    raise KeyError(n)


def expand(L):
    """Decoder ladder tables for one codeword length.

    Returns (numCodes, N, E, period, jc, codes) with codes[c] = (bpp, idx, ir)
    exactly as the reference decoder's ladder file holds them.
    """
    n, period = L["N"], L["period"]
    codes = []
    for b, idx in zip(L["bpp"], L["idx"]):
        m = (n // period) * b
        k = np.arange(m)
        bounds = idx[k % b] + (k // b) * period
        ir = np.searchsorted(bounds, L["ir_full"], side="left")
        assert ir.max() < m
        codes.append((b, np.asarray(idx), ir.astype(np.int64)))
    return len(codes), n, L["E"], period, L["jc"], codes


def full_rate_h(L):
    """Dense full-rate parity-check matrix H (N x N, uint8)."""
    n = L["N"]
    h = np.zeros((n, n), np.uint8)
    jc, ir = L["jc"], L["ir_full"]
    for col in range(n):
        for e in range(jc[col], jc[col + 1]):
            h[ir[e], col] ^= 1
    return h


def gf2_inverse(h):
    """Inverse of a square GF(2) matrix (rows packed into uint64 words)."""
    n = h.shape[0]
    w = (2 * n + 63) // 64
    aug = np.zeros((n, w * 64), np.uint8)
    aug[:, :n] = h
    aug[np.arange(n), n + np.arange(n)] = 1
    a = np.packbits(aug, axis=1, bitorder="little").view("<u8").copy()
    for col in range(n):
        wi, bit = col // 64, np.uint64(1) << np.uint64(col % 64)
        rows = np.nonzero(a[col:, wi] & bit)[0]
        if len(rows) == 0:
            raise ValueError("singular")
        p = col + rows[0]
        if p != col:
            a[[col, p]] = a[[p, col]]
        hit = np.nonzero(a[:, wi] & bit)[0]
        hit = hit[hit != col]
        a[hit] ^= a[col]
    bits = np.unpackbits(a.view(np.uint8), axis=1, bitorder="little")
    return bits[:, n:2 * n].copy()


def inverse_to_reference_bin(inv):
    """Rows of ceil(N/32) 32-bit words, bits MSB-first per byte in file order
    (the layout BitToWord produces, LdpcaDecoder.cpp:584-616)."""
    n = inv.shape[0]
    words = (n + 31) // 32
    pad = np.zeros((n, words * 32), np.uint8)
    pad[:, :n] = inv
    return np.packbits(pad, axis=1, bitorder="big").tobytes()


def write_reference_lad(path, expanded):
    n_codes, n, e, period, jc, codes = expanded
    lines = [f"{n_codes} {n} {e} {period} ", " ".join(map(str, jc))]
    for b, idx, ir in codes:
        lines.append(str(b))
        lines.append(" ".join(map(str, idx)))
        lines.append(" ".join(map(str, ir)))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
