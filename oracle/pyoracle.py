"""Test infrastructure: ctypes binding of the C restatement (oracle/_build/liboracle.so)
and a whole-sequence driver that mirrors the reference's main loop
(DvcDec/src/main.cpp:118-142, DVC_Decoder.cpp:26-474), intra blocks and
deblocking included; used as the checker in tests, smoke()
and bench's CPU leg.
"""
import ctypes as C
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "dvc_b200", "ladders"))
import ladders as lad  # noqa: E402

LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")


class Ladder(C.Structure):
    _fields_ = [("num_codes", C.c_int), ("n", C.c_int), ("e", C.c_int), ("period", C.c_int),
                ("jc", C.POINTER(C.c_int)), ("bpp", C.POINTER(C.c_int)), ("idx", C.POINTER(C.c_int)),
                ("ir", C.POINTER(C.c_int)), ("invh", C.POINTER(C.c_uint32))]


class Frame(C.Structure):
    _fields_ = [("w", C.c_int), ("h", C.c_int), ("qindex", C.c_int),
                ("past", C.c_void_p), ("future", C.c_void_p),
                ("past_idx", C.c_int), ("future_idx", C.c_int), ("cur_idx", C.c_int),
                ("mode", C.c_void_p), ("skip_mode", C.c_int), ("intra_mode", C.c_int),
                ("ac_range", C.c_void_p), ("crc", C.c_void_p), ("acc_synd", C.c_void_p),
                ("recon", C.c_void_p), ("wz_bits", C.c_int),
                ("start_code", C.c_void_p), ("accepted_code", C.c_void_p),
                ("deblock_flag", C.c_void_p), ("alpha", C.c_void_p), ("si_initial", C.c_void_p),
                ("si_final", C.c_void_p), ("entropy", C.c_void_p)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(LIB_PATH + " (run make -C oracle oracle)")
        _lib = C.CDLL(LIB_PATH)
        _lib.dvco_ldpca_decode.restype = C.c_int
        _lib.dvco_ldpca_decode_iter.restype = C.c_int
        _lib.dvco_compute_ce.restype = C.c_float
        _lib.dvco_compute_ce.argtypes = [C.c_void_p, C.c_int]
        _lib.dvco_crc8_bits.restype = C.c_uint8
        _lib.dvco_crc8_bits.argtypes = [C.c_void_p, C.c_int]
        _lib.dvco_decode_wz_frame.restype = C.c_int
        _lib.dvco_decode_wz_frame.argtypes = [C.POINTER(Ladder), C.POINTER(Frame)]
        _lib.dvco_belief_propagation.restype = C.c_int
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class OracleLadder:
    """Expanded ladder tables + GF(2) inverse in the layout the C oracle reads."""

    _cache = {}

    def __init__(self, n):
        L = lad.ladder_for(lad.read_compact(os.path.join(ROOT, "dvc_b200", "ladders", "ldpca_ladders.bin")), n)
        nc, n, e, period, jc, codes = lad.expand(L)
        self.n, self.e, self.num_codes, self.period = n, e, nc, period
        self.jc = np.ascontiguousarray(jc, np.int32)
        self.bpp = np.array([c[0] for c in codes], np.int32)
        self.idx = np.zeros((nc, period), np.int32)
        for c, (b, idx, _) in enumerate(codes):
            self.idx[c, :b] = idx
        self.ir = np.ascontiguousarray(np.stack([c[2] for c in codes]), np.int32)
        inv_path = os.path.join(HERE, "_ref", "LDPCA_LadderFile", f"Inverse_Matrix_H_Reg{n}.bin")
        if os.path.exists(inv_path):
            raw = np.fromfile(inv_path, np.uint8)
        else:
            raw = np.frombuffer(lad.inverse_to_reference_bin(lad.gf2_inverse(lad.full_rate_h(L))), np.uint8)
        self.invh = raw.view("<u4").copy()
        self.synd_len = (n // period) * self.bpp
        self.c = Ladder(nc, n, e, period, self.jc.ctypes.data_as(C.POINTER(C.c_int)),
                        self.bpp.ctypes.data_as(C.POINTER(C.c_int)), self.idx.ctypes.data_as(C.POINTER(C.c_int)),
                        self.ir.ctypes.data_as(C.POINTER(C.c_int)), self.invh.ctypes.data_as(C.POINTER(C.c_uint32)))

    @classmethod
    def get(cls, n):
        if n not in cls._cache:
            cls._cache[n] = cls(n)
        return cls._cache[n]


def ldpca_decode(ladder, lr, acc_bits, crc, entropy, max_iter=50):
    """One LdpcaDecoder call (max_iter BP iterations per code; the reference's
    cap is 50). Returns (decoded bits, rate, start code, accepted code, log-LR)."""
    lr = np.ascontiguousarray(lr, np.float32).copy()
    acc = np.ascontiguousarray(acc_bits, np.uint8)
    dec = np.zeros(ladder.n, np.uint8)
    rate = C.c_int(0)
    start = C.c_int(0)
    acc_code = lib().dvco_ldpca_decode_iter(C.byref(ladder.c), _p(lr), _p(acc), _p(dec), C.byref(rate),
                                            C.c_uint8(crc), C.c_float(entropy), C.byref(start), max_iter)
    return dec, rate.value, start.value, acc_code, lr


def compute_ce(lr):
    lr = np.ascontiguousarray(lr, np.float32)
    return float(np.float32(lib().dvco_compute_ce(_p(lr), len(lr))))


def crc8_bits(bits):
    bits = np.ascontiguousarray(bits, np.uint8)
    return int(lib().dvco_crc8_bits(_p(bits), len(bits)))


def accumulated_syndrome(ladder, src_bits):
    src = np.ascontiguousarray(src_bits, np.uint8)
    acc = np.zeros(ladder.n, np.uint8)
    lib().dvco_accumulated_syndrome(C.byref(ladder.c), _p(src), _p(acc))
    return acc


def decode_frame(stream, fr, past, future, recon_init=None, want=()):
    """Decode one WZ frame with the oracle. Returns dict(recon, wz_bits, start, accepted, ...)."""
    w, h = stream.width, stream.height
    ladder = OracleLadder.get(w * h // 16)
    qb = fr.crc.shape[0]
    recon = np.zeros(w * h, np.uint8) if recon_init is None else np.ascontiguousarray(recon_init.reshape(-1)).copy()
    past = np.ascontiguousarray(past.reshape(-1), np.uint8)
    future = np.ascontiguousarray(future.reshape(-1), np.uint8)
    mode = np.ascontiguousarray(fr.mode, np.uint8)
    acr = np.array(fr.ac_range, np.int32)
    crc = np.ascontiguousarray(fr.crc, np.uint8)
    acc = np.ascontiguousarray(fr.acc_synd, np.uint8)
    start = np.zeros(max(qb, 1), np.int32)
    accepted = np.zeros(max(qb, 1), np.int32)
    dbf = np.zeros(w * h, np.uint8)
    ent = np.zeros(max(qb, 1), np.float32)
    alpha = np.zeros(w * h, np.float32) if "alpha" in want else None
    si0 = np.zeros(w * h, np.uint8) if "si" in want else None
    si1 = np.zeros(w * h, np.uint8) if "si" in want else None
    f = Frame(w, h, stream.qindex, _p(past), _p(future), fr.past, fr.future, fr.idx, _p(mode),
              fr.skip_mode, fr.intra_mode, _p(acr), _p(crc), _p(acc), _p(recon), 0,
              _p(start), _p(accepted), _p(dbf),
              _p(alpha) if alpha is not None else None, _p(si0) if si0 is not None else None,
              _p(si1) if si1 is not None else None, _p(ent))
    rc = lib().dvco_decode_wz_frame(C.byref(ladder.c), C.byref(f))
    if rc != 0:
        raise RuntimeError("oracle decode failed rc=%d" % rc)
    out = dict(recon=recon.reshape(h, w), wz_bits=f.wz_bits, start=start[:qb].copy(),
               accepted=accepted[:qb].copy(), deblock_flag=dbf.reshape(h, w), entropy=ent[:qb].copy())
    if alpha is not None:
        out["alpha"] = alpha.reshape(h, w)
    if si0 is not None:
        out["si_initial"] = si0.reshape(h, w)
        out["si_final"] = si1.reshape(h, w)
    return out


def deblock(recon, flag, type_map, past_mode, qindex, intra_qp):
    """dvco_deblock: the reference's deblocking filter of one frame (deblock.cpp:346-386)."""
    h, w = recon.shape
    rec = np.ascontiguousarray(recon, np.uint8)
    fl = np.ascontiguousarray(flag, np.uint8).reshape(-1)
    tm = np.ascontiguousarray(type_map, np.uint8).reshape(-1)
    pm = None if past_mode is None else np.ascontiguousarray(past_mode, np.uint8).reshape(-1)
    out = np.zeros((h, w), np.uint8)
    f = lib().dvco_deblock
    f.restype = None
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
    f(_p(rec), _p(fl), _p(tm), _p(pm) if pm is not None else None, w, h, qindex, intra_qp, _p(out))
    return out


def intra_decode_frame(stream, fr, data, bit_offset, recon):
    """dvco_intra_decode_frame: the intra blocks of WZ frame `fr` from the
    sequence's intra bit string `data` (uint8 array) at `bit_offset`, written
    into `recon` ([H, W] uint8, in place); returns the new bit offset."""
    f = lib().dvco_intra_decode_frame
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t), C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    assert recon.dtype == np.uint8 and recon.flags.c_contiguous and recon.shape == (stream.height, stream.width)
    mode = np.ascontiguousarray(fr.mode, np.uint8)
    off = C.c_size_t(bit_offset)
    if f(_p(data), data.size, C.byref(off), stream.width, stream.height, stream.intra_qp, _p(mode), _p(recon)) != 0:
        raise RuntimeError("oracle: intra bit string of frame %d does not decode" % fr.idx)
    return off.value


def psnr(a, b):
    """frame.cpp:115-124"""
    d = a.astype(np.int64) - b.astype(np.int64)
    mse = float((d * d).sum()) / float(a.size)
    return 0.0 if mse == 0.0 else 10.0 * math.log10(255.0 * 255.0 / mse)


def decode_sequence(stream, key_frames, ori_frames, key_bits, key_psnr, frames=None, intra_bitstream=None):
    """Decode every WZ frame of a stream in the reference's order.

    intra_bitstream: the sequence's intra bit string (bytes), needed when frames
    have intra blocks; a frame's intra blocks are decoded into its buffer first
    and their bits count into its rate (DVC_Decoder.cpp:41-46).  With `frames`,
    only those frames are WZ-decoded (the intra bit string is still read
    through every frame, since it is one string in decoding order).

    Returns dict(recon[T,H,W], bits{frame}, psnr{frame}, planes{frame: (start, accepted)}).
    """
    from dvc_b200 import bitstream as bs
    recon = key_frames.copy()
    bits, ps, planes = dict(key_bits), dict(key_psnr), {}
    order = bs.sequence_order(stream.n_frames, stream.gop)
    data = None if intra_bitstream is None else np.frombuffer(bytes(intra_bitstream), np.uint8)
    off = 0
    for (m, b, e) in order:
        fr = stream.frames[m]
        intra_bits = 0
        if fr.intra_mode:
            if data is None:
                raise ValueError("frame %d has intra blocks; pass the intra bit string" % m)
            before = off
            off = intra_decode_frame(stream, fr, data, off, recon[m])
            intra_bits = off - before
        if frames is not None and m not in frames:
            continue
        r = decode_frame(stream, fr, recon[b], recon[e], recon_init=recon[m])
        recon[m] = r["recon"]
        if stream.deblock:
            # the filtered frame is the decoded frame and later levels' reference (DVC_Decoder.cpp:429-435)
            past = stream.frames.get(fr.past)
            recon[m] = deblock(r["recon"], r["deblock_flag"], fr.mode, None if past is None else past.mode,
                               stream.qindex, stream.intra_qp)
        bits[m] = fr.skip_bits + fr.intra_map_bits + r["wz_bits"] + intra_bits
        ps[m] = psnr(recon[m], ori_frames[m])
        planes[m] = (r["start"], r["accepted"])
    return dict(recon=recon, bits=bits, psnr=ps, planes=planes)
