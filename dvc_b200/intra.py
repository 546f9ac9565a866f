"""Intra blocks of WZ frames (IntraMode 1) from the sequence's intra bitstream.

The reference reads one bit string for the whole sequence, frame after frame
in its decoding order (DVC_Decoder.cpp:42-46, intraRecon intra.cpp:252-268).
An intra block only predicts from intra neighbours of its own frame, so every
frame's intra pixels can be decoded before, and independently of, the WZ
decoding; ``decode_all`` does that with the library's host decoder
(dvc_intra_decode_frame) and returns, per WZ frame, the pixels and the bits the
frame's blocks took.
"""
import ctypes as C

import numpy as np

from . import bitstream as bs
from . import native


def decode_all(stream, intra_bytes, base_frames=None):
    """dict frame -> (uint8 [H, W] with the intra blocks written, intra bits).

    base_frames: per-frame arrays the intra pixels are written over (the
    decoder's starting frame content); zeros when omitted."""
    data = np.frombuffer(bytes(intra_bytes), np.uint8)
    off = C.c_size_t(0)
    out = {}
    for (m, b, e) in bs.sequence_order(stream.n_frames, stream.gop):
        fr = stream.frames[m]
        if not fr.intra_mode:
            continue
        rec = (np.array(base_frames[m], np.uint8, copy=True) if base_frames is not None
               else np.zeros((stream.height, stream.width), np.uint8))
        mode = np.ascontiguousarray(fr.mode, np.uint8)
        before = off.value
        rc = native.lib().dvc_intra_decode_frame(data.ctypes.data_as(C.c_void_p), len(data), C.byref(off),
                                                stream.width, stream.height, stream.intra_qp,
                                                mode.ctypes.data_as(C.c_void_p), rec.ctypes.data_as(C.c_void_p))
        if rc != native.DVC_OK:
            raise ValueError("intra bitstream of frame %d could not be decoded (status %d)" % (m, rc))
        out[m] = (rec, off.value - before)
    return out


def encode_frame(ori, mode88, intra_qp, buf, bit_offset, with_bits=False):
    """Append the intra blocks of one frame (mode88 [H/8, W/8], 1 = intra) to the
    bit string in `buf` (a writable uint8 array) at bit_offset.  Returns (new
    bit offset, uint8 [H, W] with the intra blocks as the decoder reconstructs
    them, other pixels 0) and, with_bits, the bits of each 4x4 block
    [H/4, W/4]."""
    ori = np.ascontiguousarray(ori, np.uint8)
    h, w = ori.shape
    mode = np.ascontiguousarray(np.asarray(mode88) != 0, np.uint8)
    rec = np.zeros((h, w), np.uint8)
    bits = np.zeros((h // 4, w // 4), np.int32)
    off = C.c_size_t(bit_offset)
    rc = native.lib().dvc_intra_encode_frame(ori.ctypes.data_as(C.c_void_p), w, h, intra_qp,
                                            mode.ctypes.data_as(C.c_void_p), buf.ctypes.data_as(C.c_void_p),
                                            len(buf), C.byref(off), rec.ctypes.data_as(C.c_void_p),
                                            bits.ctypes.data_as(C.c_void_p))
    if rc != native.DVC_OK:
        raise ValueError("intra blocks could not be encoded (status %d)" % rc)
    return (off.value, rec, bits) if with_bits else (off.value, rec)
