"""JBIG mode maps of the WZ bitstream (the library's T.82 decoder, host side).

The reference codes each frame's 8x8 skip and intra maps with JBIG-KIT and
stores the coded stripe without its header (DvcEnc/src/wzbitstream.cpp:28-44);
``decode_mode_map`` returns the map and the bytes the stripe occupies, as the
reference's reader does (DvcDec/src/wzbitstream.cpp:38-66); ``encode_mode_map``
writes the same bytes as the reference's writer.
"""
import ctypes as C

import numpy as np

from . import native


def decode_mode_map(buf, w, h):
    """(map uint8 [h, w] of 0/1, bytes used) for the coded map at the start of buf."""
    data = np.frombuffer(bytes(buf), np.uint8)
    out = np.zeros((h, w), np.uint8)
    used = C.c_size_t(0)
    rc = native.lib().dvc_jbig_decode_mode_map(data.ctypes.data_as(C.c_void_p), len(data), w, h,
                                               out.ctypes.data_as(C.c_void_p), C.byref(used))
    if rc != native.DVC_OK:
        raise ValueError("JBIG mode map could not be decoded (status %d)" % rc)
    return out, used.value


def encode_mode_map(m):
    """Coded bytes (stripe data and the closing SDNORM marker) of a 0/1 map [h, w]."""
    m = np.ascontiguousarray(np.asarray(m, np.uint8) != 0, np.uint8)
    h, w = m.shape
    cap = 2 * w * h + 64
    out = np.zeros(cap, np.uint8)
    n = C.c_size_t(0)
    rc = native.lib().dvc_jbig_encode_mode_map(m.ctypes.data_as(C.c_void_p), w, h, out.ctypes.data_as(C.c_void_p),
                                               cap, C.byref(n))
    if rc != native.DVC_OK:
        raise ValueError("JBIG mode map could not be encoded (status %d)" % rc)
    return out[:n.value].tobytes()
