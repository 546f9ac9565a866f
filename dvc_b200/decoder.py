"""Whole-sequence Wyner-Ziv decoding on the GPU.

Follows the reference decoder's main loop (DvcDec/src/main.cpp:118-142) and
hierarchical GOP recursion (DVC_Decoder.cpp:26-474): key frames come from the
key-frame sequence, every WZ frame is decoded from its two references.  WZ
frames whose references are available are decoded together as one device batch
(all WZ frames of a GOP-2 sequence at once; GOP 4 needs two levels, GOP 8 three).
"""
import math

import numpy as np

from . import bitstream as bs


def psnr(a, b):
    """frame.cpp:115-124"""
    d = a.astype(np.int64) - b.astype(np.int64)
    mse = float((d * d).sum()) / float(a.size)
    return 0.0 if mse == 0.0 else 10.0 * math.log10(255.0 * 255.0 / mse)


def frame_item(stream, fr, recon):
    past_wz = stream.frames.get(fr.past)
    return dict(width=stream.width, height=stream.height, qindex=stream.qindex, past_idx=fr.past,
                future_idx=fr.future, cur_idx=fr.idx, past=recon[fr.past], future=recon[fr.future],
                mode=fr.mode, skip_mode=fr.skip_mode, intra_mode=fr.intra_mode, ac_range=fr.ac_range,
                crc=fr.crc, acc=fr.acc_synd, recon=recon[fr.idx], deblock=stream.deblock,
                intra_qp=stream.intra_qp, past_mode=None if past_wz is None else past_wz.mode)


def decode_levels(stream, start=0, end=None):
    """Group (frame, past, future) in decode order into batches whose references precede them."""
    order = bs.sequence_order(stream.n_frames, stream.gop, start, end)
    done = set(f for f in range(stream.n_frames) if f not in stream.frames)  # key frames
    levels = []
    pending = list(order)
    while pending:
        lvl = [t for t in pending if t[1] in done and t[2] in done]
        if not lvl:
            raise ValueError("WZ frame references never become available")
        levels.append(lvl)
        for t in lvl:
            done.add(t[0])
        pending = [t for t in pending if t not in lvl]
    return levels


def decode_sequence(ctx, stream, key_frames, ori_frames=None, key_bits=None, key_psnr=None, intra_bitstream=None):
    """Decode every WZ frame. Returns dict(recon, bits, psnr, planes, entropy, deblock_flag).

    intra_bitstream: bytes of the sequence's intra bitstream, needed when frames
    have intra blocks (IntraMode 1); their pixels are decoded first
    (dvc_b200.intra) and the frame's intra bits count into its rate
    (DVC_Decoder.cpp:42-46).
    """
    recon = np.array(key_frames, np.uint8, copy=True)
    bits = dict(key_bits or {})
    ps = dict(key_psnr or {})
    planes, dbf, entropy = {}, {}, {}
    intra_px = {}
    if any(fr.intra_mode for fr in stream.frames.values()):
        if intra_bitstream is None:
            raise ValueError("the stream has intra blocks; pass its intra bitstream")
        from . import intra
        intra_px = intra.decode_all(stream, intra_bitstream, recon)
    for lvl in decode_levels(stream):
        items = []
        for (m, b, e) in lvl:
            fr = stream.frames[m]
            if m in intra_px:
                recon[m] = intra_px[m][0]
            items.append(frame_item(stream, fr, recon))
        outs = ctx.decode_wz_frames(items)
        for (m, b, e), o in zip(lvl, outs):
            fr = stream.frames[m]
            recon[m] = o["recon"]
            bits[m] = fr.skip_bits + fr.intra_map_bits + o["wz_bits"] + (intra_px[m][1] if m in intra_px else 0)
            planes[m] = o["planes"]
            entropy[m] = o["entropy"]
            dbf[m] = o["deblock_flag"]
            if ori_frames is not None:
                ps[m] = psnr(recon[m], ori_frames[m])
    return dict(recon=recon, bits=bits, psnr=ps, planes=planes, entropy=entropy, deblock_flag=dbf)
