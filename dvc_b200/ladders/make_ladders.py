"""Build the compact LDPCA ladder file ``ldpca_ladders.bin`` from the reference's
shipped ladder files.

The reference decoder reads text ladders ``RegDecoder{1584,6336}.lad`` and the
GF(2) inverse of the full-rate parity-check matrix
``Inverse_Matrix_H_Reg{1584,6336}.bin`` (DvcDec/src/main.cpp:82-89,
ReadLdpcaLadderFile_LdpcaDecoder.cpp:131-201).  Only the QCIF (N=1584) pair is
shipped; the CIF (N=6336) pair is missing upstream.  Both decoder ladders follow
from two pieces of data:

* the full-rate parity-check matrix of the encoder ladder
  (release/DvcEnc/LDPCA_LadderFile/RegEncoder{1584,6336}.lad: N, E, jc[N+1], ir[E]);
* per ladder code c, the syndrome positions kept in each period of 66 rows
  (``bitsPerPeriod[c]``, ``idxPerPeriod[c]``), shared by both lengths.

Code c's row of edge e is the first kept syndrome index k whose accumulated
position ``idx[k % bpp] + (k // bpp) * period`` is >= the full-rate row of e
(the accumulated syndrome makes merged rows sums of consecutive full-rate rows).
``expand`` in ``ladders.py`` performs this; this script checks that it reproduces
the shipped QCIF decoder ladder exactly before writing anything.

Usage (needs the reference tree; the output is committed):
    python dvc_b200/ladders/make_ladders.py <reference tree>
"""
import os
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from ladders import expand, read_decoder_lad, write_compact  # noqa: E402


def read_encoder_lad(path):
    t = np.array(open(path).read().split(), dtype=np.int64)
    n, e = int(t[0]), int(t[1])
    jc = t[2:3 + n]
    ir = t[3 + n:3 + n + e]
    assert 3 + n + e == len(t), path
    return n, e, jc, ir


def main(ref):
    rel = os.path.join(ref, "release")
    dec_q = read_decoder_lad(os.path.join(rel, "DvcDec/LDPCA_LadderFile/RegDecoder1584.lad"))
    n_codes, n_q, e_q, period, jc_q, codes_q = dec_q
    n1, e1, jc1, ir1 = read_encoder_lad(os.path.join(rel, "DvcEnc/LDPCA_LadderFile/RegEncoder1584.lad"))
    n2, e2, jc2, ir2 = read_encoder_lad(os.path.join(rel, "DvcEnc/LDPCA_LadderFile/RegEncoder6336.lad"))
    assert (n1, e1) == (n_q, e_q) and np.array_equal(jc1, jc_q)
    bpp = [c[0] for c in codes_q]
    idx = [c[1] for c in codes_q]
    ladders = [
        dict(N=n1, E=e1, period=period, jc=jc1, ir_full=ir1, bpp=bpp, idx=idx),
        dict(N=n2, E=e2, period=period, jc=jc2, ir_full=ir2, bpp=bpp, idx=idx),
    ]
    # the expansion must reproduce every shipped QCIF code
    _, _, _, _, _, codes_x = expand(ladders[0])
    for c, ((b0, i0, r0), (b1, i1, r1)) in enumerate(zip(codes_q, codes_x)):
        assert b0 == b1 and np.array_equal(i0, i1) and np.array_equal(r0, r1), c
    out = os.path.join(HERE, "ldpca_ladders.bin")
    write_compact(out, ladders)
    print("wrote", out, os.path.getsize(out), "bytes;", n_codes, "codes, period", period)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_ladders.py <reference tree>")
    main(sys.argv[1])
