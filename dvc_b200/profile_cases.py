"""Small, self-contained GPU workloads for profiler captures.

    python -m dvc_b200.profile_cases ldpca-cif     # LDPCA ladder on the 11 CIF golden bitplanes
    python -m dvc_b200.profile_cases frame-cif [Q] # one CIF WZ frame (QIndex Q, default 4) through every kernel
    python -m dvc_b200.profile_cases ldpca-micro   # 148 CIF codewords of the LDPCA microbenchmark, one launch

Each case runs once after one warm-up run, so a profiler can skip the warm-up
launches and capture the second instance of a kernel.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def ldpca_cif(ctx):
    g = np.load(os.path.join(ROOT, "tests", "golden", "ldpca_cif.npz"))
    for _ in range(2):
        dec, res, ent = ctx.ldpca_decode(g["lr"], g["acc"], g["crc"])
    assert np.array_equal(res[:, 0], g["rate"])


def frame_cif(ctx, q=4):
    from . import bitstream as bs, decoder, encoder, synth
    ori, key = synth.make_sequence("cif", 3, 101)
    st = bs.parse_wz(encoder.encode_sequence(ori, 2, q))
    m, b, e = bs.sequence_order(st.n_frames, st.gop)[0]
    it = decoder.frame_item(st, st.frames[m], key)
    for _ in range(2):
        ctx.decode_wz_frames([it])


def ldpca_micro(ctx, count=148):
    from . import ldpca_bench as lb
    lr, acc, crc, x = lb.make_codewords(6336, count, 5)
    for _ in range(2):
        dec, res, ent = ctx.ldpca_decode(lr, acc, crc)
    assert np.array_equal(dec, x)
    print("bp block-iterations per launch", int(res[:, 3].sum()))


CASES = {"ldpca-cif": ldpca_cif, "frame-cif": frame_cif, "ldpca-micro": ldpca_micro}


def main():
    from . import native
    name = sys.argv[1] if len(sys.argv) > 1 else "ldpca-cif"
    ctx = native.Context(0)
    CASES[name](ctx, *[int(a) for a in sys.argv[2:]])
    ctx.close()
    print("case", name, "done")


if __name__ == "__main__":
    main()
