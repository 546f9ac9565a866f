"""Small, self-contained GPU workloads for profiler captures (not a test module).

    python tests/profile_cases.py ldpca-cif     # LDPCA ladder on the CIF golden bitplanes
    python tests/profile_cases.py frame-cif [Q] # one CIF WZ frame (QIndex Q, default 4) through every kernel
    python tests/profile_cases.py frame-cif-batch [Q] # 16 CIF WZ frames as one batch (one cohort of the bench)
    python tests/profile_cases.py ldpca-micro   # 148 CIF codewords of the LDPCA microbenchmark, one launch
    python tests/profile_cases.py ldpca-batch [N] # N codewords (default 1024) of the batched workload, one launch
    python tests/profile_cases.py bench-step    # one step of bench.py's batched session (640 CIF WZ frames)

Each case runs once after one warm-up run, so a profiler can skip the warm-up
launches and capture the second instance of a kernel; bench-step runs once,
eagerly (every launch of one step, about 6,100).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def ldpca_cif(ctx):
    g = np.load(os.path.join(ROOT, "tests", "golden", "ldpca_cif.npz"))
    for _ in range(2):
        dec, res, ent = ctx.ldpca_decode(g["lr"], g["acc"], g["crc"])
    assert np.array_equal(res[:, 0], g["rate"])


def frame_cif(ctx, q=4):
    from dvc_b200 import bitstream as bs, decoder, encoder, synth
    ori, key = synth.make_sequence("cif", 3, 101)
    st = bs.parse_wz(encoder.encode_sequence(ori, 2, q))
    m, b, e = bs.sequence_order(st.n_frames, st.gop)[0]
    it = decoder.frame_item(st, st.frames[m], key)
    for _ in range(2):
        ctx.decode_wz_frames([it])


def frame_cif_batch(ctx, q=4):
    """16 independent CIF WZ frames (a 33-frame GOP-2 sequence) as one batch:
    the grids of the batched decode (one cohort of the bench)."""
    from dvc_b200 import bitstream as bs, decoder, encoder, synth
    ori, key = synth.make_sequence("cif", 33, 102)
    st = bs.parse_wz(encoder.encode_sequence(ori, 2, q))
    its = [decoder.frame_item(st, st.frames[m], key) for (m, b, e) in bs.sequence_order(st.n_frames, st.gop)]
    for _ in range(2):
        ctx.decode_wz_frames(its)


def ldpca_micro(ctx, count=148):
    from dvc_b200 import ldpca_bench as lb
    lr, acc, crc, x = lb.make_codewords(6336, count, 5)
    for _ in range(2):
        dec, res, ent = ctx.ldpca_decode(lr, acc, crc)
    assert np.array_equal(dec, x)
    print("bp block-iterations per launch", int(res[:, 3].sum()))


def ldpca_batch(ctx, count=1024):
    from dvc_b200 import ldpca_bench as lb
    n, lr, acc, crc, start, src, where = lb.interleaved(count, 11)
    for _ in range(2):
        dec, res, ent, work, ms = ctx.ldpca_decode_batch(n, lr, acc, crc, start, 50)
    print("codewords", count, "kernel ms", ms, "bp iterations", work)


def bench_step(ctx):
    """The batched session of bench.py's workload (16 streams of 16-frame
    batches), one eager run: the kernels of one timed step."""
    import bench
    ori, key, streams, intra_bs = bench.workload()
    its, lev, src = bench.items(streams, key, bench.intra_starts(streams, intra_bs, key))
    ses = ctx.session(its, max_batch=16, streams=16)
    print("step ms", ses.run())
    ses.close()


CASES = {"ldpca-cif": ldpca_cif, "frame-cif": frame_cif, "frame-cif-batch": frame_cif_batch,
         "ldpca-micro": ldpca_micro, "ldpca-batch": ldpca_batch, "bench-step": bench_step}


def main():
    # one hardware queue per CUDA stream, as bench.py sets it
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    from dvc_b200 import native
    name = sys.argv[1] if len(sys.argv) > 1 else "ldpca-cif"
    ctx = native.Context(0)
    CASES[name](ctx, *[int(a) for a in sys.argv[2:]])
    ctx.close()
    print("case", name, "done")


if __name__ == "__main__":
    main()
