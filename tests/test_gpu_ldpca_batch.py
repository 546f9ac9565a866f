"""GPU parity of the batched LDPCA form (dvc_ldpca_decode_batch): codewords of
both lengths, each from its own start level, in one persistent launch.

* The batched workload (dvc_b200.ldpca_bench: 8192 codewords, QCIF and CIF
  interleaved, seeded flip probabilities and start levels) against the
  reference's LdpcaDecoder, codeword by codeword: rate, accepted code and
  decoded bits (a digest per codeword).
* With the entropy bound choosing the start, the reference's known-answer
  vectors and full-rate codewords, and equality with the frame path's ladder
  kernel (dvc_ldpca_decode) in every output, BP iteration count included.
* The 100-iteration variant (the reference stops at 50) against the oracle with
  the same cap.
"""
import hashlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _digest64(a):
    return int.from_bytes(hashlib.blake2b(np.ascontiguousarray(a).tobytes(), digest_size=8).digest(), "little")


def _interleave(parts):
    """Codewords of several (lengths, lr, acc, crc, start) groups, alternating, and where each came from."""
    order = []
    for g, p in enumerate(parts):
        order += [(i * len(parts) + g, g, i) for i in range(len(p[1]))]
    order.sort()
    n = np.array([parts[g][0] for _, g, _ in order], np.int32)
    lr = np.concatenate([parts[g][1][i] for _, g, i in order])
    acc = np.concatenate([parts[g][2][i] for _, g, i in order])
    crc = np.array([parts[g][3][i] for _, g, i in order], np.uint8)
    start = None if parts[0][4] is None else np.array([parts[g][4][i] for _, g, i in order], np.int32)
    return n, lr, acc, crc, start, [(g, i) for _, g, i in order]


def _split(dec, n):
    off = np.concatenate([[0], np.cumsum(n)])
    return [dec[off[k]:off[k + 1]] for k in range(len(n))]


def test_batch_workload_matches_reference_per_codeword(gpu_ctx, golden_dir):
    from dvc_b200 import ldpca_bench as lb
    g = np.load(os.path.join(golden_dir, "ldpca_batch.npz"))
    half, seed = int(g["count"]) // 2, int(g["seed"])
    parts = []
    for n in (1584, 6336):
        lr, acc, crc, x = lb.make_codewords(n, half, seed + n)
        assert [_digest64(lr), _digest64(acc), _digest64(crc)] == [int(v) for v in g["n%d_input_hash" % n]]
        st = lb.seeded_starts(n, half, seed + n)
        assert np.array_equal(st, g["n%d_start" % n])
        parts.append((n, lr, acc, crc, st))
    n, lr, acc, crc, start, where = _interleave(parts)
    dec, res, ent, work, ms = gpu_ctx.ldpca_decode_batch(n, lr, acc, crc, start, max_iter=50)
    decs = _split(dec, n)
    bad = []
    for k, (grp, i) in enumerate(where):
        L = (1584, 6336)[grp]
        if (res[k, 1] != g["n%d_start" % L][i] or res[k, 0] != g["n%d_rate" % L][i]
                or res[k, 2] != g["n%d_accepted" % L][i] or _digest64(decs[k]) != int(g["n%d_decoded_hash" % L][i])):
            bad.append(k)
    assert not bad, "%d of %d codewords differ from the reference, first %s" % (len(bad), len(n), bad[:8])
    assert work >= int(res[:, 3].sum())


def _kat_parts(golden_dir):
    parts = []
    for name in ("qcif", "cif"):
        g = np.load(os.path.join(golden_dir, "ldpca_%s.npz" % name))
        parts.append((int(g["n"]), g["lr"], g["acc"], g["crc"], None))
    return parts


def test_batch_with_entropy_start_matches_reference_and_frame_kernel(gpu_ctx, golden_dir):
    parts = _kat_parts(golden_dir)
    n, lr, acc, crc, _, where = _interleave(parts)
    dec, res, ent, work, ms = gpu_ctx.ldpca_decode_batch(n, lr, acc, crc, None, max_iter=50)
    decs = _split(dec, n)
    for name, (L, plr, pacc, pcrc, _) in zip(("qcif", "cif"), parts):
        g = np.load(os.path.join(golden_dir, "ldpca_%s.npz" % name))
        want_dec, want_res, want_ent = gpu_ctx.ldpca_decode(plr, pacc, pcrc, max_iter=50)
        ks = [k for k, (grp, _) in enumerate(where) if (1584, 6336)[grp] == L]
        idx = [where[k][1] for k in ks]
        assert np.array_equal(res[ks], want_res[idx]), name
        assert np.array_equal(ent[ks].view(np.uint32), g["entropy"][idx].view(np.uint32)), name
        assert np.array_equal(res[ks, 0], g["rate"][idx]), name
        for k, i in zip(ks, idx):
            assert np.array_equal(decs[k], g["decoded"][i]), (name, i)


def test_batch_full_rate_and_given_full_rate_start(gpu_ctx, golden_dir):
    g = np.load(os.path.join(golden_dir, "ldpca_fullrate.npz"))
    cnt = int(g["count"])
    n = np.array([int(g["c%d_n" % k]) for k in range(cnt)], np.int32)
    lr = np.concatenate([g["c%d_lr" % k] for k in range(cnt)])
    acc = np.concatenate([g["c%d_acc" % k] for k in range(cnt)])
    crc = np.array([g["c%d_crc" % k] for k in range(cnt)], np.uint8)
    for start in (None, np.full(cnt, 64, np.int32)):
        dec, res, ent, work, ms = gpu_ctx.ldpca_decode_batch(n, lr, acc, crc, start, max_iter=50)
        decs = _split(dec, n)
        for k in range(cnt):
            assert res[k, 0] == n[k] + 8 and res[k, 2] == 64
            assert np.array_equal(decs[k], g["c%d_decoded" % k])
        if start is None:
            assert np.array_equal(ent, np.array([g["c%d_entropy" % k] for k in range(cnt)], np.float32))
        else:
            assert np.all(res[:, 3] == 0) and work == 0


def test_batch_hundred_iterations_matches_oracle(gpu_ctx):
    """The longer variant: BP runs up to 100 iterations per ladder code; the
    oracle restatement with the same cap decodes the same codewords."""
    from dvc_b200 import ldpca_bench as lb
    from oracle import pyoracle as po
    parts = []
    for n, cnt in ((1584, 12), (6336, 3)):
        lr, acc, crc, x = lb.make_codewords(n, cnt, 77 + n)
        parts.append((n, lr, acc, crc, lb.seeded_starts(n, cnt, 77 + n)))
    n, lr, acc, crc, start, where = _interleave(parts)
    dec, res, ent, work, ms = gpu_ctx.ldpca_decode_batch(n, lr, acc, crc, start, max_iter=100)
    decs = _split(dec, n)
    for k, (grp, i) in enumerate(where):
        L, plr, pacc, pcrc, pst = parts[grp]
        rates = lb.code_rates(L)
        bits = np.unpackbits(pacc[i], bitorder="big")[:L]
        odec, orate, ostart, oacc, _ = po.ldpca_decode(po.OracleLadder.get(L), plr[i], bits, int(pcrc[i]),
                                                       float(rates[pst[i]]), max_iter=100)
        assert (res[k, 0], res[k, 1], res[k, 2]) == (orate, ostart, oacc)
        assert np.array_equal(decs[k], odec)
