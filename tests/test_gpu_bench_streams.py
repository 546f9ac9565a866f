"""GPU parity on the benchmark's own configuration: the first GOP of every
(GOP, QIndex) stream that bench.py times (CIF, the bench's 65-frame sequence
and seed, SkipBlock 1, IntraMode 1, DeblockingFilter 1, IntraQP 30), against the
reference decoder's output on the same bitstreams.

Each stream comes twice: encoded by the reference encoder (the bitstreams are
stored in the fixture) and by dvc_b200.encoder, which produces the streams the
bench decodes (regenerated here and checked against the fixture's digest; the
encoder codes each GOP from that GOP's frames only, so the first GOP of a
short sequence is the first GOP of the bench's stream).  GOP 4 covers both
dependent levels: frame 2 first, then frames 1 and 3 from its decoded output.
"""
import hashlib
import os

import numpy as np
import pytest

import bench
from dvc_b200 import bitstream as bs
from dvc_b200 import decoder, synth

pytestmark = pytest.mark.gpu

CASES = [(enc, g, q) for enc in ("ref", "own") for g in bench.GOPS for q in bench.QS]


def _digest64(a):
    return int.from_bytes(hashlib.blake2b(np.ascontiguousarray(a).tobytes(), digest_size=8).digest(), "little")


@pytest.fixture(scope="module")
def pin(golden_dir):
    return np.load(os.path.join(golden_dir, "bench_first_gops.npz"))


@pytest.fixture(scope="module")
def frames65():
    return synth.make_sequence(bench.KIND, bench.N_FRAMES, bench.SEED)


@pytest.mark.parametrize("enc,g,q", CASES)
def test_bench_first_gop_matches_reference(gpu_ctx, pin, frames65, enc, g, q):
    p = "%s_g%d_q%d_" % (enc, g, q)
    ori, key = frames65[0][:g + 1], frames65[1][:g + 1]
    if enc == "ref":
        wz, ib = pin[p + "wz"].tobytes(), pin[p + "intra"].tobytes()
    else:
        from dvc_b200 import encoder
        wz, ib = encoder.encode_sequence_intra(ori, g, q, bench.INTRA_QP, 1, 1, 1)
    assert [_digest64(np.frombuffer(wz, np.uint8)), _digest64(np.frombuffer(ib, np.uint8))] == \
        [int(x) for x in pin[p + "stream_hash"]], "the bitstream is not the one the reference decoded"
    st = bs.parse_wz(wz)
    ties0 = gpu_ctx.recon_near_ties()
    res = decoder.decode_sequence(gpu_ctx, st, key, ori, intra_bitstream=ib if len(ib) else None)
    assert gpu_ctx.recon_near_ties() == ties0, "a reconstruction step sat near a rounding tie"
    for k, f in enumerate(pin[p + "frames"]):
        f = int(f)
        assert hashlib.sha256(res["recon"][f].tobytes()).hexdigest() == str(pin[p + "y_sha"][k]), f"frame {f} Y"
        assert res["bits"][f] == pin[p + "bits"][k], f"frame {f} bits"
        assert "%.2f" % res["psnr"][f] == "%.2f" % pin[p + "psnr"][k], f"frame {f} PSNR"
    order = [int(m) for m in pin[p + "order"]]
    start = np.concatenate([res["planes"][m][:, 1] for m in order])
    acc = np.concatenate([res["planes"][m][:, 2] for m in order])
    ent = np.concatenate([res["entropy"][m] for m in order]).astype(np.float32)
    assert np.array_equal(start, pin[p + "ld_start"])
    assert np.array_equal(acc, pin[p + "ld_accepted"])
    assert np.array_equal(ent.view(np.uint32), pin[p + "ld_entropy"].view(np.uint32))
