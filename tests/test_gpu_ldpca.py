"""GPU parity: the device LDPCA ladder against the reference's golden vectors."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["qcif", "cif"])
def test_ldpca_kernel_matches_reference(gpu_ctx, golden_dir, name):
    g = np.load(os.path.join(golden_dir, f"ldpca_{name}.npz"))
    dec, res, ent = gpu_ctx.ldpca_decode(g["lr"], g["acc"], g["crc"], max_iter=50)
    assert np.array_equal(ent.view(np.uint32), g["entropy"].view(np.uint32))
    assert np.array_equal(res[:, 0], g["rate"])
    assert np.array_equal(dec, g["decoded"])


def test_reference_shaped_ldpca_call(gpu_ctx, golden_dir):
    g = np.load(os.path.join(golden_dir, "ldpca_qcif.npz"))
    n = int(g["n"])
    for i in range(3):
        bits = np.unpackbits(g["acc"][i], bitorder="big")[:n]
        dec, rate, llr = gpu_ctx.LdpcaDecoder(g["lr"][i], bits, int(g["crc"][i]), float(g["entropy"][i]))
        assert rate == g["rate"][i]
        assert np.array_equal(dec, g["decoded"][i])
        assert np.array_equal(llr.view(np.uint32), g["llr"][i].view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1584, 6336])
def test_device_encoder_matches_host_encoder_and_round_trips(gpu_ctx, n):
    """dvc_ldpca_encode equals the bitstream encoder's accumulated syndromes and
    CRCs bit for bit, and its output decodes back to the source."""
    from dvc_b200 import encoder, ldpca_bench
    lr, acc_host, crc_host, x = ldpca_bench.make_codewords(n, 24, 3 + n)
    acc_dev, crc_dev = gpu_ctx.ldpca_encode(x)
    assert np.array_equal(acc_dev, acc_host)
    assert np.array_equal(crc_dev, crc_host)
    dec, res, ent = gpu_ctx.ldpca_decode(lr, acc_dev, crc_dev)
    assert np.array_equal(dec, x)


@pytest.mark.parametrize("k", range(6))
def test_full_rate_inverse_matches_reference(gpu_ctx, golden_dir, k):
    """Codewords no ladder code below full rate decodes (QCIF and CIF): the
    reference ends at its GF(2) inverse (LdpcaDecoder.cpp:695-716), rate N + 8;
    the device ladder must reach the same code and the same decoded bits, with
    the entropy bound (which picks the first code) equal in bits."""
    g = np.load(os.path.join(golden_dir, "ldpca_fullrate.npz"))
    n = int(g["c%d_n" % k])
    lr = g["c%d_lr" % k][None]
    acc = g["c%d_acc" % k][None]
    crc = np.array([g["c%d_crc" % k]], np.uint8)
    dec, res, ent = gpu_ctx.ldpca_decode(lr, acc, crc, max_iter=50)
    assert np.float32(ent[0]).view(np.uint32) == np.float32(g["c%d_entropy" % k]).view(np.uint32)
    assert res[0, 0] == int(g["c%d_rate" % k]) == n + 8
    assert res[0, 2] == 64
    assert np.array_equal(dec[0], g["c%d_decoded" % k])
