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
