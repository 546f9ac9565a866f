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
