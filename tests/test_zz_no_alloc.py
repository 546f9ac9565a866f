"""GPU: the LDPCA entry point that allocates nothing at call time.

It serves callers that cannot call cudaMalloc while running (it may
synchronise the device, is not allowed under stream capture, and fails when
another framework's pool owns the memory).  The test owns every device buffer
(allocated here with torch), calls dvc_ldpca_decode_noalloc twice in a row
through the C ABI, and checks both results against dvc_ldpca_decode, which
stages its buffers itself.  The comparison is exact: decoded bits, rates,
ladder codes and the entropy bound's bits.  This file is collected last.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["qcif", "cif"])
def test_noalloc_matches_staged_entry_point(gpu_ctx, golden_dir, name):
    import torch
    from dvc_b200 import native
    g = np.load(os.path.join(golden_dir, f"ldpca_{name}.npz"))
    n, count = int(g["n"]), len(g["crc"])
    want_dec, want_res, want_ent = gpu_ctx.ldpca_decode(g["lr"], g["acc"], g["crc"])
    dev = torch.device("cuda", 0)
    lr = torch.from_numpy(np.ascontiguousarray(g["lr"], np.float32)).to(dev)
    acc = torch.from_numpy(np.ascontiguousarray(g["acc"], np.uint8)).to(dev)
    crc = torch.from_numpy(np.ascontiguousarray(g["crc"], np.uint8)).to(dev)
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        dec = torch.full((count, n), 7, dtype=torch.uint8, device=dev)
        res = torch.full((count, 4), -1, dtype=torch.int32, device=dev)
        ent = torch.full((count,), -1.0, dtype=torch.float32, device=dev)
        rc = gpu_ctx.ldpca_decode_noalloc(n, count, lr.data_ptr(), acc.data_ptr(), crc.data_ptr(), dec.data_ptr(),
                                          res.data_ptr(), ent.data_ptr(), 50, stream.cuda_stream)
        assert rc == native.DVC_OK, gpu_ctx.last_error()
        stream.synchronize()
        assert np.array_equal(dec.cpu().numpy(), want_dec), f"call {call}: decoded bits"
        assert np.array_equal(res.cpu().numpy(), want_res), f"call {call}: rate/codes/iterations"
        assert np.array_equal(ent.cpu().numpy().view(np.uint32), want_ent.view(np.uint32)), f"call {call}: entropy"


def test_noalloc_rejects_more_codewords_than_its_scratch(gpu_ctx):
    from dvc_b200 import native
    too_many = 1025
    rc = gpu_ctx.ldpca_decode_noalloc(1584, too_many, 1, 1, 1, 0, 1, 0, 50, 0)
    assert rc == native.DVC_E_ARG
    assert "exceed the limit of 1024" in gpu_ctx.last_error()
