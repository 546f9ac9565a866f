"""The autotuner's measurement on the device: a small batched CIF session decoded
under three launch shapes (threads per LDPCA codeword block, speculative-width
floor, threads per updateSI and forward-search block), each a fresh context;
tune() requires every shape to decode the same frames, rates and ladder codes."""
import os

import numpy as np
import pytest

from dvc_b200 import autotune as at

pytestmark = pytest.mark.gpu


def test_launch_shapes_decode_identically():
    from dvc_b200 import native
    items = at.workload(n_streams=2, n_frames=9)
    base = at.defaults()
    settings = [dict(base), dict(base, **{at.ENV_THREADS: "512", at.ENV_FLOOR: "1", at.ENV_SI: "64",
                                          at.ENV_FME: "512"}),
                dict(base, **{at.ENV_FLOOR: "32", at.ENV_SI: "256", at.ENV_FME: "128"})]

    def measure(setting):
        ctx = native.Context(0)
        try:
            ses = ctx.session(items, max_batch=4, streams=2)
            try:
                ms = [ses.run() for _ in range(3)]  # direct, captured, replayed
                return ms, [ses.frame(i) for i in range(len(items))]
            finally:
                ses.close()
        finally:
            ctx.close()

    before = {k: os.environ.get(k) for k in at.ENV_ALL}
    best, results = at.tune(measure, settings)
    assert len(results) == 3 and best["setting"] in settings
    assert all(np.isfinite(r["ms"]).all() and min(r["ms"]) > 0 for r in results)
    assert {k: os.environ.get(k) for k in at.ENV_ALL} == before
