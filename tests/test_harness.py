"""CPU: the workloads of the serving and large-GOP runs are built as intended
(no GPU: only the encoding, parsing and dependency bookkeeping)."""
import numpy as np

from dvc_b200 import bitstream as bs, encoder, serve_bench, stress_bench, synth


def test_mixed_serving_requests_follow_their_references():
    reqs = serve_bench.build(5)
    kinds = {}
    for k, it in enumerate(reqs):
        kinds.setdefault(it["_stream"], it["_kind"])
        for d in it["_deps"]:
            # a reference is an earlier request of the same stream, and one of the frame's two references
            assert d < k and reqs[d]["_stream"] == it["_stream"]
            assert reqs[d]["_frame"] in (it["past_idx"], it["future_idx"])
    assert sum(1 for v in kinds.values() if v == "qcif") == 48 and sum(1 for v in kinds.values() if v == "cif") == 16
    # round-robin interleaving: the first 64 requests come from 64 different streams
    assert len({it["_stream"] for it in reqs[:64]}) == 64


def test_gop8_session_items_chain_three_levels():
    ori, key = synth.make_sequence("cif_fast", 9, 3000)
    wz, ib = encoder.encode_sequence_intra(ori, 8, 4, 30, 1, 1, 1)
    st = bs.parse_wz(wz)
    items, levels = stress_bench.session_items(st, key, ib)
    assert levels == 3 and len(items) == 7
    for k, it in enumerate(items):
        for name in ("past_from", "future_from"):
            ref = it.get(name)
            if ref is not None:
                assert ref < k and it[name.replace("_from", "")] is None
    # frames with intra blocks start from their host-decoded intra pixels
    with_intra = [it for it in items if it["intra_mode"]]
    assert with_intra and all(not np.array_equal(it["recon"], key[it["cur_idx"]]) for it in with_intra)
