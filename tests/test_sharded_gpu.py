"""One micrograph across ranks on one B200: two ranks emulated one after the other (two
handles on cuda:0; no kernel waits on another), their exported states merged with torch on
the device, against the unsharded search."""
import numpy as np
import pytest

import gisspa
from parity import small_case
from sharded import angle_ranges, shard_finish, shard_sweep1

pytestmark = pytest.mark.gpu


def _merge(states):
    import torch
    s0 = states[0]
    for st in states[1:]:
        s0.sum += st.sum
        s0.sum_sq += st.sum_sq
        if s0.key is not None:
            s0.key.copy_(torch.maximum(s0.key, st.key))
    for st in states[1:]:
        st.sum.copy_(s0.sum)
        st.sum_sq.copy_(s0.sum_sq)
        if st.key is not None:
            st.key.copy_(s0.key)


@pytest.mark.parametrize("mode,world", [("topk", 2), ("topk", 3), ("chunk", 2)])
def test_sharded_equals_single(mode, world):
    import torch
    img, tmpl, ctf, cfg = small_case("norm_l256_w9")
    if mode == "topk":
        cfg = cfg.copy(pick_mode=gisspa.PICK_TOPK, topk=40, exclusion_radius=20.0, threshold=2.0)
    single = gisspa.Searcher(cfg)
    single.set_templates(tmpl)
    ref = single.search(img, ctf)
    assert len(ref) > 0
    ranks = [gisspa.Searcher(cfg) for _ in range(world)]
    for s in ranks:
        s.set_templates(tmpl)
    runs = [shard_sweep1(s, img, ctf, r, world, "cuda:0") for r, s in enumerate(ranks)]
    assert [x[1] for x in runs] == angle_ranges(runs[0][0].n_angles, world)
    _merge([x[2] for x in runs])
    out = [shard_finish(s, info, rng, st) for s, (info, rng, st) in zip(ranks, runs)]
    key = ["x", "y", "template_id", "angle_index", "window"]
    if mode == "topk":
        for o in out:  # every rank returns the merged list
            assert len(o) == len(ref)
            for f in key:
                assert np.array_equal(o[f], ref[f]), f
            assert np.allclose(o["score"], ref["score"], rtol=1e-6, atol=1e-6)
    else:
        cat = np.concatenate(out)
        assert len(cat) == len(ref)
        for f in key + ["chunk"]:
            assert np.array_equal(cat[f], ref[f]), f
        assert np.allclose(cat["score"], ref["score"], rtol=1e-6, atol=1e-6)


def test_shard_calls_out_of_order_are_rejected():
    img, tmpl, ctf, cfg = small_case("norm_l256_w9")
    s = gisspa.Searcher(cfg)
    s.set_templates(tmpl)
    with pytest.raises(gisspa.GisspaError):
        s.shard_picks()
    info = s.shard_begin(img, ctf)
    with pytest.raises(gisspa.GisspaError):
        s.shard_sweep(2, 0, 1)       # sweep 2 needs the merged statistics
    with pytest.raises(gisspa.GisspaError):
        s.shard_sweep(1, 0, info.n_angles + 1)
