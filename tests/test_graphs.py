"""CUDA-graph replay of the sweeps' angles (config cuda_graphs = 1, the default) against host
launches of every kernel (cuda_graphs = 0): the same kernels in the same order, so picks and
scores must be bit-identical, also after a size change forces a new capture, for the hand-tuned
and the generic correlation kernels."""
import numpy as np
import pytest

import gisspa
import synth
from parity import small_case

pytestmark = pytest.mark.gpu


def _searchers(cfg, tmpl):
    out = []
    for g in (1, 0):
        s = gisspa.Searcher(cfg.copy(cuda_graphs=g))
        s.set_templates(tmpl)
        out.append(s)
    return out


# norm_l336_w4: a window size without hand-tuned kernels (the generic column / row kernels; its
# chunk scan needs more than the default 48 KB of shared memory)
@pytest.mark.parametrize("name", ["norm_l256_w9", "norm_l336_w4"])
@pytest.mark.parametrize("mode", ["chunk", "topk"])
def test_graph_replay_bit_identical(name, mode):
    img, tmpl, ctf, cfg = small_case(name)
    cfg = cfg.copy(phistep=30.0)  # 12 angles: 1 from the host, 11 replays per sweep
    if mode == "topk":
        cfg = cfg.copy(pick_mode=gisspa.PICK_TOPK, topk=40, exclusion_radius=20.0, threshold=2.0)
    sg, se = _searchers(cfg, tmpl)
    other = synth.make_case(shape=(700, 900), n_particles=12, snr=0.1, n_templates=tmpl.shape[0],
                            tsize=tmpl.shape[1], seed=5)
    for image in (img, other.image, img):  # new shape -> reallocation -> new capture, then back
        pg, pe = sg.search(image, ctf), se.search(image, ctf)
        assert len(pg) == len(pe) and len(pe) > 0
        assert pg.tobytes() == pe.tobytes()
        stg, ste = sg.stats(), se.stats()
        assert stg.pairs == ste.pairs
        # replays count their captured kernels; the graph path adds one angle-select per replay
        assert stg.kernel_launches >= ste.kernel_launches
        assert stg.graph_replays > 0 and ste.graph_replays == 0
