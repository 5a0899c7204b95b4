"""The batched workload at its stated size, checked against the reference's
own CPU solver: 256 independent 2D 4-connected RGB instances with sides drawn
uniformly in [128, 2048] (the bench's seeds), solved as one batch with the
autotuned schedule; every instance's int64 max-flow and canonical cut must
equal BK 3.03's (benchmark/GridCut/code/BK303, built from the reference
sources under oracle/_ref) on the graph the CPU restatement of the capacity
build makes from the same image — the reference harness's gate is exactly
"solver flow == recorded max-flow" (benchmark/GridCut/bench-BK303.cpp:411-416),
held here per instance, cut included."""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import jfcut
import oracle
from bench import MODEL, SEED, full_flow, make_workload

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def mix(n_inst=256):
    """The bench's batched workload: sides and per-instance seeds."""
    rng = np.random.default_rng(SEED + 256)
    sides = rng.integers(128, 2049, size=(n_inst, 2))
    return [(int(w), int(h), SEED + 5000 + i) for i, (w, h) in enumerate(sides)]


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref (reference CPU solvers) not built")
def test_batched_mix_equals_bk_per_instance(ctx):
    inst = mix()
    inputs = [make_workload(w, h, s) for w, h, s in inst]
    graphs = []
    b = jfcut.Batch(ctx)
    for (w, h, _), (img, seeds) in zip(inst, inputs):
        g = jfcut.Graph(ctx, (h, w))
        g.build_from_image(img, seeds, jfcut.PIX_RGB8, MODEL)
        graphs.append(g)
        b.add(g)
    b.autotune()
    stats = b.solve()
    assert all(st.status == 0 for st in stats)
    got = [(g.flow(), g.labels().ravel()) for g in graphs]
    b.close()
    for g in graphs:
        g.close()

    # CPU side: the same graphs from the CPU build (parallel inside), then BK
    # per instance on every host thread (each call is single-threaded)
    built = [oracle.build_graph(img, seeds, 1, MODEL) for img, seeds in inputs]

    def bk(k):
        (w, h, _), (e, caps, sink) = inst[k], built[k]
        f, lab, _ = oracle.bk_maxflow((h, w), e, caps, want_labels=True)
        return full_flow(e, f, sink), lab

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        want = list(pool.map(bk, range(len(inst))))
    bad = [k for k in range(len(inst)) if got[k][0] != want[k][0] or not np.array_equal(got[k][1], want[k][1])]
    assert not bad, "instances differing from BK: %s" % bad[:10]
    assert sum(w * h for w, h, _ in inst) > 2.5e8       # the stated size (~3e8 nodes)
