"""GPU: the serving loop (continuous batching, HBM-budget admission, warm
stroke edits).  Every result, cold or warm-edited, 2D or 3D, must be
bit-identical to the CPU oracle's max-flow and canonical cut of the same graph
(and so to the plain solver's), whether the request ran alone or shared its
launches with others."""
import threading
import time

import numpy as np
import pytest

import jfcut
import oracle
import synthetic

pytestmark = pytest.mark.gpu

MODEL5 = dict(lambda_n=100, z_weight_pct=100, lambda_t=10, k_fg=5, k_bg=5, seed_cap=1000000, kmeans_iters=32)
MODEL2 = dict(MODEL5, k_fg=2, k_bg=2)


def make_requests(seed, n2d, n3d, lo=24, hi=400):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n2d):
        w, h = (int(v) for v in rng.integers(lo, hi, 2))
        if i % 2 == 0:
            img, seeds = synthetic.rgb_ellipses(w, h, seed=seed * 1000 + i)
            reqs.append((img, seeds, jfcut.PIX_RGB8, MODEL5))
        else:
            img, seeds = synthetic.gray_ellipse(w, h, seed=seed * 1000 + i)
            reqs.append((img, seeds, jfcut.PIX_GRAY8, MODEL2))
    for j in range(n3d):
        w, h, d = (int(v) for v in rng.integers(16, 48, 3))
        img, seeds = synthetic.i16_phantom(w, h, d, seed=seed * 1000 + 500 + j)
        reqs.append((img, seeds, jfcut.PIX_I16, MODEL2))
    return reqs


def strokes(shape, seed, count):
    rng = np.random.default_rng(seed)
    n = int(np.prod(shape))
    out = []
    for k in range(count):
        m = max(1, int(n * rng.uniform(0.001, 0.02)))
        out.append(synthetic.stroke(shape, seed=seed * 10 + k, n=m, label=1 + (k % 2)))
    return out


def cpu_oracle(img, seeds, pf, model, edits=()):
    """The CPU oracle on the graph a session holds after `edits`: colour
    models fit on the original seeds, t-links from the edited seeds; returns
    the full int64 max-flow and the canonical source side."""
    cur = seeds.ravel().copy()
    for idx, ns in edits:
        cur[idx] = ns
    e, caps, sink = oracle.build_graph(img, seeds, pf, model, seeds_tl=cur)
    _, ef, _, lab = oracle.maxflow(seeds.shape, e, caps)
    return sink + int(np.minimum(ef.astype(np.int64), 0).sum()), lab.reshape(seeds.shape)


def plain(ctx, img, seeds, pf, model, edits=()):
    """Cold reference: build, apply every edit so far (the colour model stays
    the one of the original seeds, as on the warm path), solve from scratch
    with the plain solver; both it and the server are held to the CPU oracle."""
    g = jfcut.Graph(ctx, seeds.shape)
    g.build_from_image(img, seeds, pf, model)
    for idx, ns in edits:
        g.edit_seeds(idx, ns)
    g.solve()
    out = g.flow(), g.labels().copy()
    g.close()
    want = cpu_oracle(img, seeds, pf, model, edits)
    assert out[0] == want[0]
    assert np.array_equal(out[1], want[1])
    return want


def test_mix_equals_alone_with_warm_edits(ctx):
    reqs = make_requests(7, 10, 3)
    srv = jfcut.Server(ctx, 0, max_slots=64)
    try:
        sids = [srv.submit(img, seeds, pf, model) for img, seeds, pf, model in reqs]
        for sid, (img, seeds, pf, model) in zip(sids, reqs):
            info = srv.wait(sid)
            assert info.status == 0 and info.warm == 0
            flow, lab = plain(ctx, img, seeds, pf, model)
            assert info.flow == flow
            assert np.array_equal(srv.labels(sid, seeds.shape), lab)
        # every session gets 1-3 stroke edits, all in flight together
        plan = [strokes(seeds.shape, 40 + i, 1 + i % 3) for i, (_, seeds, _, _) in enumerate(reqs)]
        for sid, ed in zip(sids, plan):
            for idx, ns in ed:
                srv.edit(sid, idx, ns)
        for sid, ed, (img, seeds, pf, model) in zip(sids, plan, reqs):
            info = srv.wait(sid)
            assert info.status == 0 and info.warm == 1
            flow, lab = plain(ctx, img, seeds, pf, model, ed)
            assert info.flow == flow
            assert np.array_equal(srv.labels(sid, seeds.shape), lab)
        st = srv.stats()
        assert st["peak_solving"] > 1           # requests shared launches
        assert st["peak_used"] <= st["budget"]
        assert st["requests_done"] == len(reqs) + sum(len(e) for e in plan)
    finally:
        srv.close()


def test_alone_in_server_equals_mix(ctx):
    """The same request served alone and inside a mix gives the same result."""
    reqs = make_requests(9, 6, 1)
    alone = []
    for img, seeds, pf, model in reqs:
        srv = jfcut.Server(ctx, 0, max_slots=1)
        sid = srv.submit(img, seeds, pf, model)
        info = srv.wait(sid)
        alone.append((info.flow, srv.labels(sid, seeds.shape)))
        srv.close()
        flow, lab = cpu_oracle(img, seeds, pf, model)
        assert alone[-1][0] == flow and np.array_equal(alone[-1][1], lab)
    srv = jfcut.Server(ctx, 0, max_slots=64)
    try:
        sids = [srv.submit(*r) for r in reqs]
        for sid, (img, seeds, pf, model), (flow, lab) in zip(sids, reqs, alone):
            info = srv.wait(sid)
            assert info.status == 0 and info.flow == flow
            assert np.array_equal(srv.labels(sid, seeds.shape), lab)
    finally:
        srv.close()


def test_budget_admission(ctx):
    reqs = make_requests(11, 8, 0, lo=200, hi=300)
    biggest = max(jfcut.graph_bytes(s.shape) for _, s, _, _ in reqs)
    budget = 3 * biggest   # roughly one session's state + build temporaries at a time
    srv = jfcut.Server(ctx, budget, max_slots=64)
    try:
        # a session that can never fit is refused up front
        img, seeds = synthetic.rgb_ellipses(2000, 2000, seed=1)
        with pytest.raises(jfcut.JfcError) as ex:
            srv.submit(img, seeds, jfcut.PIX_RGB8, MODEL5)
        assert ex.value.code == jfcut.ERR_OOM
        sids = [srv.submit(*r) for r in reqs]
        for sid, (img, seeds, pf, model) in zip(sids, reqs):
            info = srv.wait(sid)
            assert info.status == 0
            flow, lab = plain(ctx, img, seeds, pf, model)
            assert info.flow == flow
            # resident sessions hold the budget: close to admit the next ones
            srv.close_session(sid)
        st = srv.stats()
        assert st["peak_used"] <= budget
    finally:
        srv.close()


def test_arrivals_while_solving(ctx):
    """Requests submitted from another thread while earlier ones are on the
    device join the running solving set."""
    reqs = make_requests(13, 12, 2, lo=100, hi=600)
    srv = jfcut.Server(ctx, 0, max_slots=64)
    sids = [None] * len(reqs)
    rng = np.random.default_rng(5)
    gaps = rng.exponential(0.002, len(reqs))

    def client():
        for i, r in enumerate(reqs):
            time.sleep(float(gaps[i]))
            sids[i] = srv.submit(*r)

    try:
        t = threading.Thread(target=client)
        t.start()
        t.join()
        for sid, (img, seeds, pf, model) in zip(sids, reqs):
            info = srv.wait(sid)
            assert info.status == 0
            assert info.ms_total >= info.ms_solve >= 0 and info.ms_queue >= 0
            flow, lab = plain(ctx, img, seeds, pf, model)
            assert info.flow == flow
            assert np.array_equal(srv.labels(sid, seeds.shape), lab)
    finally:
        srv.close()


def test_cancel_and_close(ctx):
    reqs = make_requests(17, 4, 0, lo=300, hi=500)
    srv = jfcut.Server(ctx, 0, max_slots=64)
    try:
        sids = [srv.submit(*r) for r in reqs]
        srv.cancel(sids[0])
        info = srv.wait(sids[0])
        assert info.status in (jfcut.OK, jfcut.ERR_CANCELLED)
        for sid, (img, seeds, pf, model) in zip(sids[1:], reqs[1:]):
            i1 = srv.wait(sid)
            assert i1.status == 0
            assert i1.flow == cpu_oracle(img, seeds, pf, model)[0]
        # a cancelled session that has a graph can still be edited and re-solved
        img, seeds, pf, model = reqs[0]
        ed = strokes(seeds.shape, 99, 1)
        if info.status == jfcut.ERR_CANCELLED:
            try:
                srv.edit(sids[0], *ed[0])
                info2 = srv.wait(sids[0])
                if info2.status == 0:
                    flow, lab = cpu_oracle(img, seeds, pf, model, ed)
                    assert info2.flow == flow
                    assert np.array_equal(srv.labels(sids[0], seeds.shape), lab)
            except jfcut.JfcError as e:
                assert e.code == jfcut.ERR_STATE    # cancelled before its build
        for sid in sids:
            srv.close_session(sid)
        with pytest.raises(jfcut.JfcError):
            srv.wait(sids[1])
        deadline = time.time() + 10
        while srv.stats()["sessions"] and time.time() < deadline:
            time.sleep(0.01)
        st = srv.stats()
        assert st["sessions"] == 0 and st["used"] == 0
    finally:
        srv.close()


def test_close_right_after_result_while_others_solve(ctx):
    """A session closed the moment its last result arrives, while it is still
    held by its lane and other sessions keep solving, is freed once (no use
    after free, no leak); results stay the oracle's."""
    reqs = make_requests(23, 20, 4, lo=40, hi=260)
    srv = jfcut.Server(ctx, 0, max_slots=64)
    results, errors = {}, []
    lock = threading.Lock()

    def client(i):
        img, seeds, pf, model = reqs[i]
        try:
            sid = srv.submit(img, seeds, pf, model)
            info = srv.wait(sid, 120000)
            ed = strokes(seeds.shape, 300 + i, 1 + i % 3)
            for idx, ns in ed:
                srv.edit(sid, idx, ns)
                info = srv.wait(sid, 120000)
            srv.close_session(sid)          # right after the result
            with lock:
                results[i] = (info.status, info.flow, ed)
        except Exception as ex:
            with lock:
                errors.append(repr(ex))

    try:
        threads = [threading.Thread(target=client, args=(i,)) for i in range(len(reqs))]
        for t in threads:
            t.start()
            time.sleep(0.002)
        for t in threads:
            t.join()
        assert not errors, errors[:3]
        for i, (status, flow, ed) in results.items():
            img, seeds, pf, model = reqs[i]
            assert status == 0
            assert flow == cpu_oracle(img, seeds, pf, model, ed)[0]
        deadline = time.time() + 20
        while srv.stats()["sessions"] and time.time() < deadline:
            time.sleep(0.01)
        st = srv.stats()
        assert st["sessions"] == 0 and st["used"] == 0
    finally:
        srv.close()
