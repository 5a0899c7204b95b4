"""GPU parity: the CUDA path through the C ABI against the CPU oracle (pinned
to the reference), bit-exact on max-flow (int64) and the canonical cut."""
import numpy as np
import pytest

import jfcut
import oracle
import synthetic
from conftest import FIXTURES, SCHEDULES, load_fixture, random_grid, use_schedule

pytestmark = pytest.mark.gpu

MODEL5 = dict(lambda_n=100, z_weight_pct=100, lambda_t=10, k_fg=5, k_bg=5, seed_cap=1000000, kmeans_iters=32)
MODEL2 = dict(MODEL5, k_fg=2, k_bg=2)


def solve_set(ctx, shape, e, caps, offset=0):
    g = jfcut.Graph(ctx, shape)
    g.set(e, caps, offset)
    st = g.solve()
    return g, st


def check_against_oracle(shape, e, caps, flow, labels, offset=0, sink_total=None):
    """offset: sum min(cs, ct) of a graph given in net-excess form; sink_total:
    sum ct of a graph built from an image (full flow = sum ct + sum min(e_final, 0))."""
    f, ef, _, lab = oracle.maxflow(shape, e, caps)
    if sink_total is not None:
        assert flow == sink_total + int(np.minimum(ef.astype(np.int64), 0).sum())
    else:
        assert flow == f + offset
    assert np.array_equal(labels.ravel(), lab)


@pytest.mark.parametrize("name", FIXTURES)
def test_golden_fixtures(ctx, name):
    use_schedule(ctx, "default")
    shape, e, caps, published, ref_obj = load_fixture(name)
    g, st = solve_set(ctx, shape, e, caps)
    assert st.status == 0
    assert g.flow() == published
    lab = g.labels().ravel()
    _, _, _, olab = oracle.maxflow(shape, e, caps)
    assert np.array_equal(lab, olab)
    if ref_obj.sum():
        assert np.array_equal(lab, ref_obj)    # the reference GPU's own cut
    # the final residual state is a valid flow and its reachability is the cut
    ef, r, _ = g.state()
    assert oracle.check_residual(shape, e, caps, ef, r) == 0
    lab2, bad = oracle.cut_from_residual(shape, ef, r)
    assert bad == 0 and np.array_equal(lab2, lab)


# pr_mode 0 with 32x16 tiles runs push-relabel on 32x8 halves of the relabel
# tiles; pr_mode 2 on whole tiles
@pytest.mark.parametrize("tile_rows,local_iters,interval,pr_mode",
                         [(8, 1, 1, 0), (16, 4, 2, 0), (8, 32, 16, 0), (16, 16, 8, 0), (16, 12, 3, 2), (16, 1, 1, 2)])
def test_schedules_agree(ctx, tile_rows, local_iters, interval, pr_mode):
    ctx.set_params(tile_rows=tile_rows, local_iters=local_iters, relabel_interval=interval, pr_mode=pr_mode)
    shape, e, caps, published, _ = load_fixture("sponge")
    g, st = solve_set(ctx, shape, e, caps)
    assert g.flow() == published
    _, _, _, olab = oracle.maxflow(shape, e, caps)
    assert np.array_equal(g.labels().ravel(), olab)


def test_graph_replay_matches_direct_launches(ctx):
    """Relabel cycles replayed from CUDA graphs give the same result as direct
    launches, also when the cached graphs are reused by a second solve."""
    shape, e, caps, published, _ = load_fixture("sponge")
    results = []
    for use_graph in (0, 1, 1):
        ctx.set_params(use_graph=use_graph, relabel_interval=2)
        g, st = solve_set(ctx, shape, e, caps)
        assert g.flow() == published
        assert st.global_relabels > 1
        assert st.used_graph == use_graph
        results.append(g.labels().copy())
        g2 = jfcut.Graph(ctx, shape)   # a second graph on the same context
        g2.set(e, caps)
        assert g2.solve().flow == published
        g2.close()
        g.close()
    assert all(np.array_equal(results[0], r) for r in results[1:])


SHAPES = [(1, 1), (1, 37), (37, 1), (17, 33), (16, 32), (33, 65), (100, 1000), (257, 131),
          (1, 1, 1), (5, 5, 5), (3, 17, 9), (8, 33, 31), (13, 40, 70), (1, 1, 40), (40, 1, 1)]


@pytest.mark.parametrize("sched", SCHEDULES)
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("seed", [0, 1])
def test_random_grids(ctx, shape, seed, sched):
    use_schedule(ctx, sched)
    rng = np.random.default_rng(1000 + seed)
    e, caps = random_grid(shape, rng, cap_max=50 if seed else 1000, density=0.3 if seed else 0.8)
    g, st = solve_set(ctx, shape, e, caps, offset=seed * 7)
    check_against_oracle(shape, e, caps, g.flow(), g.labels(), offset=seed * 7)


@pytest.mark.parametrize("tile_rows,tile_depth", [(16, 4), (16, 2), (16, 1), (8, 2), (8, 1)])
def test_3d_tile_shapes(ctx, tile_rows, tile_depth):
    """Every 3D tile shape (32 x rows/depth x depth) gives the oracle's flow and cut."""
    ctx.set_params(tile_rows=tile_rows, tile_depth=tile_depth)
    for k, shape in enumerate([(5, 5, 5), (3, 17, 9), (13, 40, 70), (20, 33, 18)]):
        rng = np.random.default_rng(500 + k)
        e, caps = random_grid(shape, rng, cap_max=60, density=0.4)
        g, st = solve_set(ctx, shape, e, caps)
        check_against_oracle(shape, e, caps, g.flow(), g.labels())
        g.close()
    img, seeds = synthetic.rgb_video(80, 48, 6, seed=11)
    g = jfcut.Graph(ctx, seeds.shape)
    g.build_from_image(img, seeds, jfcut.PIX_RGB8, dict(MODEL5, z_weight_pct=50))
    e0, c0, _ = g.state()
    g.solve()
    f, _, _, lab = oracle.maxflow(seeds.shape, e0, c0)
    assert np.array_equal(g.labels().ravel(), lab)
    g.close()


@pytest.mark.parametrize("shape,tile_rows,tile_depth", [((64, 96), 16, 4), ((33, 65), 8, 2), ((100, 1000), 16, 4),
                                                      ((700, 1900), 16, 4), ((700, 1900), 8, 2),
                                                      ((700, 1900), 8, 0), ((13, 40, 70), 8, 0),
                                                      ((8, 33, 31), 16, 4), ((13, 40, 70), 8, 2), ((9, 21, 40), 16, 1)])
def test_final_heights_are_exact_distances(ctx, shape, tile_rows, tile_depth):
    """The last global relabel of a solve leaves the exact residual BFS
    distance to the deficits in every node (INF where none is reachable).
    The 700 x 1900 grids keep hundreds of CTAs busy at once on the 2D
    relabel worklist, so concurrent visits of neighbouring tiles happen."""
    ctx.set_params(tile_rows=tile_rows, tile_depth=tile_depth)
    rng = np.random.default_rng(sum(shape))
    e, caps = random_grid(shape, rng, cap_max=40, density=0.35)
    g, st = solve_set(ctx, shape, e, caps)
    ef, rf, hf = g.state()
    dist = oracle.sink_distances(shape, ef, rf)
    dist[dist == oracle.ORC_INF] = 1 << 30
    assert np.array_equal(hf, dist)
    g.close()


@pytest.mark.parametrize("sched", SCHEDULES)
@pytest.mark.parametrize("h,w", [(96, 200), (300, 700)])
def test_long_paths(ctx, sched, h, w):
    # a serpentine corridor: flow has to travel across many tiles
    use_schedule(ctx, sched)
    n = h * w
    caps = [np.zeros(n, np.int32) for _ in range(4)]
    c = [x.reshape(h, w) for x in caps]
    for y in range(0, h, 2):
        c[0][y, :-1] = 5; c[3][y, 1:] = 5
        x = w - 1 if (y // 2) % 2 == 0 else 0
        if y + 2 < h:
            c[1][y, x] = 5; c[2][y + 1, x] = 5
            c[1][y + 1, x] = 5; c[2][y + 2, x] = 5
    e = np.zeros(n, np.int32)
    e[0] = 1000
    e[(h - 2) * w + (w - 1 if ((h - 2) // 2) % 2 == 0 else 0)] = -1000
    g, st = solve_set(ctx, (h, w), e, caps)
    check_against_oracle((h, w), e, caps, g.flow(), g.labels())
    assert g.flow() == 5


@pytest.mark.parametrize("sched", SCHEDULES)
def test_gray_ellipse_build_and_solve(ctx, sched):
    use_schedule(ctx, sched)
    img, seeds = synthetic.gray_ellipse(512, 512, seed=3)
    g = jfcut.Graph(ctx, img.shape)
    g.build_from_image(img, seeds, jfcut.PIX_GRAY8, MODEL2)
    e_dev, r_dev, _ = g.state()
    e, caps, st = oracle.build_graph(img, seeds, 0, MODEL2)
    assert np.array_equal(e_dev, e)
    for k in range(4):
        assert np.array_equal(r_dev[k], caps[k])
    s = g.solve()
    check_against_oracle(img.shape, e, caps, g.flow(), g.labels(), sink_total=st)


@pytest.mark.parametrize("sched", SCHEDULES)
@pytest.mark.parametrize("w,h,seed", [(257, 131, 1), (640, 480, 2), (33, 1000, 3)])
def test_rgb_build_and_solve(ctx, w, h, seed, sched):
    use_schedule(ctx, sched)
    img, seeds = synthetic.rgb_ellipses(w, h, seed=seed)
    g = jfcut.Graph(ctx, (h, w))
    g.build_from_image(img, seeds, jfcut.PIX_RGB8, MODEL5)
    e_dev, r_dev, _ = g.state()
    e, caps, st = oracle.build_graph(img, seeds, 1, MODEL5)
    assert np.array_equal(e_dev, e)
    assert all(np.array_equal(r_dev[k], caps[k]) for k in range(4))
    g.solve()
    check_against_oracle((h, w), e, caps, g.flow(), g.labels(), sink_total=st)


@pytest.mark.parametrize("sched", SCHEDULES)
def test_video_build_and_solve(ctx, sched):
    use_schedule(ctx, sched)
    img, seeds = synthetic.rgb_video(96, 64, 8, seed=4)
    model = dict(MODEL5, z_weight_pct=50)
    g = jfcut.Graph(ctx, seeds.shape)
    g.build_from_image(img, seeds, jfcut.PIX_RGB8, model)
    e_dev, r_dev, _ = g.state()
    e, caps, st = oracle.build_graph(img, seeds, 1, model)
    assert np.array_equal(e_dev, e)
    assert all(np.array_equal(r_dev[k], caps[k]) for k in range(6))
    g.solve()
    check_against_oracle(seeds.shape, e, caps, g.flow(), g.labels(), sink_total=st)


@pytest.mark.parametrize("sched", SCHEDULES)
def test_i16_phantom_build_and_solve(ctx, sched):
    use_schedule(ctx, sched)
    img, seeds = synthetic.i16_phantom(40, 36, 28, seed=5)
    g = jfcut.Graph(ctx, seeds.shape)
    g.build_from_image(img, seeds, jfcut.PIX_I16, MODEL2)
    e_dev, r_dev, _ = g.state()
    e, caps, st = oracle.build_graph(img, seeds, 2, MODEL2)
    assert np.array_equal(e_dev, e)
    assert all(np.array_equal(r_dev[k], caps[k]) for k in range(6))
    g.solve()
    check_against_oracle(seeds.shape, e, caps, g.flow(), g.labels(), sink_total=st)


def test_warm_seed_edits(ctx):
    use_schedule(ctx, "default")
    img, seeds = synthetic.rgb_ellipses(300, 200, seed=11)
    g = jfcut.Graph(ctx, seeds.shape)
    g.build_from_image(img, seeds, jfcut.PIX_RGB8, MODEL5)
    g.solve()
    cur = seeds.copy().ravel()
    for k in range(3):
        idx, ns = synthetic.stroke(seeds.shape, seed=50 + k, n=600, label=1 + (k % 2))
        g.edit_seeds(idx, ns)
        g.solve()
        cur[idx] = ns
        # cold reference: the same edits applied to a freshly built graph (the colour
        # model stays the one of the original seeds, as on the warm path), solved cold
        e_dev, r_dev, _ = g.state()
        cold = jfcut.Graph(ctx, seeds.shape)
        cold.build_from_image(img, seeds, jfcut.PIX_RGB8, MODEL5)
        cold.edit_seeds(np.nonzero(cur != seeds.ravel())[0], cur[cur != seeds.ravel()])
        e0, c0, _ = cold.state()
        cold.solve()
        assert g.flow() == cold.flow()
        assert np.array_equal(g.labels(), cold.labels())
        # and both equal the oracle on the edited graph
        f, _, _, lab = oracle.maxflow(seeds.shape, e0, c0)
        assert np.array_equal(g.labels().ravel(), lab)
        cold.close()


def test_seed_edit_duplicates_last_wins(ctx):
    # (the final residual state of a solve is not unique, and the adaptive
    # relabel interval follows device clocks: flows and cuts are unique, and
    # the change an edit makes to the excess is fixed by the seeds alone)
    img, seeds = synthetic.rgb_ellipses(160, 120, seed=12)
    rng = np.random.default_rng(4)
    n = seeds.size
    idx = rng.integers(0, n, 3000).astype(np.uint32)          # many repeated nodes
    ns = rng.integers(0, 3, 3000).astype(np.uint8)
    last = {}
    for i, v in zip(idx.tolist(), ns.tolist()):
        last[i] = v
    ui = np.array(sorted(last), np.uint32)
    us = np.array([last[i] for i in ui.tolist()], np.uint8)
    out = []
    for a, b in ((idx, ns), (ui, us)):
        g = jfcut.Graph(ctx, seeds.shape)
        g.build_from_image(img, seeds, jfcut.PIX_RGB8, MODEL5)
        g.solve()
        e_solved = g.state()[0].copy()
        g.edit_seeds(a, b)
        e_edit = g.state()[0] - e_solved   # the edit's change of the excess
        g.solve()
        out.append((g.flow(), g.labels().copy(), e_edit))
        g.close()
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])


def test_edit_tlinks_deltas(ctx):
    rng = np.random.default_rng(3)
    shape = (70, 90)
    e, caps = random_grid(shape, rng)
    g, _ = solve_set(ctx, shape, e, caps)
    idx = rng.choice(e.size, 300, replace=False).astype(np.uint32)
    dcs = rng.integers(0, 200, 300).astype(np.int32)
    dct = rng.integers(0, 200, 300).astype(np.int32)
    g.edit_tlinks(idx, dcs, dct)
    g.solve()
    e2 = e.copy()
    e2[idx] += dcs - dct
    offset = int(np.minimum(dcs, dct).sum())
    # sum ct grows by dct; the folded oracle sees e2 with the extra min(dcs, dct) offset
    f, _, _, lab = oracle.maxflow(shape, e2, caps)
    # flow of the edited graph = sum_i min(cs', ct') + folded flow; with e given as net excess
    cs0 = np.maximum(e, 0).astype(np.int64); ct0 = np.maximum(-e, 0).astype(np.int64)
    cs1 = cs0.copy(); ct1 = ct0.copy()
    np.add.at(cs1, idx, dcs); np.add.at(ct1, idx, dct)
    assert g.flow() == f + int(np.minimum(cs1, ct1).sum())
    assert np.array_equal(g.labels().ravel(), lab)


def test_batch_matches_plain(ctx):
    use_schedule(ctx, "default")
    rng = np.random.default_rng(8)
    b = jfcut.Batch(ctx)
    graphs, refs = [], []
    for i in range(12):
        w, h = int(rng.integers(20, 300)), int(rng.integers(20, 300))
        img, seeds = synthetic.rgb_ellipses(w, h, seed=100 + i)
        g = jfcut.Graph(ctx, (h, w))
        g.build_from_image(img, seeds, jfcut.PIX_RGB8, MODEL5)
        e, caps, st = oracle.build_graph(img, seeds, 1, MODEL5)
        refs.append((e, caps, st))
        graphs.append(g)
        b.add(g)
    # one 3D grid in the same batch
    img, seeds = synthetic.i16_phantom(20, 24, 16, seed=9)
    g3 = jfcut.Graph(ctx, seeds.shape)
    g3.build_from_image(img, seeds, jfcut.PIX_I16, MODEL2)
    e3, c3, st3 = oracle.build_graph(img, seeds, 2, MODEL2)
    b.add(g3)
    stats = b.solve()
    assert all(s.status == 0 for s in stats)
    for g, (e, caps, st) in zip(graphs, refs):
        check_against_oracle(g.shape, e, caps, g.flow(), g.labels(), sink_total=st)
    check_against_oracle(g3.shape, e3, c3, g3.flow(), g3.labels(), sink_total=st3)


def test_batch_autotune_restores_and_matches(ctx):
    rng = np.random.default_rng(21)
    b = jfcut.Batch(ctx)
    graphs, flows = [], []
    for i in range(6):
        w, h = int(rng.integers(40, 260)), int(rng.integers(40, 260))
        img, seeds = synthetic.rgb_ellipses(w, h, seed=700 + i)
        g = jfcut.Graph(ctx, (h, w))
        g.build_from_image(img, seeds, jfcut.PIX_RGB8, MODEL5)
        ref = jfcut.Graph(ctx, (h, w))
        ref.build_from_image(img, seeds, jfcut.PIX_RGB8, MODEL5)
        ref.solve()
        flows.append((ref.flow(), ref.labels().copy()))
        ref.close()
        graphs.append(g)
        b.add(g)
    p = b.autotune()
    assert p.tile_rows in (8, 16) and p.local_iters in (8, 12, 16, 32) and p.relabel_interval in (0, 2, 3, 4, 8, 16)
    # the choice belongs to the batch: the context stays on the defaults
    use_schedule(ctx, "default")
    # the graphs are back in their built state: solving now gives the plain results
    st = b.solve()
    assert all(s.status == 0 for s in st)
    for g, (f, lab) in zip(graphs, flows):
        assert g.flow() == f
        assert np.array_equal(g.labels(), lab)
    b.close()


def test_solve_from_data_files(ctx, tmp_path):
    """Graphs loaded from the reference's file formats solve to the recorded
    max-flow: .ef/.c1/.c2 (flower, published value) and .mfi (its header)."""
    shape, e, caps, published, ref_object = load_fixture("flower")
    base = str(tmp_path / "flower")
    jfcut.save_graph_files(base, e.reshape(shape), [c.reshape(shape) for c in caps])
    g = jfcut.Graph(ctx, shape)
    g.load_files(base)
    g.solve()
    assert g.flow() == published
    jfcut.write_cut(base + ".cut", None, g.labels())
    _, lab = jfcut.read_cut(base + ".cut", shape)
    assert np.array_equal(lab, g.labels())
    jfcut.save_mfi(base + ".mfi", e.reshape(shape), [c.reshape(shape) for c in caps], published)
    g2 = jfcut.Graph(ctx, shape)
    assert g2.load_mfi(base + ".mfi") == published
    g2.solve()
    assert g2.flow() == published
    # a 3D instance with terminal caps on both sides of many nodes
    rng = np.random.default_rng(31)
    shp = (9, 20, 33)
    e3, c3 = random_grid(shp, rng, cap_max=200)
    f3, _, _, lab3 = oracle.maxflow(shp, e3, c3)
    jfcut.save_mfi(base + "3.mfi", e3.reshape(shp), [c.reshape(shp) for c in c3], f3)
    g3 = jfcut.Graph(ctx, shp)
    assert g3.load_mfi(base + "3.mfi") == f3
    g3.solve()
    assert g3.flow() == f3 and np.array_equal(g3.labels().ravel(), lab3)
    for x in (g, g2, g3):
        x.close()


def test_energy_certificate(ctx):
    """data + smooth energy of the canonical cut over the original graph equals
    the max-flow (device energy kernel vs oracle), 2D fixture and 3D random."""
    import torch
    cases = [load_fixture("sponge")[:4]]
    rng = np.random.default_rng(41)
    shp = (7, 19, 26)
    e3, c3 = random_grid(shp, rng)
    cases.append((shp, e3, c3, None))
    for shape, e, caps, published in cases:
        g, st = solve_set(ctx, shape, e, caps)
        flow = g.flow()
        if published is not None:
            assert flow == published
        lab = torch.from_numpy(g.labels().ravel().copy()).cuda()
        de = torch.from_numpy(np.ascontiguousarray(e, np.int32).ravel()).cuda()
        dc = [torch.from_numpy(np.ascontiguousarray(c, np.int32).ravel()).cuda() for c in caps]
        torch.cuda.synchronize()
        data, smooth = jfcut.energy_device(0, shape, de.data_ptr(), [c.data_ptr() for c in dc], lab.data_ptr())
        assert data + smooth == flow
        assert data + smooth == oracle.cut_energy(shape, e, caps, g.labels().ravel())
        # a worse labelling has a higher energy
        lab2 = lab.clone()
        lab2[: lab2.numel() // 3] = 1 - lab2[: lab2.numel() // 3]
        torch.cuda.synchronize()
        d2, s2 = jfcut.energy_device(0, shape, de.data_ptr(), [c.data_ptr() for c in dc], lab2.data_ptr())
        assert d2 + s2 >= flow
        assert d2 + s2 == oracle.cut_energy(shape, e, caps, lab2.cpu().numpy())
        g.close()


def _tag_oracle(obj, fg):
    """Object nodes connected through object nodes to a foreground seed (plus
    the seeds), by repeated 4/6-neighbour dilation."""
    tag = fg.copy()
    while True:
        grow = tag.copy()
        for ax in range(obj.ndim):
            for sh in (1, -1):
                rolled = np.roll(tag, sh, axis=ax)
                idx = [slice(None)] * obj.ndim
                idx[ax] = 0 if sh == 1 else -1
                rolled[tuple(idx)] = False
                grow |= rolled & obj
        if np.array_equal(grow, tag):
            return tag
        tag = grow


def test_tag_post_process(ctx):
    img, seeds = synthetic.gray_ellipse(300, 200, seed=21)
    g = jfcut.Graph(ctx, seeds.shape)
    g.build_from_image(img, seeds, jfcut.PIX_GRAY8, MODEL2)
    g.solve()
    lab = g.labels().copy()
    tag = g.tag()
    want = _tag_oracle(lab.astype(bool), seeds == jfcut.SEED_FG)
    assert np.array_equal(tag.astype(bool), want)
    assert np.array_equal(g.labels(), lab)          # labels untouched
    # explicit seeds on a graph given as arrays, 3D
    rng = np.random.default_rng(77)
    shp = (6, 17, 40)
    e, caps = random_grid(shp, rng, cap_max=30, density=0.5)
    g3, _ = solve_set(ctx, shp, e, caps)
    lab3 = g3.labels().reshape(shp).astype(bool)
    fg = np.zeros(shp, np.uint8)
    fg.ravel()[rng.choice(fg.size, 25, replace=False)] = jfcut.SEED_FG
    tag3 = g3.tag(fg)
    assert np.array_equal(tag3.astype(bool), _tag_oracle(lab3, fg == jfcut.SEED_FG))
    g.close()
    g3.close()


def test_fastcut_comparison_mode(ctx):
    """The reference's Fast-Cut line sweeps (pr_mode 1) reach the same exact
    max-flow and canonical cut as the block-wise solver."""
    ctx.set_params(pr_mode=1, relabel_interval=2)
    shape, e, caps, published, ref_object = load_fixture("flower")
    g, st = solve_set(ctx, shape, e, caps)
    assert g.flow() == published and st.status == 0
    assert np.array_equal(g.labels().ravel(), ref_object)
    g.close()
    for k, shp in enumerate([(37, 53), (100, 300), (6, 20, 33), (13, 40, 70)]):
        rng = np.random.default_rng(900 + k)
        e, caps = random_grid(shp, rng, cap_max=60, density=0.4)
        g, st = solve_set(ctx, shp, e, caps)
        check_against_oracle(shp, e, caps, g.flow(), g.labels())
        g.close()


def _view_matrix():
    """Column-major inverse view-projection: NDC (u, v, z) -> world, an
    orthographic camera looking down -z, rotated a little about y and x."""
    ca, sa, cb, sb = np.cos(0.3), np.sin(0.3), np.cos(0.2), np.sin(0.2)
    ry = np.array([[ca, 0, sa, 0], [0, 1, 0, 0], [-sa, 0, ca, 0], [0, 0, 0, 1]])
    rx = np.array([[1, 0, 0, 0], [0, cb, -sb, 0], [0, sb, cb, 0], [0, 0, 0, 1]])
    ortho = np.array([[1.3, 0, 0, 0], [0, 1.3, 0, 0], [0, 0, -4.0, -1.0], [0, 0, 0, 1]])
    mat = rx @ ry @ ortho                      # world = mat @ (u, v, z, 1)
    return mat.T.ravel().astype(np.float32)    # column-major


def test_stroke_to_seeds_matches_cpu_restatement(ctx):
    """Visibility mapping of a stroke through a volume (float ray march):
    device and CPU restatement agree on the marked voxels up to samples that
    sit on the opacity threshold (tolerance: 1% of the marked set)."""
    import torch
    import visibility
    d, h, w = 20, 28, 36
    zz, yy, xx = np.mgrid[0:d, 0:h, 0:w].astype(np.float32)
    vol = (np.exp(-(((xx - 18) / 9) ** 2 + ((yy - 14) / 7) ** 2 + ((zz - 10) / 5) ** 2))
           + 0.4 * np.exp(-(((xx - 6) / 4) ** 2 + ((yy - 20) / 4) ** 2 + ((zz - 4) / 3) ** 2))).astype(np.float32)
    vol = np.clip(vol, 0, 1).astype(np.float32)
    n = 64
    ramp = np.linspace(0, 1, n, dtype=np.float32)
    tf = np.stack([ramp, 1 - ramp, ramp * 0.5, ramp ** 2], 1).astype(np.float32)
    ih, iw = 24, 32
    mask = np.zeros((ih, iw), np.uint8)
    mask[4:20, 6:26] = 1
    view = jfcut.View()
    m = _view_matrix()
    for i in range(16):
        view.inverse_mvp[i] = float(m[i])
    for i in range(3):
        view.box[i] = 1.0
    view.image_w, view.image_h, view.samples = iw, ih, 96
    view.sample_ratio, view.sample_step_scale = 0.9, 2.0
    view.window_width, view.window_level, view.alpha = 1.0, 0.5, 0.3
    dv = torch.from_numpy(vol).cuda()
    dt = torch.from_numpy(tf).cuda()
    dm = torch.from_numpy(mask).cuda()
    ds = torch.zeros(d * h * w, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    jfcut.stroke_to_seeds(0, view, (d, h, w), dv.data_ptr(), dt.data_ptr(), n, dm.data_ptr(), jfcut.SEED_FG,
                          ds.data_ptr())
    gpu = ds.cpu().numpy().reshape(d, h, w)
    cpu = visibility.stroke_to_seeds(vol, tf, mask, m, [1.0, 1.0, 1.0], 96, 0.9, 2.0, 1.0, 0.5, 0.3,
                                     jfcut.SEED_FG, np.zeros((d, h, w), np.uint8))
    marked = (gpu > 0) | (cpu > 0)
    assert marked.sum() > 50                                  # the stroke does see the object
    assert ((gpu > 0) != (cpu > 0)).sum() <= max(1, marked.sum() // 100)
    assert set(np.unique(gpu)) <= {0, jfcut.SEED_FG}


def test_errors(ctx):
    img, seeds = synthetic.gray_ellipse(64, 64, seed=1)
    g = jfcut.Graph(ctx, img.shape)
    with pytest.raises(jfcut.JfcError) as ei:
        g.solve()
    assert ei.value.code == jfcut.ERR_STATE
    s2 = seeds.copy()
    s2[s2 == 2] = 0
    with pytest.raises(jfcut.JfcError) as ei:
        g.build_from_image(img, s2, jfcut.PIX_GRAY8)
    assert ei.value.code == jfcut.ERR_NO_SEEDS
    with pytest.raises(jfcut.JfcError) as ei:
        g.labels()
    assert ei.value.code == jfcut.ERR_STATE
    with pytest.raises(jfcut.JfcError) as ei:
        jfcut.Graph(ctx, (0, 5))
    assert ei.value.code == jfcut.ERR_INVALID_ARG
    bad = [np.full(4096, -1, np.int32)] * 4
    with pytest.raises(jfcut.JfcError) as ei:
        g.set(np.zeros(4096, np.int32), bad)
    assert ei.value.code == jfcut.ERR_INVALID_ARG


def test_budget_reports_not_converged(ctx):
    # a one-sweep budget on a long-path instance must fail loudly, never return a cut silently
    ctx.set_params(max_sweeps=1, relabel_interval=1, local_iters=1)
    shape, e, caps, published, _ = load_fixture("flower")
    g = jfcut.Graph(ctx, shape)
    g.set(e, caps)
    with pytest.raises(jfcut.JfcError) as ei:
        g.solve()
    assert ei.value.code == jfcut.ERR_NOT_CONVERGED
