"""CPU checker pinned against the reference: the published max-flows of the
three graphs that ship with JF-Cut, the reference GPU's own cut of flower, and
BK 3.03 built from the reference sources (oracle/_ref)."""
import numpy as np
import pytest

import oracle
import synthetic
from conftest import FIXTURES, load_fixture, random_grid

MODEL = dict(lambda_n=100, z_weight_pct=100, lambda_t=10, k_fg=2, k_bg=2, seed_cap=1000000, kmeans_iters=32)


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_golden_maxflow(name):
    shape, e, caps, published, ref_obj = load_fixture(name)
    f, ef, r, lab = oracle.maxflow(shape, e, caps)
    assert f == published                      # section-5-results.tex:31-41
    assert oracle.cut_energy(shape, e, caps, lab) == published   # energy check, QGCWidget.cpp:2452-2520
    assert oracle.check_residual(shape, e, caps, ef, r) == 0
    lab2, bad = oracle.cut_from_residual(shape, ef, r)
    assert bad == 0 and np.array_equal(lab, lab2)


def test_oracle_matches_reference_gpu_cut():
    # flower's .cut file carries the reference GPU's own object labels
    shape, e, caps, published, ref_obj = load_fixture("flower")
    _, _, _, lab = oracle.maxflow(shape, e, caps)
    assert ref_obj.sum() > 0
    assert np.array_equal(lab, ref_obj)


needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU solvers not built")


@needs_ref
@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_matches_bk303_fixture(name):
    shape, e, caps, published, _ = load_fixture(name)
    fb, labb, _ = oracle.bk_maxflow(shape, e, caps)
    f, _, _, lab = oracle.maxflow(shape, e, caps)
    assert fb == f == published
    assert np.array_equal(lab, labb)          # minimal source side, what_segment(i, SINK)


@needs_ref
@pytest.mark.parametrize("shape,seed", [((1, 1), 0), ((1, 37), 1), ((37, 1), 2), ((17, 33), 3), ((64, 64), 4),
                                        ((129, 67), 5), ((5, 5, 5), 6), ((3, 17, 9), 7), ((16, 20, 24), 8),
                                        ((1, 1, 40), 9)])
def test_oracle_matches_bk303_random(shape, seed):
    rng = np.random.default_rng(seed)
    e, caps = random_grid(shape, rng)
    fb, labb, _ = oracle.bk_maxflow(shape, e, caps)
    f, ef, r, lab = oracle.maxflow(shape, e, caps)
    assert f == fb
    assert np.array_equal(lab, labb)
    assert oracle.cut_energy(shape, e, caps, lab) == f
    assert oracle.check_residual(shape, e, caps, ef, r) == 0


@needs_ref
def test_oracle_gridcut_agrees():
    shape, e, caps, published, _ = load_fixture("sponge")
    fg, _ = oracle.gridcut_maxflow(shape, e, caps, 4)
    assert fg == published


def test_edge_cases():
    # no excess anywhere -> flow 0, empty source side
    shape = (9, 11)
    e = np.zeros(99, np.int32)
    caps = [np.full(99, 5, np.int32) for _ in range(4)]
    f, _, _, lab = oracle.maxflow(shape, e, caps)
    assert f == 0 and lab.sum() == 0
    # only excess -> nothing absorbed, every node reachable from excess is source side
    e = np.full(99, 3, np.int32)
    f, _, _, lab = oracle.maxflow(shape, e, caps)
    assert f == 0 and lab.sum() == 99
    # single node with both terminals
    f, _, _, lab = oracle.maxflow((1, 1), np.array([-4], np.int32), [np.zeros(1, np.int32)] * 4)
    assert f == 0 and lab[0] == 0


def test_build_model_gray_ellipse():
    img, seeds = synthetic.gray_ellipse(512, 512, seed=7)
    e, caps, st = oracle.build_graph(img, seeds, 0, MODEL)
    h, w = img.shape
    c = [x.reshape(h, w) for x in caps]
    # symmetric n-links, zero at the border, weights in [0, lambda_n]
    assert np.array_equal(c[0][:, :-1], c[3][:, 1:]) and np.array_equal(c[1][:-1], c[2][1:])
    assert (c[0][:, -1] == 0).all() and (c[3][:, 0] == 0).all()
    assert 0 <= min(x.min() for x in caps) and max(x.max() for x in caps) <= 100
    # hard seeds
    ee = e.reshape(h, w)
    assert (ee[seeds == 1] == 1000000).all() and (ee[seeds == 2] == -1000000).all()
    assert st > 0
    # deterministic
    e2, caps2, st2 = oracle.build_graph(img, seeds, 0, MODEL)
    assert np.array_equal(e, e2) and st == st2


def test_no_seeds_rejected():
    img, seeds = synthetic.gray_ellipse(64, 64, seed=1)
    seeds[seeds == 2] = 0
    with pytest.raises(ValueError):
        oracle.build_graph(img, seeds, 0, MODEL)


@needs_ref
def test_gray_ellipse_flow_vs_bk():
    img, seeds = synthetic.gray_ellipse(512, 512, seed=3)
    e, caps, st = oracle.build_graph(img, seeds, 0, MODEL)
    fb, labb, _ = oracle.bk_maxflow(img.shape, e, caps)
    f, _, _, lab = oracle.maxflow(img.shape, e, caps)
    assert f == fb and np.array_equal(lab, labb)
    # the object is recovered: most of the ellipse interior is source side
    assert 0.05 < lab.mean() < 0.5
