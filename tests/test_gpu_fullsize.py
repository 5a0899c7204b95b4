"""Full-size certificates: the plain workload (2D 4-conn 15000 x 10000 RGB, 150M
nodes) and the video workload (3D 6-conn 2560 x 1440 x 50 RGB, 184M nodes) are
too large for the sequential oracle, so their results are certified by
size-independent properties instead:
  * the final state is a valid preflow of the original graph (capacities,
    antisymmetry, conservation: checked on the CPU),
  * the labels are exactly the nodes reachable from excess in that residual
    graph and no deficit is reachable (CPU residual BFS),
  * the energy of the cut over the ORIGINAL capacities (device kernel) equals
    the flow: a feasible flow and a cut of equal value are both optimal."""
import numpy as np
import pytest

import jfcut
import oracle
import synthetic

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

MODEL5 = dict(lambda_n=100, z_weight_pct=100, lambda_t=10, k_fg=5, k_bg=5, seed_cap=1000000, kmeans_iters=32)


def _workload(kind):
    if kind == "plain":
        img, seeds = synthetic.rgb_ellipses(15000, 10000, seed=20240601, n_ellipses=20, noise_sigma=15,
                                              stroke_permille_x10=50)
        return img, seeds, MODEL5
    img, seeds = synthetic.rgb_video(2560, 1440, 50, seed=20240601 + 50)
    return img, seeds, dict(MODEL5, z_weight_pct=50)


@pytest.mark.parametrize("kind", ["plain", "video"])
def test_full_size_certificate(ctx, kind):
    import torch
    img, seeds, model = _workload(kind)
    shape = seeds.shape
    g = jfcut.Graph(ctx, shape)
    g.build_from_image(img, seeds, jfcut.PIX_RGB8, model)
    e0, c0, _ = g.state()                       # the original graph (net-excess form)
    st = g.solve()
    assert st.status == 0
    flow = g.flow()
    ef, rf, _ = g.state()
    labels = g.labels().ravel()
    # valid preflow of the original graph
    assert oracle.check_residual(shape, e0, c0, ef, rf) == 0
    # canonical cut = residual reachability from excess, no deficit reachable
    lab, bad = oracle.cut_from_residual(shape, ef, rf)
    assert bad == 0
    assert np.array_equal(lab, labels)
    # energy of the cut over the original capacities equals the folded flow
    folded = int(np.minimum(ef.astype(np.int64), 0).sum()) - int(np.minimum(e0.astype(np.int64), 0).sum())
    de = torch.from_numpy(e0).cuda()
    dc = [torch.from_numpy(c).cuda() for c in c0]
    dl = torch.from_numpy(labels.copy()).cuda()
    torch.cuda.synchronize()
    data, smooth = jfcut.energy_device(0, shape, de.data_ptr(), [c.data_ptr() for c in dc], dl.data_ptr())
    assert data + smooth == folded
    assert flow == st.flow
    g.close()
