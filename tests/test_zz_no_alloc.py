"""The allocation-free 2D solve (jfc_solve_grid2d_noalloc) against the
regular entry points (jfc_graph_set + jfc_solve + jfc_read_labels).

The no-allocation entry point is for callers that cannot allocate device
memory when they need a cut (real-time frame loops that must not stall on the
allocator, hosts with a fixed memory budget): its working set is a fixed
device array shared by every call, so this file checks calls in a row (a call
must not see the previous one's leftovers) under both tile heights, a grid at
the size limit, that a call allocates no device memory, and the limit itself.
It sits in its own file, collected last."""
import numpy as np
import pytest

import jfcut
from conftest import load_fixture, random_grid

pytestmark = pytest.mark.gpu


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def noalloc_solve(shape, e, caps, offset=0, params=None):
    torch = _torch()
    h, w = shape
    d_e = torch.from_numpy(np.ascontiguousarray(e, dtype=np.int32)).cuda()
    d_c = [torch.from_numpy(np.ascontiguousarray(c, dtype=np.int32)).cuda() for c in caps]
    d_lab = torch.full((h * w,), 7, dtype=torch.uint8, device="cuda")   # poison: every byte must be written
    torch.cuda.synchronize()
    flow = jfcut.solve_grid2d_noalloc(w, h, d_e.data_ptr(), [c.data_ptr() for c in d_c], d_lab.data_ptr(),
                                      flow_offset=offset, params=params)
    torch.cuda.synchronize()
    return flow, d_lab.cpu().numpy()


def graph_solve(ctx, shape, e, caps, offset=0):
    g = jfcut.Graph(ctx, shape)
    g.set(e, caps, offset)
    g.solve()
    f, lab = g.flow(), g.labels().ravel()
    g.close()
    return f, lab


@pytest.mark.parametrize("tile_rows", [8, 16])
def test_noalloc_matches_graph_api_on_consecutive_calls(ctx, tile_rows):
    params = jfcut.default_params(tile_rows=tile_rows)
    shape_f, e_f, caps_f, published, _ = load_fixture("flower")
    rng = np.random.default_rng(77)
    shape_r = (130, 257)
    e_r, caps_r = random_grid(shape_r, rng, cap_max=300, density=0.6)
    shape_l = (512, 1024)                      # exactly the 524,288-node limit
    e_l, caps_l = random_grid(shape_l, np.random.default_rng(78), cap_max=200, density=0.4)
    cases = [(shape_f, e_f, caps_f, 0), (shape_r, e_r, caps_r, 11), (shape_l, e_l, caps_l, 5),
             (shape_f, e_f, caps_f, 0)]
    for shape, e, caps, off in cases:
        f_ref, lab_ref = graph_solve(ctx, shape, e, caps, off)
        f, lab = noalloc_solve(shape, e, caps, off, params)
        assert f == f_ref                      # int64 max-flow, bit-exact
        assert np.array_equal(lab, lab_ref)    # canonical cut, bit-exact
    assert noalloc_solve(shape_f, e_f, caps_f, params=params)[0] == published


def test_noalloc_call_allocates_no_device_memory(ctx):
    torch = _torch()
    shape, e, caps, published, _ = load_fixture("person")
    h, w = shape
    d_e = torch.from_numpy(np.ascontiguousarray(e, dtype=np.int32)).cuda()
    d_c = [torch.from_numpy(np.ascontiguousarray(c, dtype=np.int32)).cuda() for c in caps]
    d_lab = torch.empty(h * w, dtype=torch.uint8, device="cuda")
    ptrs = [c.data_ptr() for c in d_c]
    torch.cuda.synchronize()
    assert jfcut.solve_grid2d_noalloc(w, h, d_e.data_ptr(), ptrs, d_lab.data_ptr()) == published   # warm-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert jfcut.solve_grid2d_noalloc(w, h, d_e.data_ptr(), ptrs, d_lab.data_ptr()) == published
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_grids_over_the_limit():
    torch = _torch()
    w, h = 1024, 520                           # 1024 x 528 padded > 524288 nodes
    d = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(jfcut.JfcError) as ei:
        jfcut.solve_grid2d_noalloc(w, h, d.data_ptr(), [d.data_ptr()] * 4, d.data_ptr())
    assert ei.value.code == jfcut.ERR_INVALID_ARG
    assert "no-allocation limit" in str(ei.value)
