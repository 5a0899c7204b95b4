"""Device-side waits give up cleanly.  Every spin-wait of the persistent
kernels (the grid barrier, the relabel worklist's slot, lock and ring waits)
is bounded by jfc_params.spin_limit polls.  With a limit of one poll a
many-CTA solve must run a wait out: the kernels leave, the call returns
JFC_ERR_CUDA with the "timed out" message, and the same context then solves
the same graph bit-exactly once the limit is back to its default.  No wait
is made endless and nothing faults: the expiry is a flag the host reads."""
import numpy as np
import pytest

import jfcut
import oracle
from conftest import random_grid

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(700, 1900), (24, 90, 120)])
def test_expired_wait_reports_and_context_recovers(ctx, shape):
    rng = np.random.default_rng(61)
    e, caps = random_grid(shape, rng, cap_max=80, density=0.5)
    f_ref, _, _, lab_ref = oracle.maxflow(shape, e, caps)
    g = jfcut.Graph(ctx, shape)
    g.set(e, caps)
    ctx.set_params(spin_limit=1)
    with pytest.raises(jfcut.JfcError) as ei:
        g.solve()
    assert ei.value.code == jfcut.ERR_CUDA
    assert "timed out" in str(ei.value)
    ctx.reset_params()
    assert ctx.params().spin_limit == 0
    # the same graph object, reloaded, and a fresh one: both exact
    g.set(e, caps)
    st = g.solve()
    assert st.status == 0 and g.flow() == f_ref
    assert np.array_equal(g.labels().ravel(), lab_ref)
    g2 = jfcut.Graph(ctx, shape)
    g2.set(e, caps)
    g2.solve()
    assert g2.flow() == f_ref and np.array_equal(g2.labels().ravel(), lab_ref)
    g.close()
    g2.close()
