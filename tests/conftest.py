"""Shared test setup.  `-m gpu` tests need a B200 and call the CUDA library
through its C ABI; everything else runs on the CPU."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "jf-cut_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")
FIXTURES = ("flower", "person", "sponge")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running full-size case")


def _ensure_built():
    if not os.path.exists(os.path.join(PKG, "libjfcut.so")):
        subprocess.run(["make", "-s", "-j8", "-C", PKG], check=True)
    if not all(os.path.exists(os.path.join(ORACLE, f)) for f in ("liboracle.so", "libsynthetic.so")):
        subprocess.run(["make", "-s", "-f", os.path.join(ORACLE, "Makefile")], check=True, cwd=ORACLE)


_ensure_built()


def load_fixture(name):
    """Golden graph from the reference data: (shape, excess, caps[4], maxflow, ref_object)."""
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    w, h = int(z["width"]), int(z["height"])
    px = z["caps_px"].astype(np.int32).reshape(h, w)
    py = z["caps_py"].astype(np.int32).reshape(h, w)
    mx = np.zeros_like(px)
    mx[:, 1:] = px[:, :-1]
    my = np.zeros_like(py)
    my[1:] = py[:-1]
    caps = [px.ravel(), py.ravel(), my.ravel(), mx.ravel()]
    return (h, w), z["excess"].astype(np.int32), caps, int(z["maxflow"]), z["ref_object"]


def random_grid(shape, rng, cap_max=100, excess_max=300, density=0.5):
    """Random folded grid graph (arcs leaving the grid are zero)."""
    dims = len(shape)
    n = int(np.prod(shape))
    conn = 4 if dims == 2 else 6
    caps = [rng.integers(0, cap_max + 1, n).astype(np.int32) for _ in range(conn)]
    mask = rng.random(n) < density
    e = np.where(mask, rng.integers(-excess_max, excess_max + 1, n), 0).astype(np.int32)
    zero_boundary(shape, caps)
    return e, caps


def zero_boundary(shape, caps):
    if len(shape) == 2:
        h, w = shape
        c = [x.reshape(h, w) for x in caps]
        c[0][:, -1] = 0; c[1][-1, :] = 0; c[2][0, :] = 0; c[3][:, 0] = 0
    else:
        d, h, w = shape
        c = [x.reshape(d, h, w) for x in caps]
        c[0][:, :, -1] = 0; c[1][:, -1, :] = 0; c[2][-1] = 0
        c[3][0] = 0; c[4][:, 0, :] = 0; c[5][:, :, 0] = 0


def gpu_available():
    try:
        import jfcut
        jfcut.Context(0).close()
        return True
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx():
    import jfcut
    c = jfcut.Context(0)
    yield c
    c.close()


@pytest.fixture(autouse=True)
def _default_schedule(request):
    """Every test that uses the shared context starts, and leaves it, on the
    library's default schedule (the one bench.py times): a test that changes
    the schedule cannot leak it into the tests after it."""
    if "ctx" not in request.fixturenames:
        yield
        return
    c = request.getfixturevalue("ctx")
    c.reset_params()
    yield
    c.reset_params()


# Schedules the parity tests run under: the default (32 x 8 tiles, 12 rounds
# per visit, automatic relabel interval, relabel distance cap and visit
# scheduling), 32 x 16 relabel tiles with push-relabel on their 32 x 8
# halves, whole 32 x 16 push-relabel tiles, every relabel exact (no cap), a
# cap of 2 (almost every node starts unreachable, so the exact certifying
# relabel and the uncapped continuation after it carry the solve), and the
# two visit schedulers (checkerboard sweeps, asynchronous worklist) named
# explicitly.
SCHEDULES = {"default": {}, "rows16": dict(tile_rows=16), "whole16": dict(tile_rows=16, pr_mode=2),
             "exact": dict(relabel_cap=-1), "cap2": dict(relabel_cap=2),
             "sweeps": dict(pr_sched=1), "worklist": dict(pr_sched=2), "hybrid": dict(pr_sched=3),
             "rows16_sweeps": dict(tile_rows=16, pr_sched=1)}


def use_schedule(ctx, name):
    """Switch the shared context to a named schedule; for "default" also check
    that the context really is on the library defaults."""
    import jfcut
    if name == "default":
        p, d = ctx.params(), jfcut.default_params()
        assert all(getattr(p, f) == getattr(d, f) for f, _ in p._fields_), "context is not on the defaults"
    else:
        ctx.set_params(**SCHEDULES[name])
