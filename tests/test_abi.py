"""The C-ABI library loads and exports every entry point include/jfcut.h
declares; host-only helpers behave without a GPU."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import PKG, ROOT, gpu_available

HEADER = os.path.join(ROOT, "include", "jfcut.h")
LIB = os.path.join(PKG, "libjfcut.so")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(jfc_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for must in ("jfc_create", "jfc_graph_create_grid", "jfc_graph_build_from_image", "jfc_graph_set",
                 "jfc_solve", "jfc_get_flow", "jfc_read_labels", "jfc_edit_tlinks", "jfc_batch_solve",
                 "jfc_server_submit", "jfc_strerror"):
        assert must in syms


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (jfc_[a-z0-9_]+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    lib = ctypes.CDLL(LIB)
    for s in declared_symbols():
        assert getattr(lib, s) is not None


def test_build_targets_sm100a_only():
    mk = open(os.path.join(PKG, "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk


def test_strerror_and_defaults():
    import jfcut
    L = jfcut.lib()
    assert L.jfc_strerror(0) == b"ok"
    assert b"no labels" in L.jfc_strerror(2)
    p = jfcut.default_params()
    # the measured defaults: 32x8 tiles, 12 rounds per visit, automatic relabel
    # interval (2D every 2 sweep pairs, 3D every 3), interval cap 64, graphs on
    assert (p.tile_rows, p.local_iters, p.relabel_interval, p.relabel_interval_max) == (8, 12, 0, 64)
    assert p.use_graph == 1 and p.pr_mode == 0 and p.tile_depth == 0
    m = jfcut.default_model()
    assert m.lambda_n == 100 and m.lambda_t == 10 and m.seed_cap == 1000000


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_no_device_fails_loudly():
    import jfcut
    with pytest.raises(jfcut.JfcError) as ei:
        jfcut.Context(0)
    assert ei.value.code == jfcut.ERR_NO_DEVICE


def test_synth_deterministic():
    import jfcut
    a = jfcut.synth_rgb_ellipses(301, 197, seed=5)
    b = jfcut.synth_rgb_ellipses(301, 197, seed=5)
    c = jfcut.synth_rgb_ellipses(301, 197, seed=6)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert not np.array_equal(a[0], c[0])
    img, seeds = a
    frac = (seeds > 0).mean()
    assert 0.004 < frac < 0.02 and (seeds == 1).any() and (seeds == 2).any()
    g, s = jfcut.synth_gray_ellipse(128, 96, seed=1)
    assert g.dtype == np.uint8 and (s == 1).any() and (s == 2).any()
    v, vs = jfcut.synth_rgb_video(64, 48, 6, seed=2)
    assert v.shape == (6, 48, 64, 3) and (vs[0] > 0).any() and (vs[5] > 0).any() and not (vs[2] > 0).any()
    p, ps = jfcut.synth_i16_phantom(24, 24, 24, seed=3)
    assert p.dtype == np.int16 and (ps == 1).any() and (ps == 2).any()
    idx, ns = jfcut.synth_stroke((40, 50), seed=9, n=100, label=1)
    assert len(np.unique(idx)) == len(idx) > 50 and (ns == 1).all() and idx.max() < 2000
