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


def test_product_library_carries_no_input_generators():
    """Synthetic workload generators are test / bench inputs, not part of the
    drop-in library: the product exports only the graph-cut ABI."""
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    assert "synth" not in out and "syn_" not in out
