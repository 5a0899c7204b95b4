"""ctypes loader for the CPU checker (oracle/liboracle.so) and the reference's
own CPU solvers (oracle/_ref/libjfcref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker, never as the measured or
shipped path.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

I32P = ctypes.POINTER(ctypes.c_int32)
U8P = ctypes.POINTER(ctypes.c_uint8)


class OrcModel(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in
                ("lambda_n", "z_weight_pct", "lambda_t", "k_fg", "k_bg", "seed_cap", "kmeans_iters")]


def build():
    """Compile liboracle.so (and _ref/ when the reference tree is present)."""
    import subprocess
    subprocess.run(["make", "-s", "-f", os.path.join(HERE, "Makefile")], check=True, cwd=HERE)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_build_graph.restype = ctypes.c_int
        L.orc_build_graph_ex.restype = ctypes.c_int
        L.orc_maxflow.restype = ctypes.c_int64
        L.orc_cut_from_residual.restype = ctypes.c_int64
        L.orc_cut_energy.restype = ctypes.c_int64
        L.orc_check_residual.restype = ctypes.c_int64
        _LIB = L
    return _LIB


def ref_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libjfcref.so"))


def ref():
    global _REF
    if _REF is None:
        R = ctypes.CDLL(os.path.join(HERE, "_ref", "libjfcref.so"))
        R.ref_bk_maxflow.restype = ctypes.c_longlong
        R.ref_gridcut_maxflow.restype = ctypes.c_longlong
        _REF = R
    return _REF


def _ptrs(arrs):
    arrs = [np.ascontiguousarray(a, dtype=np.int32) for a in arrs]
    P = (I32P * len(arrs))(*[a.ctypes.data_as(I32P) for a in arrs])
    return arrs, P


def _shape(shape):
    if len(shape) == 2:
        h, w = shape
        return 2, w, h, 1
    d, h, w = shape
    return 3, w, h, d


def build_graph(img, seeds, pixfmt, model, seeds_tl=None):
    """Capacity build.  img: (H,W)/(H,W,3)/(D,H,W) array; seeds same grid.
    Returns (e, caps[conn], sink_total) or raises on missing seeds.
    seeds_tl: the seeds after stroke edits — the colour models are fit on
    `seeds`, the t-links follow `seeds_tl` (the graph a warm-edited session
    holds)."""
    shape = seeds.shape
    dims, w, h, d = _shape(shape)
    conn = 4 if dims == 2 else 6
    n = w * h * d
    e = np.zeros(n, np.int32)
    caps = [np.zeros(n, np.int32) for _ in range(conn)]
    _, P = _ptrs(caps)
    st = ctypes.c_int64(0)
    m = OrcModel(*[int(model[k]) for k in ("lambda_n", "z_weight_pct", "lambda_t", "k_fg", "k_bg",
                                            "seed_cap", "kmeans_iters")])
    img = np.ascontiguousarray(img)
    seeds = np.ascontiguousarray(seeds, dtype=np.uint8)
    tl = seeds if seeds_tl is None else np.ascontiguousarray(seeds_tl, dtype=np.uint8).reshape(seeds.shape)
    rc = lib().orc_build_graph_ex(dims, w, h, d, pixfmt, img.ctypes.data_as(ctypes.c_void_p),
                                  seeds.ctypes.data_as(U8P), tl.ctypes.data_as(U8P), ctypes.byref(m),
                                  e.ctypes.data_as(I32P), P, ctypes.byref(st), None)
    if rc != 0:
        raise ValueError("oracle build failed: %d" % rc)
    return e, caps, st.value


def maxflow(shape, e, caps):
    """Folded max-flow, final residual state and the minimal source side."""
    dims, w, h, d = _shape(shape)
    e = np.array(e, dtype=np.int32, copy=True)
    caps = [np.array(c, dtype=np.int32, copy=True) for c in caps]
    _, P = _ptrs(caps)
    lab = np.zeros(e.size, np.uint8)
    f = lib().orc_maxflow(dims, w, h, d, e.ctypes.data_as(I32P), P, lab.ctypes.data_as(U8P))
    return int(f), e, caps, lab


def cut_from_residual(shape, e, r):
    dims, w, h, d = _shape(shape)
    e = np.ascontiguousarray(e, dtype=np.int32)
    keep, P = _ptrs(r)
    lab = np.zeros(e.size, np.uint8)
    bad = lib().orc_cut_from_residual(dims, w, h, d, e.ctypes.data_as(I32P), P, lab.ctypes.data_as(U8P))
    return lab, int(bad)


ORC_INF = 0x3FFFFFFF


def sink_distances(shape, e, r):
    """Exact residual BFS distance to the nearest deficit (ORC_INF if none)."""
    dims, w, h, d = _shape(shape)
    e = np.ascontiguousarray(e, dtype=np.int32)
    keep, P = _ptrs(r)
    out = np.empty(e.size, np.int32)
    lib().orc_sink_distances(dims, w, h, d, e.ctypes.data_as(I32P), P, out.ctypes.data_as(I32P))
    return out


def cut_energy(shape, e0, caps0, labels):
    dims, w, h, d = _shape(shape)
    e0 = np.ascontiguousarray(e0, dtype=np.int32)
    keep, P = _ptrs(caps0)
    labels = np.ascontiguousarray(labels, dtype=np.uint8)
    return int(lib().orc_cut_energy(dims, w, h, d, e0.ctypes.data_as(I32P), P, labels.ctypes.data_as(U8P)))


def check_residual(shape, e0, c0, e, r):
    dims, w, h, d = _shape(shape)
    e0 = np.ascontiguousarray(e0, dtype=np.int32)
    e = np.ascontiguousarray(e, dtype=np.int32)
    k0, P0 = _ptrs(c0)
    k1, P1 = _ptrs(r)
    return int(lib().orc_check_residual(dims, w, h, d, e0.ctypes.data_as(I32P), P0,
                                        e.ctypes.data_as(I32P), P1))


def bk_maxflow(shape, e, caps, want_labels=True):
    """Reference BK 3.03 (compiled from the reference sources).  Returns
    (folded flow, labels or None, (t_init, t_maxflow, t_output))."""
    dims, w, h, d = _shape(shape)
    e = np.ascontiguousarray(e, dtype=np.int32)
    keep, P = _ptrs(caps)
    lab = np.zeros(e.size, np.uint8) if want_labels else None
    times = (ctypes.c_double * 3)()
    f = ref().ref_bk_maxflow(dims, w, h, d, e.ctypes.data_as(I32P), P,
                             lab.ctypes.data_as(U8P) if want_labels else None, times)
    return int(f), lab, tuple(times)


def gridcut_maxflow(shape, e, caps, threads, labels=None):
    """Reference GridCut 1.1 multi-threaded.  Returns (folded flow,
    (t_init, t_maxflow, t_output)); `labels` (uint8 array of the grid's size,
    optional) receives the source side GridCut reports."""
    dims, w, h, d = _shape(shape)
    e = np.ascontiguousarray(e, dtype=np.int32)
    keep, P = _ptrs(caps)
    times = (ctypes.c_double * 3)()
    lp = labels.ctypes.data_as(U8P) if labels is not None else None
    f = ref().ref_gridcut_maxflow(dims, w, h, d, e.ctypes.data_as(I32P), P, int(threads), lp, times)
    return int(f), tuple(times)
