"""Python host mirror of the JF-Cut graph-cut operator over libjfcut.so (C ABI).

The reference's operator is the QGCWidget class (src/QVisualizer/Graph Cut/
QGCWidget.h:160-243).  This module keeps its vocabulary: a Graph is built from
an image plus seed strokes (slotModelClicked, QGCWidget.cpp:2560-2606) or loaded
from excess / capacity arrays (slotLoadGraphClicked, :2631-2736), solved
(slotCutClicked, :2364-2558) and read back as labels (cut.object) and an int64
max-flow.  Every call goes to the CUDA library; there is no CPU fallback — if
the library is missing or no GPU is present the call raises.
"""
import ctypes
import os
import weakref

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# JFCUT_LIB selects another build of the library (e.g. an instrumented one)
LIB_PATH = os.environ.get("JFCUT_LIB") or os.path.join(HERE, "libjfcut.so")

OK, ERR_INVALID_ARG, ERR_NO_SEEDS, ERR_OOM, ERR_NOT_CONVERGED, ERR_CUDA, ERR_NO_DEVICE, ERR_STATE, \
    ERR_CANCELLED, ERR_BUSY, ERR_IO = range(11)
FMT_UCHAR, FMT_CHAR, FMT_USHORT, FMT_SHORT, FMT_UINT, FMT_INT, FMT_FLOAT = range(7)
PIX_GRAY8, PIX_RGB8, PIX_I16 = 0, 1, 2
SEED_NONE, SEED_FG, SEED_BG = 0, 1, 2


class JfcError(RuntimeError):
    def __init__(self, code, where=""):
        self.code = code
        lib = _lib()
        msg = lib.jfc_strerror(code).decode()
        detail = lib.jfc_last_error().decode()
        super().__init__("%s: %s (%s)%s" % (where, msg, detail, "" if code else ""))


class Params(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("tile_rows", "local_iters", "relabel_interval", "max_sweeps",
                                             "max_bfs_passes", "use_graph", "verbose", "relabel_interval_max",
                                             "tile_depth", "pr_mode", "spin_limit", "relabel_cap", "pr_sched",
                                             "local_iters_tail")]


class Model(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("lambda_n", "z_weight_pct", "lambda_t", "k_fg", "k_bg",
                                             "seed_cap", "kmeans_iters")]


class Stats(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("sweeps", ctypes.c_int), ("global_relabels", ctypes.c_int),
                ("bfs_passes", ctypes.c_int), ("tile_visits", ctypes.c_longlong), ("flow", ctypes.c_longlong),
                ("source_nodes", ctypes.c_longlong), ("ms_total", ctypes.c_double), ("ms_build", ctypes.c_double),
                ("ms_push_relabel", ctypes.c_double), ("ms_global_relabel", ctypes.c_double),
                ("ms_cut", ctypes.c_double), ("pr_rounds", ctypes.c_longlong), ("bfs_visits", ctypes.c_longlong),
                ("ms_gr_first", ctypes.c_double), ("ms_gr_frontier", ctypes.c_double), ("used_graph", ctypes.c_int),
                ("pr_phases", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class RequestInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("flow", ctypes.c_int64), ("ms_queue", ctypes.c_double),
                ("ms_solve", ctypes.c_double), ("ms_total", ctypes.c_double), ("warm", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("budget", ctypes.c_size_t), ("used", ctypes.c_size_t), ("peak_used", ctypes.c_size_t),
                ("sessions", ctypes.c_int), ("waiting", ctypes.c_int), ("solving", ctypes.c_int),
                ("peak_solving", ctypes.c_int), ("loops", ctypes.c_int64), ("requests_done", ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class VolumeInfo(ctypes.Structure):
    _fields_ = [("object_file", ctypes.c_char * 256), ("w", ctypes.c_int), ("h", ctypes.c_int), ("d", ctypes.c_int),
                ("thickness", ctypes.c_float * 3), ("format", ctypes.c_int), ("big_endian", ctypes.c_int),
                ("intensity_min", ctypes.c_float), ("intensity_max", ctypes.c_float)]


class View(ctypes.Structure):
    """Ray-casting view of the stroke-to-seed mapping (jfc_view)."""
    _fields_ = [("inverse_mvp", ctypes.c_float * 16), ("box", ctypes.c_float * 3), ("image_w", ctypes.c_int),
                ("image_h", ctypes.c_int), ("samples", ctypes.c_int), ("sample_ratio", ctypes.c_float),
                ("sample_step_scale", ctypes.c_float), ("window_width", ctypes.c_float),
                ("window_level", ctypes.c_float), ("alpha", ctypes.c_float)]


class MfiInfo(ctypes.Structure):
    _fields_ = [("dims", ctypes.c_int), ("conn", ctypes.c_int), ("w", ctypes.c_int), ("h", ctypes.c_int),
                ("d", ctypes.c_int), ("maxflow", ctypes.c_int64), ("active_count", ctypes.c_int),
                ("type_terminal", ctypes.c_int), ("type_neighbor", ctypes.c_int)]

    @property
    def shape(self):
        return (self.h, self.w) if self.dims == 2 else (self.d, self.h, self.w)


_LIB = None
VP = ctypes.c_void_p
I32P = ctypes.POINTER(ctypes.c_int32)
U8P = ctypes.POINTER(ctypes.c_uint8)
U32P = ctypes.POINTER(ctypes.c_uint32)


def _lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libjfcut.so is not built (run `make -C jf-cut_b200`)")
        L = ctypes.CDLL(LIB_PATH)
        L.jfc_strerror.restype = ctypes.c_char_p
        L.jfc_last_error.restype = ctypes.c_char_p
        L.jfc_graph_bytes.restype = ctypes.c_size_t
        L.jfc_graph_bytes.argtypes = [ctypes.c_int] * 4
        L.jfc_create.argtypes = [ctypes.c_int, ctypes.POINTER(Params), ctypes.POINTER(VP)]
        L.jfc_destroy.argtypes = [VP]
        L.jfc_destroy.restype = None
        L.jfc_set_params.argtypes = [VP, ctypes.POINTER(Params)]
        L.jfc_set_stream.argtypes = [VP, VP]
        L.jfc_kernel_launches.restype = ctypes.c_ulonglong
        L.jfc_get_params.argtypes = [VP, ctypes.POINTER(Params)]
        L.jfc_default_params.argtypes = [ctypes.POINTER(Params)]
        L.jfc_default_params.restype = None
        L.jfc_default_model.argtypes = [ctypes.POINTER(Model)]
        L.jfc_default_model.restype = None
        L.jfc_graph_create_grid.argtypes = [VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.POINTER(VP)]
        L.jfc_graph_destroy.argtypes = [VP]
        L.jfc_graph_destroy.restype = None
        L.jfc_graph_build_from_image.argtypes = [VP, VP, ctypes.c_int, U8P, ctypes.POINTER(Model)]
        L.jfc_graph_build_from_device.argtypes = [VP, VP, ctypes.c_int, VP, ctypes.POINTER(Model)]
        L.jfc_graph_set.argtypes = [VP, I32P, ctypes.POINTER(I32P), ctypes.c_int64]
        L.jfc_graph_set_device.argtypes = [VP, VP, ctypes.POINTER(VP), ctypes.c_int64]
        L.jfc_graph_get_state.argtypes = [VP, I32P, ctypes.POINTER(I32P), I32P]
        L.jfc_solve.argtypes = [VP, ctypes.POINTER(Stats)]
        L.jfc_get_flow.argtypes = [VP, ctypes.POINTER(ctypes.c_int64)]
        L.jfc_read_labels.argtypes = [VP, U8P]
        L.jfc_read_labels_device.argtypes = [VP, VP]
        L.jfc_edit_tlinks.argtypes = [VP, U32P, I32P, I32P, ctypes.c_size_t]
        L.jfc_graph_edit_seeds.argtypes = [VP, U32P, U8P, ctypes.c_size_t]
        L.jfc_solve_grid2d_noalloc.argtypes = [ctypes.c_int, VP, ctypes.POINTER(Params), ctypes.c_int,
                                               ctypes.c_int, VP, ctypes.POINTER(VP), ctypes.c_int64, VP,
                                               ctypes.POINTER(ctypes.c_int64)]
        L.jfc_batch_create.argtypes = [VP, ctypes.POINTER(VP)]
        L.jfc_batch_destroy.argtypes = [VP]
        L.jfc_batch_destroy.restype = None
        L.jfc_batch_add.argtypes = [VP, VP]
        L.jfc_batch_clear.argtypes = [VP]
        L.jfc_batch_size.argtypes = [VP]
        L.jfc_batch_solve.argtypes = [VP, ctypes.POINTER(Stats)]
        L.jfc_batch_autotune.argtypes = [VP, ctypes.POINTER(Params)]
        L.jfc_server_create.argtypes = [VP, ctypes.c_size_t, ctypes.c_int, ctypes.POINTER(VP)]
        L.jfc_server_destroy.argtypes = [VP]
        L.jfc_server_destroy.restype = None
        L.jfc_server_submit.argtypes = [VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, VP,
                                        ctypes.c_int, U8P, ctypes.POINTER(Model), ctypes.POINTER(ctypes.c_int)]
        L.jfc_server_edit.argtypes = [VP, ctypes.c_int, U32P, U8P, ctypes.c_size_t]
        L.jfc_server_wait.argtypes = [VP, ctypes.c_int, ctypes.c_int, ctypes.POINTER(RequestInfo)]
        L.jfc_server_read_labels.argtypes = [VP, ctypes.c_int, U8P]
        L.jfc_server_close.argtypes = [VP, ctypes.c_int]
        L.jfc_server_cancel.argtypes = [VP, ctypes.c_int]
        L.jfc_server_get_stats.argtypes = [VP, ctypes.POINTER(ServerStats)]
        L.jfc_graph_compute_tag.argtypes = [VP, U8P, U8P]
        L.jfc_stroke_to_seeds.argtypes = [ctypes.c_int, VP, ctypes.POINTER(View), ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, VP, VP, ctypes.c_int, VP, ctypes.c_uint8, VP]
        L.jfc_energy_device.argtypes = [ctypes.c_int, VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        VP, ctypes.POINTER(VP), VP, ctypes.POINTER(ctypes.c_int64),
                                        ctypes.POINTER(ctypes.c_int64)]
        CP = ctypes.c_char_p
        L.jfc_read_dat.argtypes = [CP, ctypes.POINTER(VolumeInfo)]
        L.jfc_write_dat.argtypes = [CP, ctypes.POINTER(VolumeInfo)]
        L.jfc_read_raw.argtypes = [CP, ctypes.POINTER(VolumeInfo), ctypes.POINTER(ctypes.c_float)]
        L.jfc_load_graph_files.argtypes = [CP] + [ctypes.c_int] * 4 + [I32P, ctypes.POINTER(I32P)]
        L.jfc_save_graph_files.argtypes = [CP] + [ctypes.c_int] * 4 + [I32P, ctypes.POINTER(I32P)]
        L.jfc_read_cut.argtypes = [CP, ctypes.c_size_t, U8P, U8P]
        L.jfc_write_cut.argtypes = [CP, ctypes.c_size_t, U8P, U8P]
        L.jfc_read_mfi_info.argtypes = [CP, ctypes.POINTER(MfiInfo)]
        L.jfc_load_mfi.argtypes = [CP, I32P, ctypes.POINTER(I32P), ctypes.POINTER(ctypes.c_int64), U8P]
        L.jfc_save_mfi.argtypes = [CP] + [ctypes.c_int] * 4 + [I32P, ctypes.POINTER(I32P), ctypes.c_int64, U8P]
        _LIB = L
    return _LIB


def lib():
    return _lib()


def _check(rc, where):
    if rc != OK:
        raise JfcError(rc, where)


def _p(a, t):
    return a.ctypes.data_as(t)


def kernel_launches():
    return int(_lib().jfc_kernel_launches())


def default_params(**kw):
    p = Params()
    _lib().jfc_default_params(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, int(v))
    return p


def default_model(**kw):
    m = Model()
    _lib().jfc_default_model(ctypes.byref(m))
    for k, v in kw.items():
        setattr(m, k, int(v))
    return m


def model_dict(m):
    return {k: getattr(m, k) for k, _ in Model._fields_}


class Context:
    """One device + stream (QGCWidget::initContext / initOpenCL, QGCWidget.cpp:686-813)."""

    def __init__(self, device=0, **params):
        self.handle = VP()
        self._children = weakref.WeakSet()
        p = default_params(**params)
        _check(_lib().jfc_create(device, ctypes.byref(p), ctypes.byref(self.handle)), "jfc_create")

    def set_params(self, **params):
        p = self.params()
        for k, v in params.items():
            setattr(p, k, int(v))
        _check(_lib().jfc_set_params(self.handle, ctypes.byref(p)), "jfc_set_params")

    def reset_params(self):
        """Back to the library's default schedule (jfc_default_params)."""
        p = default_params()
        _check(_lib().jfc_set_params(self.handle, ctypes.byref(p)), "jfc_set_params")

    def set_stream(self, stream_ptr):
        """Run this context's work on a caller-owned cudaStream_t (int pointer; 0 = own)."""
        _check(_lib().jfc_set_stream(self.handle, VP(stream_ptr or None)), "jfc_set_stream")

    def params(self):
        p = Params()
        _check(_lib().jfc_get_params(self.handle, ctypes.byref(p)), "jfc_get_params")
        return p

    def close(self):
        """Destroy the context; graphs, batches and servers made from it go first."""
        if self.handle:
            for child in list(self._children):
                child.close()
            _lib().jfc_destroy(self.handle)
            self.handle = VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Graph:
    """A 4-connected 2D or 6-connected 3D grid graph resident on the device.

    shape: (H, W) or (D, H, W).  Residual arcs follow the reference channel
    order (+x, +y, -y, -x) / (+x, +y, +z, -z, -y, -x)."""

    def __init__(self, ctx, shape):
        self.ctx = ctx
        self.shape = tuple(int(s) for s in shape)
        if len(self.shape) == 2:
            self.dims, (self.h, self.w), self.d, self.conn = 2, self.shape, 1, 4
        else:
            self.dims, (self.d, self.h, self.w), self.conn = 3, self.shape, 6
        self.n = self.w * self.h * self.d
        self.handle = VP()
        _check(_lib().jfc_graph_create_grid(ctx.handle, self.dims, self.w, self.h, self.d, self.conn,
                                            ctypes.byref(self.handle)), "jfc_graph_create_grid")
        ctx._children.add(self)

    # -- build (slotModelClicked: computeCapacity + kmeans + computeExcessFlowLazy)
    def build_from_image(self, img, seeds, pixfmt, model=None):
        img = np.ascontiguousarray(img)
        seeds = np.ascontiguousarray(seeds, dtype=np.uint8)
        if seeds.size != self.n:
            raise ValueError("seeds size mismatch")
        m = model if isinstance(model, Model) else default_model(**(model or {}))
        _check(_lib().jfc_graph_build_from_image(self.handle, img.ctypes.data_as(VP), int(pixfmt),
                                                 _p(seeds, U8P), ctypes.byref(m)), "jfc_graph_build_from_image")

    slotModelClicked = build_from_image

    def build_from_device(self, d_img_ptr, d_seeds_ptr, pixfmt, model=None):
        m = model if isinstance(model, Model) else default_model(**(model or {}))
        _check(_lib().jfc_graph_build_from_device(self.handle, VP(d_img_ptr), int(pixfmt), VP(d_seeds_ptr),
                                                  ctypes.byref(m)), "jfc_graph_build_from_device")

    # -- explicit graph (slotLoadGraphClicked: .ef / .c1 / .c2)
    def set(self, excess, caps, flow_offset=0):
        e = np.ascontiguousarray(excess, dtype=np.int32).ravel()
        cs = [np.ascontiguousarray(c, dtype=np.int32).ravel() for c in caps]
        if len(cs) != self.conn or e.size != self.n or any(c.size != self.n for c in cs):
            raise ValueError("graph arrays do not match the grid")
        P = (I32P * self.conn)(*[_p(c, I32P) for c in cs])
        _check(_lib().jfc_graph_set(self.handle, _p(e, I32P), P, int(flow_offset)), "jfc_graph_set")

    slotLoadGraphClicked = set

    def tag(self, seeds=None):
        """Object nodes connected to a foreground seed (the reference's tag pass)."""
        out = np.empty(self.n, np.uint8)
        sp = None if seeds is None else np.ascontiguousarray(seeds, np.uint8).ravel()
        _check(_lib().jfc_graph_compute_tag(self.handle, None if sp is None else _p(sp, U8P), _p(out, U8P)),
               "jfc_graph_compute_tag")
        return out.reshape(self.shape)

    def load_files(self, base):
        """Load <base>.ef/.c1/.c2 (the reference's graph files) into this grid."""
        e, caps = load_graph_files(base, self.shape)
        self.set(e, caps, 0)

    def load_mfi(self, path):
        """Load a GridCut-benchmark .mfi instance; returns its recorded max-flow."""
        info, e, caps, off, _ = load_mfi(path)
        if tuple(info.shape) != tuple(self.shape):
            raise ValueError("MFI shape %s does not match the grid %s" % (info.shape, self.shape))
        self.set(e, caps, off)
        return info.maxflow

    def set_device(self, d_excess, d_caps, flow_offset=0):
        P = (VP * self.conn)(*[VP(p) for p in d_caps])
        _check(_lib().jfc_graph_set_device(self.handle, VP(d_excess), P, int(flow_offset)),
               "jfc_graph_set_device")

    # -- solve (slotCutClicked)
    def solve(self):
        st = Stats()
        rc = _lib().jfc_solve(self.handle, ctypes.byref(st))
        _check(rc, "jfc_solve")
        return st

    slotCutClicked = solve

    def flow(self):
        f = ctypes.c_int64()
        _check(_lib().jfc_get_flow(self.handle, ctypes.byref(f)), "jfc_get_flow")
        return f.value

    def labels(self):
        out = np.empty(self.n, np.uint8)
        _check(_lib().jfc_read_labels(self.handle, _p(out, U8P)), "jfc_read_labels")
        return out.reshape(self.shape)

    def read_labels_device(self, d_out_ptr):
        _check(_lib().jfc_read_labels_device(self.handle, VP(d_out_ptr)), "jfc_read_labels_device")

    def state(self):
        e = np.empty(self.n, np.int32)
        h = np.empty(self.n, np.int32)
        r = [np.empty(self.n, np.int32) for _ in range(self.conn)]
        P = (I32P * self.conn)(*[_p(c, I32P) for c in r])
        _check(_lib().jfc_graph_get_state(self.handle, _p(e, I32P), P, _p(h, I32P)), "jfc_graph_get_state")
        return e, r, h

    # -- warm edits
    def edit_tlinks(self, idx, dcs, dct):
        idx = np.ascontiguousarray(idx, dtype=np.uint32)
        dcs = np.ascontiguousarray(dcs, dtype=np.int32)
        dct = np.ascontiguousarray(dct, dtype=np.int32)
        _check(_lib().jfc_edit_tlinks(self.handle, _p(idx, U32P), _p(dcs, I32P), _p(dct, I32P), idx.size),
               "jfc_edit_tlinks")

    def edit_seeds(self, idx, new_seed):
        idx = np.ascontiguousarray(idx, dtype=np.uint32)
        ns = np.ascontiguousarray(new_seed, dtype=np.uint8)
        _check(_lib().jfc_graph_edit_seeds(self.handle, _p(idx, U32P), _p(ns, U8P), idx.size),
               "jfc_graph_edit_seeds")

    def close(self):
        if self.handle:
            _lib().jfc_graph_destroy(self.handle)
            self.handle = VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_grid2d_noalloc(w, h, d_excess, d_caps, d_labels, flow_offset=0, device=0, stream=0, params=None):
    """2D solve that allocates nothing (fixed device working set, grids up to
    524,288 padded nodes).  d_excess, d_caps[4], d_labels are device pointers
    (ints); returns the int64 max-flow."""
    P = (VP * 4)(*[VP(int(p)) for p in d_caps])
    f = ctypes.c_int64()
    _check(_lib().jfc_solve_grid2d_noalloc(int(device), VP(stream or None),
                                           ctypes.byref(params) if params is not None else None,
                                           int(w), int(h), VP(int(d_excess)), P, int(flow_offset),
                                           VP(int(d_labels)), ctypes.byref(f)), "jfc_solve_grid2d_noalloc")
    return f.value


class Batch:
    """Many independent grids solved together (one persistent launch per phase)."""

    def __init__(self, ctx):
        self.ctx = ctx
        self.handle = VP()
        self.graphs = []
        _check(_lib().jfc_batch_create(ctx.handle, ctypes.byref(self.handle)), "jfc_batch_create")
        ctx._children.add(self)

    def add(self, g):
        _check(_lib().jfc_batch_add(self.handle, g.handle), "jfc_batch_add")
        self.graphs.append(g)

    def clear(self):
        _check(_lib().jfc_batch_clear(self.handle), "jfc_batch_clear")
        self.graphs = []

    def solve(self):
        st = (Stats * max(1, len(self.graphs)))()
        rc = _lib().jfc_batch_solve(self.handle, st)
        _check(rc, "jfc_batch_solve")
        return list(st)[:len(self.graphs)]

    def autotune(self):
        p = Params()
        _check(_lib().jfc_batch_autotune(self.handle, ctypes.byref(p)), "jfc_batch_autotune")
        return p

    def close(self):
        if self.handle:
            _lib().jfc_batch_destroy(self.handle)
            self.handle = VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching server with HBM-budget admission and warm edits."""

    def __init__(self, ctx, hbm_budget_bytes, max_slots=64):
        self.ctx = ctx
        self.handle = VP()
        _check(_lib().jfc_server_create(ctx.handle, int(hbm_budget_bytes), int(max_slots),
                                        ctypes.byref(self.handle)), "jfc_server_create")
        ctx._children.add(self)

    def submit(self, img, seeds, pixfmt, model=None):
        img = np.ascontiguousarray(img)
        seeds = np.ascontiguousarray(seeds, dtype=np.uint8)
        if seeds.ndim == 2:
            dims, (h, w), d = 2, seeds.shape, 1
        else:
            dims, (d, h, w) = 3, seeds.shape
        m = model if isinstance(model, Model) else default_model(**(model or {}))
        sid = ctypes.c_int(-1)
        _check(_lib().jfc_server_submit(self.handle, dims, w, h, d, img.ctypes.data_as(VP), int(pixfmt),
                                        _p(seeds, U8P), ctypes.byref(m), ctypes.byref(sid)), "jfc_server_submit")
        return sid.value

    def edit(self, sid, idx, new_seed):
        idx = np.ascontiguousarray(idx, dtype=np.uint32)
        ns = np.ascontiguousarray(new_seed, dtype=np.uint8)
        _check(_lib().jfc_server_edit(self.handle, int(sid), _p(idx, U32P), _p(ns, U8P), idx.size),
               "jfc_server_edit")

    def wait(self, sid, timeout_ms=-1):
        """Wait for the session's latest request; returns its RequestInfo (a
        failed or cancelled request is reported in info.status, not raised)."""
        info = RequestInfo()
        info.status = -1
        rc = _lib().jfc_server_wait(self.handle, int(sid), int(timeout_ms), ctypes.byref(info))
        if rc != OK and info.status != rc:
            _check(rc, "jfc_server_wait")
        return info

    def stats(self):
        st = ServerStats()
        _check(_lib().jfc_server_get_stats(self.handle, ctypes.byref(st)), "jfc_server_get_stats")
        return st.as_dict()

    def labels(self, sid, shape):
        out = np.empty(int(np.prod(shape)), np.uint8)
        _check(_lib().jfc_server_read_labels(self.handle, int(sid), _p(out, U8P)), "jfc_server_read_labels")
        return out.reshape(shape)

    def close_session(self, sid):
        _check(_lib().jfc_server_close(self.handle, int(sid)), "jfc_server_close")

    def cancel(self, sid):
        _check(_lib().jfc_server_cancel(self.handle, int(sid)), "jfc_server_cancel")

    def close(self):
        if self.handle:
            _lib().jfc_server_destroy(self.handle)
            self.handle = VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def energy_device(device, shape, d_excess, d_caps, d_labels, stream=0):
    """Energy (data, smooth) of a labelling over dense device arrays (int
    pointers): the reference's post-solve energy check."""
    dims, w, h, d = _dims(shape)
    data, smooth = ctypes.c_int64(0), ctypes.c_int64(0)
    P = (VP * len(d_caps))(*[VP(p) for p in d_caps])
    _check(_lib().jfc_energy_device(int(device), VP(stream or None), dims, w, h, d, VP(d_excess), P, VP(d_labels),
                                    ctypes.byref(data), ctypes.byref(smooth)), "jfc_energy_device")
    return data.value, smooth.value


def stroke_to_seeds(device, view, shape, d_volume, d_tf, tf_size, d_mask, label, d_seeds, stream=0):
    """Mark the voxels a stroke sees through the volume (device pointers; shape (d, h, w))."""
    d, h, w = (int(v) for v in shape)
    _check(_lib().jfc_stroke_to_seeds(int(device), VP(stream or None), ctypes.byref(view), w, h, d, VP(d_volume),
                                      VP(d_tf), int(tf_size), VP(d_mask), int(label), VP(d_seeds)),
           "jfc_stroke_to_seeds")


# ---------------------------------------------------------------- data files
def _dims(shape):
    if len(shape) == 2:
        return 2, int(shape[1]), int(shape[0]), 1
    return 3, int(shape[2]), int(shape[1]), int(shape[0])


def _b(path):
    return os.fsencode(path)


def read_dat(path):
    """Volume header (.dat) -> VolumeInfo."""
    info = VolumeInfo()
    _check(_lib().jfc_read_dat(_b(path), ctypes.byref(info)), "jfc_read_dat")
    return info


def write_dat(path, info):
    _check(_lib().jfc_write_dat(_b(path), ctypes.byref(info)), "jfc_write_dat")


def read_raw(path, info):
    """Samples of a .raw volume as float32, shape (h, w) or (d, h, w)."""
    out = np.empty(info.w * info.h * info.d, np.float32)
    _check(_lib().jfc_read_raw(_b(path), ctypes.byref(info), out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
           "jfc_read_raw")
    return out.reshape((info.h, info.w) if info.d == 1 else (info.d, info.h, info.w))


def load_graph_files(base, shape):
    """<base>.ef/.c1/.c2 -> (excess, caps) in the solver's channel order."""
    dims, w, h, d = _dims(shape)
    n = w * h * d
    e = np.empty(n, np.int32)
    caps = [np.empty(n, np.int32) for _ in range(4 if dims == 2 else 6)]
    P = (I32P * len(caps))(*[_p(c, I32P) for c in caps])
    _check(_lib().jfc_load_graph_files(_b(base), dims, w, h, d, _p(e, I32P), P), "jfc_load_graph_files")
    return e.reshape(shape), [c.reshape(shape) for c in caps]


def save_graph_files(base, excess, caps):
    dims, w, h, d = _dims(np.shape(excess))
    e = np.ascontiguousarray(excess, np.int32).ravel()
    cs = [np.ascontiguousarray(c, np.int32).ravel() for c in caps]
    P = (I32P * len(cs))(*[_p(c, I32P) for c in cs])
    _check(_lib().jfc_save_graph_files(_b(base), dims, w, h, d, _p(e, I32P), P), "jfc_save_graph_files")


def read_cut(path, shape):
    """.cut -> (seeds JFC_SEED_*, labels 1 = object)."""
    n = int(np.prod(shape))
    seeds = np.empty(n, np.uint8)
    labels = np.empty(n, np.uint8)
    _check(_lib().jfc_read_cut(_b(path), n, _p(seeds, U8P), _p(labels, U8P)), "jfc_read_cut")
    return seeds.reshape(shape), labels.reshape(shape)


def write_cut(path, seeds, labels):
    s_ = None if seeds is None else np.ascontiguousarray(seeds, np.uint8).ravel()
    l_ = None if labels is None else np.ascontiguousarray(labels, np.uint8).ravel()
    n = (s_ if s_ is not None else l_).size
    _check(_lib().jfc_write_cut(_b(path), n, None if s_ is None else _p(s_, U8P),
                                None if l_ is None else _p(l_, U8P)), "jfc_write_cut")


def read_mfi_info(path):
    info = MfiInfo()
    _check(_lib().jfc_read_mfi_info(_b(path), ctypes.byref(info)), "jfc_read_mfi_info")
    return info


def load_mfi(path):
    """.mfi -> (info, excess, caps, flow_offset, mask)."""
    info = read_mfi_info(path)
    shape = info.shape
    n = int(np.prod(shape))
    e = np.empty(n, np.int32)
    caps = [np.empty(n, np.int32) for _ in range(info.conn)]
    mask = np.empty(n, np.uint8)
    off = ctypes.c_int64(0)
    P = (I32P * len(caps))(*[_p(c, I32P) for c in caps])
    _check(_lib().jfc_load_mfi(_b(path), _p(e, I32P), P, ctypes.byref(off), _p(mask, U8P)), "jfc_load_mfi")
    return info, e.reshape(shape), [c.reshape(shape) for c in caps], off.value, mask.reshape(shape)


def save_mfi(path, excess, caps, maxflow, mask=None):
    dims, w, h, d = _dims(np.shape(excess))
    e = np.ascontiguousarray(excess, np.int32).ravel()
    cs = [np.ascontiguousarray(c, np.int32).ravel() for c in caps]
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8).ravel()
    P = (I32P * len(cs))(*[_p(c, I32P) for c in cs])
    _check(_lib().jfc_save_mfi(_b(path), dims, w, h, d, _p(e, I32P), P, int(maxflow),
                               None if m is None else _p(m, U8P)), "jfc_save_mfi")


def graph_bytes(shape):
    """Device bytes of a grid graph's resident state (shape (h, w) or (d, h, w))."""
    if len(shape) == 2:
        return int(_lib().jfc_graph_bytes(2, int(shape[1]), int(shape[0]), 1))
    return int(_lib().jfc_graph_bytes(3, int(shape[2]), int(shape[1]), int(shape[0])))
