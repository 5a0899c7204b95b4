"""Seeded synthetic inputs (images, videos, volumes, stroke edits) over
oracle/libsynthetic.so.

INPUT GENERATION ONLY: used by tests/, __graft_entry__.smoke() and bench.py
before any timed region, by both bench arms alike, so that the reference arm
builds the same graph from the same bytes without loading the product
library.  Nothing on the solve path imports it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
U8P = ctypes.POINTER(ctypes.c_uint8)
U32P = ctypes.POINTER(ctypes.c_uint32)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "libsynthetic.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.run(["make", "-s", "-f", os.path.join(HERE, "Makefile"), path], check=True, cwd=HERE)
        L = ctypes.CDLL(path)
        L.syn_gray_ellipse.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_int, U8P, U8P]
        L.syn_rgb_ellipses.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, U8P, U8P]
        L.syn_rgb_video.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64, U8P, U8P]
        L.syn_i16_phantom.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_int16), U8P]
        L.syn_stroke.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                 ctypes.c_size_t, ctypes.c_uint8, U32P, U8P, ctypes.POINTER(ctypes.c_size_t)]
        _LIB = L
    return _LIB


def _ok(rc, what):
    if rc != 0:
        raise ValueError("%s: invalid arguments" % what)


def _p(a, t):
    return a.ctypes.data_as(t)


def gray_ellipse(w, h, seed=0, noise_sigma=20):
    """8-bit grayscale: blurred ellipse (fg mean 170) on a mean-80 background,
    N(0, noise_sigma) noise; a fg and a bg line stroke."""
    img = np.empty((h, w), np.uint8)
    seeds = np.empty((h, w), np.uint8)
    _ok(lib().syn_gray_ellipse(w, h, seed, noise_sigma, _p(img, U8P), _p(seeds, U8P)), "gray_ellipse")
    return img, seeds


def rgb_ellipses(w, h, seed=0, n_ellipses=20, noise_sigma=15, stroke_permille_x10=50):
    """RGB: n random overlapping ellipses with U(0,255)^3 colour means plus
    N(0, noise_sigma) noise; random strokes over stroke_permille_x10 / 10000
    of the pixels."""
    img = np.empty((h, w, 3), np.uint8)
    seeds = np.empty((h, w), np.uint8)
    _ok(lib().syn_rgb_ellipses(w, h, seed, n_ellipses, noise_sigma, stroke_permille_x10,
                               _p(img, U8P), _p(seeds, U8P)), "rgb_ellipses")
    return img, seeds


def rgb_video(w, h, frames, seed=0):
    """RGB video: an ellipse moving 4 px per frame over seeded value noise;
    strokes on the first and last frames."""
    img = np.empty((frames, h, w, 3), np.uint8)
    seeds = np.empty((frames, h, w), np.uint8)
    _ok(lib().syn_rgb_video(w, h, frames, seed, _p(img, U8P), _p(seeds, U8P)), "rgb_video")
    return img, seeds


def i16_phantom(w, h, d, seed=0, noise_sigma=10):
    """int16 volume: a sphere and a tube with N(0, noise_sigma) noise; a fg
    seed cube in the sphere and a bg cube in a corner."""
    img = np.empty((d, h, w), np.int16)
    seeds = np.empty((d, h, w), np.uint8)
    _ok(lib().syn_i16_phantom(w, h, d, seed, noise_sigma, img.ctypes.data_as(ctypes.POINTER(ctypes.c_int16)),
                              _p(seeds, U8P)), "i16_phantom")
    return img, seeds


def stroke(shape, seed, n, label):
    """A random-walk stroke over up to n distinct nodes of a (h, w) or
    (d, h, w) grid: (node indices uint32, new seed bytes)."""
    if len(shape) == 2:
        dims, (h, w), d = 2, shape, 1
    else:
        dims, (d, h, w) = 3, shape
    idx = np.empty(n, np.uint32)
    ns = np.empty(n, np.uint8)
    k = ctypes.c_size_t(0)
    _ok(lib().syn_stroke(dims, w, h, d, seed, n, label, _p(idx, U32P), _p(ns, U8P), ctypes.byref(k)), "stroke")
    return idx[:k.value].copy(), ns[:k.value].copy()
