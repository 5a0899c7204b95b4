"""The seeded synthetic inputs (oracle/synthetic.cpp) on the CPU: they are
deterministic, have the shapes and seed coverage the workloads name, and
reproduce the recorded bytes (tests/golden/synthetic_hashes.json holds the
SHA-256 prefixes of the images, videos, volumes and strokes the tests and the
bench use, so the plain, video, batched and serving inputs stay the same
bytes wherever they are generated)."""
import hashlib
import json
import os

import numpy as np
import pytest

import synthetic
from conftest import GOLDEN


def _hash(*arrs):
    m = hashlib.sha256()
    for a in arrs:
        m.update(np.ascontiguousarray(a).tobytes())
    return m.hexdigest()[:32]


def _make(key):
    kind, *a = key.split()
    if kind == "gray_ellipse":
        return synthetic.gray_ellipse(int(a[0]), int(a[1]), seed=int(a[2]))
    if kind == "rgb_ellipses":
        return synthetic.rgb_ellipses(int(a[0]), int(a[1]), seed=int(a[2]))
    if kind == "rgb_video":
        return synthetic.rgb_video(int(a[0]), int(a[1]), int(a[2]), seed=int(a[3]))
    if kind == "i16_phantom":
        return synthetic.i16_phantom(int(a[0]), int(a[1]), int(a[2]), seed=int(a[3]))
    shape = tuple(int(x) for x in a[0].split("x"))
    return synthetic.stroke(shape, seed=int(a[1]), n=int(a[2]), label=int(a[3]))


RECORDED = json.load(open(os.path.join(GOLDEN, "synthetic_hashes.json")))


@pytest.mark.parametrize("key", sorted(RECORDED))
def test_recorded_bytes(key):
    assert _hash(*_make(key)) == RECORDED[key]


def test_deterministic_and_shaped():
    a = synthetic.rgb_ellipses(301, 197, seed=5)
    b = synthetic.rgb_ellipses(301, 197, seed=5)
    c = synthetic.rgb_ellipses(301, 197, seed=6)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert not np.array_equal(a[0], c[0])
    img, seeds = a
    frac = (seeds > 0).mean()
    assert 0.004 < frac < 0.02 and (seeds == 1).any() and (seeds == 2).any()
    g, s = synthetic.gray_ellipse(128, 96, seed=1)
    assert g.dtype == np.uint8 and (s == 1).any() and (s == 2).any()
    v, vs = synthetic.rgb_video(64, 48, 6, seed=2)
    assert v.shape == (6, 48, 64, 3) and (vs[0] > 0).any() and (vs[5] > 0).any() and not (vs[2] > 0).any()
    p, ps = synthetic.i16_phantom(24, 24, 24, seed=3)
    assert p.dtype == np.int16 and (ps == 1).any() and (ps == 2).any()
    idx, ns = synthetic.stroke((40, 50), seed=9, n=100, label=1)
    assert len(np.unique(idx)) == len(idx) > 50 and (ns == 1).all() and idx.max() < 2000


def test_invalid_arguments_raise():
    with pytest.raises(ValueError):
        synthetic.rgb_ellipses(4, 4)
