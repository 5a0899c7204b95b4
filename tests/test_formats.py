"""The reference's data files (.dat, .raw, .ef/.c1/.c2, .cut, .mfi): host-side
readers and writers of libjfcut.so, no GPU.  Round trips on the golden
fixtures; where the reference tree is present, the readers are checked against
the reference's own files byte for byte (the fixtures were made from them)."""
import os

import numpy as np
import pytest

import jfcut
import oracle
from conftest import FIXTURES, load_fixture, random_grid

# the reference checkout, when JFC_REFERENCE names it: its data files are read directly
REF_DATA = os.path.join(os.environ.get("JFC_REFERENCE", ""), "src", "QVisualizer", "data")
have_ref = bool(os.environ.get("JFC_REFERENCE")) and os.path.isdir(REF_DATA)


def test_graph_files_round_trip(tmp_path):
    shape, e, caps, flow, _ = load_fixture("flower")
    base = str(tmp_path / "g")
    jfcut.save_graph_files(base, e.reshape(shape), [c.reshape(shape) for c in caps])
    assert os.path.getsize(base + ".ef") == e.size * 4
    assert os.path.getsize(base + ".c1") == e.size * 4    # ushort2 per node
    e2, c2 = jfcut.load_graph_files(base, shape)
    assert np.array_equal(e2.ravel(), e)
    for a, b in zip(c2, caps):
        assert np.array_equal(a.ravel(), b)


def test_graph_files_3d_round_trip(tmp_path):
    rng = np.random.default_rng(5)
    shape = (5, 7, 9)
    e, caps = random_grid(shape, rng, cap_max=255)
    base = str(tmp_path / "v")
    jfcut.save_graph_files(base, e.reshape(shape), [c.reshape(shape) for c in caps])
    assert os.path.getsize(base + ".c1") == e.size * 4    # uchar4 per node
    e2, c2 = jfcut.load_graph_files(base, shape)
    assert np.array_equal(e2.ravel(), e)
    assert all(np.array_equal(a.ravel(), b) for a, b in zip(c2, caps))


def test_graph_files_reject_wide_capacities(tmp_path):
    rng = np.random.default_rng(6)
    shape = (4, 5, 6)
    e, caps = random_grid(shape, rng, cap_max=255)
    caps[0][3] = 256                       # does not fit the 3D uchar channel
    with pytest.raises(jfcut.JfcError) as ex:
        jfcut.save_graph_files(str(tmp_path / "w"), e.reshape(shape), [c.reshape(shape) for c in caps])
    assert ex.value.code == jfcut.ERR_INVALID_ARG


def test_missing_files_are_io_errors(tmp_path):
    with pytest.raises(jfcut.JfcError) as ex:
        jfcut.load_graph_files(str(tmp_path / "nothing"), (4, 4))
    assert ex.value.code == jfcut.ERR_IO
    with pytest.raises(jfcut.JfcError) as ex:
        jfcut.read_dat(str(tmp_path / "nothing.dat"))
    assert ex.value.code == jfcut.ERR_IO
    bad = tmp_path / "bad.mfi"
    bad.write_bytes(b"XYZ" + bytes(100))
    with pytest.raises(jfcut.JfcError) as ex:
        jfcut.read_mfi_info(str(bad))
    assert ex.value.code == jfcut.ERR_IO


def test_cut_round_trip(tmp_path):
    rng = np.random.default_rng(7)
    seeds = rng.integers(0, 3, 1000).astype(np.uint8)
    labels = rng.integers(0, 2, 1000).astype(np.uint8)
    p = str(tmp_path / "x.cut")
    jfcut.write_cut(p, seeds, labels)
    raw = np.fromfile(p, np.uint8).reshape(-1, 4)
    assert np.array_equal(raw[:, 0], seeds == 1) and np.array_equal(raw[:, 1], seeds == 2)
    assert np.array_equal(raw[:, 2], labels) and not raw[:, 3].any()
    s2, l2 = jfcut.read_cut(p, (1000,))
    assert np.array_equal(s2, seeds) and np.array_equal(l2, labels)


def test_dat_round_trip(tmp_path):
    info = jfcut.VolumeInfo()
    info.object_file = b"vol.raw"
    info.w, info.h, info.d = 12, 10, 3
    info.format = jfcut.FMT_SHORT
    info.big_endian = 1
    info.thickness[0], info.thickness[1], info.thickness[2] = 1.0, 1.0, 2.5
    p = str(tmp_path / "vol.raw.dat")
    jfcut.write_dat(p, info)
    r = jfcut.read_dat(p)
    assert (r.object_file, r.w, r.h, r.d, r.format, r.big_endian) == (b"vol.raw", 12, 10, 3, jfcut.FMT_SHORT, 1)
    assert abs(r.thickness[2] - 2.5) < 1e-6
    vals = np.arange(-180, 180, dtype=np.int16)
    vals.astype(">i2").tofile(str(tmp_path / "vol.raw"))
    got = jfcut.read_raw(str(tmp_path / "vol.raw"), r)
    assert got.shape == (3, 10, 12) and np.array_equal(got.ravel(), vals.astype(np.float32))


@pytest.mark.parametrize("shape,cap_max", [((37, 53), 100), ((40, 30), 70000), ((6, 9, 11), 200), ((5, 6, 7), 300)])
def test_mfi_round_trip(tmp_path, shape, cap_max):
    rng = np.random.default_rng(8)
    e, caps = random_grid(shape, rng, cap_max=cap_max)
    mask = rng.integers(0, 5, e.size).astype(np.uint8)
    p = str(tmp_path / "g.mfi")
    jfcut.save_mfi(p, e.reshape(shape), [c.reshape(shape) for c in caps], 12345, mask)
    info, e2, c2, off, m2 = jfcut.load_mfi(p)
    assert tuple(info.shape) == tuple(shape) and info.maxflow == 12345
    assert info.conn == (4 if len(shape) == 2 else 6)
    # the reference's neighbour type (uint16 2D / uint8 3D) unless a capacity is wider
    small = 1 if len(shape) == 2 else 0
    assert info.type_neighbor == (small if cap_max <= (65535 if small else 255) else 2)
    assert info.active_count == int((e >= 0).sum())
    assert off == 0                        # terminals stored as max(e, 0) / max(-e, 0)
    assert np.array_equal(e2.ravel(), e) and np.array_equal(m2.ravel(), mask)
    assert all(np.array_equal(a.ravel(), b) for a, b in zip(c2, caps))


def test_mfi_flow_matches_oracle(tmp_path):
    """A written instance carries its max-flow; loading it back and solving
    with the oracle reproduces the recorded value (benchmark semantics:
    cap_neighbor[dir][i] is the arc from node i towards dir)."""
    rng = np.random.default_rng(9)
    shape = (30, 41)
    e, caps = random_grid(shape, rng)
    f, _, _, _ = oracle.maxflow(shape, e, caps)
    p = str(tmp_path / "f.mfi")
    jfcut.save_mfi(p, e.reshape(shape), [c.reshape(shape) for c in caps], f)
    info, e2, c2, off, _ = jfcut.load_mfi(p)
    f2, _, _, _ = oracle.maxflow(shape, e2.ravel(), [c.ravel() for c in c2])
    assert f2 + off == info.maxflow == f
    if oracle.ref_available():
        fb, _, _ = oracle.bk_maxflow(shape, e2.ravel(), [c.ravel() for c in c2])
        assert fb + off == f


@pytest.mark.skipif(not have_ref, reason="reference data files not present")
@pytest.mark.parametrize("name", FIXTURES)
def test_readers_match_reference_files(name):
    """The readers decode the reference's own files into exactly the golden
    fixture (which tests/golden/make_golden.py made from the same bytes)."""
    shape, e, caps, flow, ref_object = load_fixture(name)
    base = os.path.join(REF_DATA, name, "normalized_%s.raw" % name)
    info = jfcut.read_dat(base + ".dat")
    assert (info.h, info.w, info.d) == (shape[0], shape[1], 1)
    assert info.object_file.decode() == "normalized_%s.raw" % name and info.format == jfcut.FMT_FLOAT
    e2, c2 = jfcut.load_graph_files(base, shape)
    assert np.array_equal(e2.ravel(), e)
    assert all(np.array_equal(a.ravel(), b) for a, b in zip(c2, caps))
    _, labels = jfcut.read_cut(base + ".cut", shape)
    assert np.array_equal(labels.ravel(), ref_object)
    raw = jfcut.read_raw(os.path.join(REF_DATA, name, info.object_file.decode()), info)
    assert raw.shape == shape and 0.0 <= raw.min() and raw.max() <= 1.0
