"""Generate tests/golden/*.npz from the graphs that ship with the reference.

Reads src/QVisualizer/data/{flower,person,sponge}/normalized_*.raw.{ef,c1,c2,cut}
(int32 net excess, ushort2 c1 = (+x,+y), ushort2 c2 = (-y,-x), 4-byte cl_cut;
formats per QGCWidget.cpp:2631-2736 and QGCSetting.h:31-51) and stores them
compressed together with the published max-flow values
(latex/sources/section-5-results.tex:31-41) and the reference GPU's cut
(cl_cut.object, non-zero only in flower's file).

Run in a container that has the reference tree:
    python tests/golden/make_golden.py <reference checkout>     (or JFC_REFERENCE=<checkout>)
"""
import os
import sys

import numpy as np

FIXTURES = {
    # name: (width, height, published max-flow)
    "flower": (600, 450, 1208089),
    "person": (600, 450, 880461),
    "sponge": (640, 480, 343591),
}


def main(ref_root):
    out_dir = os.path.dirname(os.path.abspath(__file__))
    for name, (w, h, flow) in FIXTURES.items():
        p = os.path.join(ref_root, "src", "QVisualizer", "data", name, "normalized_%s.raw" % name)
        ef = np.fromfile(p + ".ef", np.int32)
        c1 = np.fromfile(p + ".c1", np.uint16).reshape(-1, 2)
        c2 = np.fromfile(p + ".c2", np.uint16).reshape(-1, 2)
        cut = np.fromfile(p + ".cut", np.int8).reshape(-1, 4)
        assert ef.size == w * h
        px, py = c1[:, 0].reshape(h, w), c1[:, 1].reshape(h, w)
        my, mx = c2[:, 0].reshape(h, w), c2[:, 1].reshape(h, w)
        assert (px[:, :-1] == mx[:, 1:]).all() and (py[:-1] == my[1:]).all()
        assert (px[:, -1] == 0).all() and (mx[:, 0] == 0).all()
        assert (py[-1] == 0).all() and (my[0] == 0).all()
        np.savez_compressed(
            os.path.join(out_dir, name + ".npz"),
            width=np.int32(w), height=np.int32(h), maxflow=np.int64(flow),
            excess=ef,
            # n-links are symmetric in these files (asserted above), so only the
            # +x and +y channels are stored; -y / -x are the shifted copies.
            caps_px=c1[:, 0].astype(np.uint16),
            caps_py=c1[:, 1].astype(np.uint16),
            ref_object=(cut[:, 2] != 0).astype(np.uint8),
            seeds_fg=(cut[:, 0] != 0).astype(np.uint8),
            seeds_bg=(cut[:, 1] != 0).astype(np.uint8),
        )
        print(name, os.path.getsize(os.path.join(out_dir, name + ".npz")), "bytes")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("JFC_REFERENCE")
    if not root:
        sys.exit("usage: make_golden.py <reference checkout>   (or set JFC_REFERENCE)")
    main(root)
