"""Writes tests/golden/vertex_algos.npz: the vertex products of the
reference's own serial chain (oracle/ref checker build) configured with
useDBSCAN and with useIterative (PixelVertexProducerCUDA's non-default
clusterers) on one seeded PU50 event.  Needs the reference tree; run from the
repository root:

    python tests/golden/make_golden_vertex_algos.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "pixeltrack-standalone_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import build  # noqa: E402
import pixgpu  # noqa: E402
import oracle  # noqa: E402

EVENT = (pixgpu.BASE_SEED + 401, 50)  # (seed, pile-up)
VERTEX_PRODUCTS = ("nVertices", "zv", "wv", "vchi2", "ptv2", "ndof", "sortInd", "idv")


def main():
    build.build_synth()
    if build.build_ref() is None:
        raise SystemExit("the reference sources are needed to regenerate the fixture")
    det = pixgpu.Detector()
    d = tempfile.mkdtemp()
    det.write(d)
    raw = det.event(*EVENT)
    arrays = {"event": np.array(EVENT, dtype=np.float64)}
    for algo, name in ((1, "dbscan"), (2, "iterative")):
        p = oracle.Reference(d, vertex_algo=algo).process(raw, names=list(VERTEX_PRODUCTS))
        for k in VERTEX_PRODUCTS:
            arrays[name + "_" + k] = np.asarray(p[k])
    np.savez_compressed(os.path.join(HERE, "vertex_algos.npz"), **arrays)


if __name__ == "__main__":
    main()
